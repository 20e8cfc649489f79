"""GPU parity: the CUDA path through the C ABI against the oracle.

Every case compares the sorted, deduplicated (offset, id) reports of the
engine with the oracle's restatement of the reference CPU matcher
(code/src/ngap/ngap.cu:2171-2344) on the same seeded input: bit-exact.
"""
import os

import numpy as np
import pytest

import ngap_b200 as nb
from ngap_b200 import workloads as W
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
ALGOS = list(nb.ALGORITHMS)

pytestmark = pytest.mark.gpu


def run_both(engine, anml, data, num_seg, seg_len, group_num=1, depth=0, is_dup=False, **kw):
    nfa = nb.Nfa.from_string(anml)
    groups = nb.Groups(nfa, group_num=group_num)
    tables = nb.Tables(groups, precompute_depth=depth, tile_states=kw.pop("tile_states", 0),
                       tile_mode=kw.pop("tile_mode", "auto"))
    got = engine.match(tables, data[:num_seg * seg_len], num_seg, seg_len, is_dup=is_dup, **kw)
    want, _ = oracle.match(groups.views(), data[:num_seg * seg_len], num_seg, seg_len,
                           is_dup=is_dup)
    return got, want


@pytest.mark.parametrize("algo", ALGOS)
def test_apple_known_answer(engine, algo):
    """README.md:156-186: state 4 reports at offsets 5, 47, 64 and 75."""
    anml = open(os.path.join(GOLD, "apple.anml")).read()
    data = np.fromfile(os.path.join(GOLD, "apple_input.txt"), dtype=np.uint8)
    got, want = run_both(engine, anml, data, 1, len(data), depth=3, algorithm=algo)
    assert [hex(x) for x in got] == ["0x400000005", "0x40000002f", "0x400000040", "0x40000004b"]
    assert np.array_equal(got, want)


@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("num_seg,group_num,depth", [(1, 1, 0), (4, 3, 2), (8, 10, 3)])
def test_literal_set(engine, algo, num_seg, group_num, depth):
    anml, data = W.literal_set(seed=5, input_len=1 << 18, plant_every=1 << 12)
    seg = len(data) // num_seg
    got, want = run_both(engine, anml, data, num_seg, seg, group_num=group_num, depth=depth,
                         algorithm=algo)
    assert len(want) > 10
    assert np.array_equal(got, want)


@pytest.mark.parametrize("algo", ["blockinggroups", "nonblockinggroups", "nonblockingpcgroups",
                                  "nonblockingallgroups", "nonblockingr2groups"])
def test_hamming(engine, algo):
    anml, data = W.hamming_set(seed=7, n_patterns=60, input_len=1 << 18, plant_every=1 << 11)
    got, want = run_both(engine, anml, data, 4, len(data) // 4, group_num=4, depth=3,
                         algorithm=algo)
    assert len(want) > 50
    assert np.array_equal(got, want)


@pytest.mark.parametrize("algo", ["NAPgroups", "nonblockinggroups", "nonblockingallgroups"])
def test_levenshtein_degree_limited(engine, algo):
    anml, data = W.levenshtein_set(seed=8, n_patterns=40, input_len=1 << 17, plant_every=1 << 11)
    got, want = run_both(engine, anml, data, 2, len(data) // 2, group_num=5, depth=2,
                         algorithm=algo)
    assert len(want) > 20
    assert np.array_equal(got, want)


@pytest.mark.parametrize("algo", ["blockinggroups", "nonblockinggroups", "nonblockingallgroups"])
@pytest.mark.parametrize("window", [0, 64])
def test_dotstar_unbounded(engine, algo, window):
    """`.*` states with self-loops make tiles unbounded (one unit per segment,
    carried across windows)."""
    anml, data = W.dotstar_set(seed=9, n_patterns=150, input_len=1 << 17, plant_every=1 << 11)
    got, want = run_both(engine, anml, data, 2, len(data) // 2, group_num=3, depth=3,
                         algorithm=algo, window=window)
    assert len(want) > 20
    assert np.array_equal(got, want)


@pytest.mark.parametrize("depth", [4, 6, -1])
@pytest.mark.parametrize("gen,kw,g", [
    (W.hamming_set, dict(seed=17, n_patterns=40, input_len=1 << 17, plant_every=1 << 10), 3),
    (W.levenshtein_set, dict(seed=18, n_patterns=25, input_len=1 << 16, plant_every=1 << 10), 2),
    (W.dotstar_set, dict(seed=19, n_patterns=60, input_len=1 << 16, plant_every=1 << 10), 2),
    (W.literal_set, dict(seed=20, input_len=1 << 16, plant_every=1 << 10), 1),
])
def test_deep_prefix_tables(engine, gen, kw, g, depth):
    """Class-keyed prefix tables deeper than the reference's 3 levels."""
    anml, data = gen(**kw)
    for algo in ("nonblockingpcgroups", "nonblockingallgroups"):
        got, want = run_both(engine, anml, data, 2, len(data) // 2, group_num=g, depth=depth,
                             algorithm=algo)
        assert len(want) > 0
        assert np.array_equal(got, want), algo


@pytest.mark.parametrize("window,tile_states", [(0, 0), (64, 0), (0, 6000), (97, 6000)])
@pytest.mark.parametrize("algo", ["nonblockingpcgroups", "nonblockingallgroups", "blockinggroups"])
def test_sticky_dotstar(engine, window, tile_states, algo):
    """`.*` states that are not always active: registered per warp when they
    first match (with catch-up of injected positions), more than a warp can
    track with large tiles."""
    anml, data = W.dotstar_set(seed=21, n_patterns=300, lit_lo=2, lit_hi=4, aas_frac=0.0,
                               input_len=1 << 16, plant_every=1 << 9, zipf_s=1.6)
    got, want = run_both(engine, anml, data, 2, len(data) // 2, group_num=2, depth=-1,
                         algorithm=algo, window=window, tile_states=tile_states)
    assert len(want) > 100
    assert np.array_equal(got, want)


def test_sticky_report_and_start_states(engine):
    w = W.AnmlWriter()
    w.ste("a", [ord("x")], ["s"], start="all-input")
    w.ste("s", None, ["s", "b"], symbol_set="*", report=True)        # reporting .*
    w.ste("b", [ord("y")], ["c"])
    w.ste("c", [ord("z")], [], report=True)
    w.ste("t", None, ["t", "d"], symbol_set="*", start="start-of-data")  # .* from the start
    w.ste("d", [ord("q")], [], report=True)
    rng = np.random.default_rng(3)
    data = rng.choice(np.frombuffer(b"xyzqab", dtype=np.uint8), size=5000)
    for algo in ("nonblockingpcgroups", "NAPgroups", "blockinggroups"):
        for window in (0, 50):
            got, want = run_both(engine, w.text(), data, 4, 1250, group_num=2, depth=2,
                                 algorithm=algo, window=window)
            assert np.array_equal(got, want), (algo, window)


@pytest.mark.parametrize("tile_mode,tile_states", [("shared", 0), ("global", 0), ("global", 2500)])
@pytest.mark.parametrize("gen,kw,g,depth", [
    (W.hamming_set, dict(seed=31, n_patterns=80, input_len=1 << 17, plant_every=1 << 10), 4, -1),
    (W.levenshtein_set, dict(seed=32, n_patterns=40, input_len=1 << 16, plant_every=1 << 10), 3, 5),
    (W.dotstar_set, dict(seed=33, n_patterns=80, input_len=1 << 16, plant_every=1 << 10), 2, 3),
    (W.literal_set, dict(seed=34, input_len=1 << 16, plant_every=1 << 10), 2, -1),
])
def test_tile_modes(engine, tile_mode, tile_states, gen, kw, g, depth):
    """Global tiles (CCs of several groups read through L2) and shared-memory
    tiles give the same reports; a state cap splits global tiles across groups."""
    anml, data = gen(**kw)
    for algo in ("nonblockingpcgroups", "blockinggroups", "NAPgroups", "nonblockingallgroups"):
        got, want = run_both(engine, anml, data, 2, len(data) // 2, group_num=g, depth=depth,
                             algorithm=algo, tile_mode=tile_mode, tile_states=tile_states)
        assert len(want) > 0
        assert np.array_equal(got, want), algo


@pytest.mark.parametrize("window,chunk", [(3, 0), (5, 100), (10, 0), (64, 333), (1000, 0)])
@pytest.mark.parametrize("tile_mode", ["shared", "global"])
def test_deferred_window_tail(engine, window, chunk, tile_mode):
    """Deep tables: the last depth - 1 positions of a window are injected from
    the next window's look-behind bytes, also when windows are shorter than that."""
    anml, data = W.hamming_set(seed=35, n_patterns=50, input_len=1 << 15, plant_every=1 << 9)
    for depth in (8, 12):
        got, want = run_both(engine, anml, data, 3, len(data) // 3, group_num=2, depth=depth,
                             algorithm="nonblockingpcgroups", window=window, chunk=chunk,
                             tile_mode=tile_mode)
        assert len(want) > 10
        assert np.array_equal(got, want), depth


@pytest.mark.parametrize("chunk,window,tile_states",[(100, 128, 0), (1000, 0, 64), (0, 33, 300)])
def test_chunking_and_tiling(engine, chunk, window, tile_states):
    """Small chunks, windows and tiles exercise warm-up, carry and tile splits."""
    anml, data = W.hamming_set(seed=12, n_patterns=30, input_len=1 << 16, plant_every=1 << 10)
    got, want = run_both(engine, anml, data, 2, len(data) // 2, group_num=3, depth=2,
                         algorithm="nonblockingallgroups", chunk=chunk, window=window,
                         tile_states=tile_states)
    assert np.array_equal(got, want)


def test_start_of_data_and_dup(engine):
    """Start-of-data states: segment 0 only, or every segment when duplicated."""
    anml = W.AnmlWriter()
    anml.ste("a", [ord("x")], ["b"], start="start-of-data")
    anml.ste("b", [ord("y")], ["c"])
    anml.ste("c", [ord("z")], [], report=True)
    anml.ste("d", [ord("y")], ["e"], start="all-input")
    anml.ste("e", [ord("z")], [], report=True)
    data = np.frombuffer(b"xyzxyz" * 4, dtype=np.uint8).copy()
    for is_dup in (False, True):
        for algo in ALGOS:
            got, want = run_both(engine, anml.text(), data, 4, 6, group_num=2, is_dup=is_dup,
                                 depth=2, algorithm=algo)
            assert np.array_equal(got, want), (algo, is_dup)


@pytest.mark.parametrize("seg_len", [1, 2, 3, 17])
def test_ragged_tiny_segments(engine, seg_len):
    anml, data = W.literal_set(seed=13, n_patterns=20, len_lo=1, len_hi=3, input_len=1 << 12,
                               plant_every=64)
    n = len(data) // seg_len
    got, want = run_both(engine, anml, data, n, seg_len, group_num=2, depth=3,
                         algorithm="nonblockingallgroups")
    assert np.array_equal(got, want)


def test_unique_flag(engine):
    anml, data = W.levenshtein_set(seed=14, n_patterns=20, input_len=1 << 15, plant_every=1 << 10)
    got, want = run_both(engine, anml, data, 1, len(data), group_num=2, depth=1,
                         algorithm="nonblockinggroups", unique=True)
    assert np.array_equal(got, want)


def test_report_off_and_capacity(engine):
    anml, data = W.literal_set(seed=15, input_len=1 << 16, plant_every=1 << 9)
    nfa = nb.Nfa.from_string(anml)
    groups = nb.Groups(nfa, group_num=1)
    tables = nb.Tables(groups, precompute_depth=1)
    want, _ = oracle.match(groups.views(), data, 1, len(data))
    engine.match(tables, data, 1, len(data), report_off=True)
    raw, uniq = engine.counts()
    assert raw >= len(want) and uniq == 0
    with pytest.raises(nb.NgapError) as ei:
        engine.match(tables, data, 1, len(data), result_capacity=3)
    assert ei.value.status == 7  # NGAP_E_OVERFLOW_RESULTS


def test_device_input_and_sort_api(engine):
    import torch
    anml, data = W.hamming_set(seed=16, n_patterns=20, input_len=1 << 16, plant_every=1 << 10)
    nfa = nb.Nfa.from_string(anml)
    groups = nb.Groups(nfa, group_num=2)
    tables = nb.Tables(groups, precompute_depth=3)
    d = torch.from_numpy(data).cuda()
    got = engine.match(tables, d, 4, len(data) // 4)
    want, _ = oracle.match(groups.views(), data, 4, len(data) // 4)
    assert np.array_equal(got, want)
    # the standalone radix sort + unique on a shuffled, duplicated copy
    rng = np.random.default_rng(0)
    shuffled = np.concatenate([want, want[: len(want) // 2]])
    rng.shuffle(shuffled)
    din = torch.from_numpy(shuffled.view(np.int64)).cuda()
    dout = torch.empty_like(din)
    n = engine.sort_unique_device(din.data_ptr(), len(shuffled), dout.data_ptr())
    torch.cuda.synchronize()
    assert n == len(want)
    assert np.array_equal(dout[:n].cpu().numpy().view(np.uint64), want)


@pytest.mark.parametrize("n", [1, 2, 5000, 8192, 8193, 60000])
def test_sort_unique_sizes(engine, n):
    """Device sort + unique on both sides of the single-CTA cutoff (8192 keys)."""
    import torch
    rng = np.random.default_rng(n)
    ids = rng.integers(0, 1 << 24, size=n, dtype=np.uint64)
    offs = rng.integers(0, 1 << 30, size=n, dtype=np.uint64)
    keys = (ids << np.uint64(32)) | offs
    keys = np.concatenate([keys, keys[: n // 3]])
    rng.shuffle(keys)
    swapped = np.unique((keys << np.uint64(32)) | (keys >> np.uint64(32)))
    want = (swapped << np.uint64(32)) | (swapped >> np.uint64(32))
    din = torch.from_numpy(keys.view(np.int64)).cuda()
    dout = torch.empty_like(din)
    m = engine.sort_unique_device(din.data_ptr(), len(keys), dout.data_ptr())
    torch.cuda.synchronize()
    assert m == len(want)
    assert np.array_equal(dout[:m].cpu().numpy().view(np.uint64), want)


@pytest.mark.parametrize("algo", ["nonblockingpcgroups", "NAPgroups"])
def test_dense_reports(engine, algo):
    """A report at almost every position: tens of thousands of reports take the
    radix pipeline, a handful the single-CTA sort."""
    w = W.AnmlWriter()
    w.ste("a", list(range(1, 256)), ["b"], start="all-input", report=True)
    w.ste("b", [ord("x")], [], report=True)
    rng = np.random.default_rng(4)
    for size in (40000, 3000):
        data = rng.integers(0, 256, size=size, dtype=np.uint8)
        got, want = run_both(engine, w.text(), data, 4, size // 4, group_num=1, depth=2,
                             algorithm=algo)
        assert len(want) > size // 2
        assert np.array_equal(got, want), size


@pytest.mark.parametrize("tile_mode", ["shared", "global"])
def test_layered_many_active(engine, tile_mode):
    """Dot-star CCs matched in chunks (activation pass, then layered tiles):
    1-2 byte prefixes activate hundreds of `.*` states early, more than a
    warp's shared sticky list holds."""
    anml, data = W.dotstar_set(seed=41, n_patterns=300, lit_lo=1, lit_hi=2, aas_frac=0.0,
                               input_len=1 << 16, plant_every=1 << 9)
    for algo in ("nonblockingpcgroups", "nonblockinggroups", "NAPgroups"):
        for window in (0, 100):
            got, want = run_both(engine, anml, data, 3, len(data) // 3, group_num=2, depth=-1,
                                 algorithm=algo, tile_mode=tile_mode, window=window, chunk=1000)
            assert len(want) > 100
            assert np.array_equal(got, want), (algo, window)


def _two_star(w, p, rng, lo=2, hi=3):
    """lit .* lit .* lit: a sticky state reachable from another (not layered)."""
    lits = [rng.integers(97, 101, size=int(rng.integers(lo, hi + 1))) for _ in range(3)]
    names = []
    for k, lit in enumerate(lits):
        for i, c in enumerate(lit):
            names.append((f"t{p}l{k}c{i}", int(c)))
    prev = None
    for k, lit in enumerate(lits):
        for i, c in enumerate(lit):
            nm = f"t{p}l{k}c{i}"
            last = i == len(lit) - 1
            nxt = ([f"t{p}s{k}", f"t{p}l{k + 1}c0"] if k < 2 else []) if last else [f"t{p}l{k}c{i + 1}"]
            w.ste(nm, [int(c)], nxt, start="all-input" if (k == 0 and i == 0) else None,
                  report=(k == 2 and last))
        if k < 2:
            w.ste(f"t{p}s{k}", None, [f"t{p}s{k}", f"t{p}l{k + 1}c0"], symbol_set="*")


def test_layered_mixed_with_cyclic(engine):
    """Layered dot-star CCs next to CCs that stay sequential (two `.*` in a
    row, a reporting `.*`) and plain literals, over several segments."""
    rng = np.random.default_rng(42)
    w = W.AnmlWriter()
    for p in range(12):
        _two_star(w, p, rng)
    for p in range(20):  # lit .* lit with a reporting star
        a = rng.integers(97, 101, size=2)
        w.ste(f"r{p}a0", [int(a[0])], [f"r{p}a1"], start="all-input")
        w.ste(f"r{p}a1", [int(a[1])], [f"r{p}s"])
        w.ste(f"r{p}s", None, [f"r{p}s", f"r{p}b"], symbol_set="*", report=(p % 2 == 0))
        w.ste(f"r{p}b", [int(rng.integers(97, 101))], [], report=True)
    for p in range(10):
        w.ste(f"x{p}", [int(rng.integers(97, 101))], [f"y{p}"], start="all-input")
        w.ste(f"y{p}", [int(rng.integers(97, 101))], [], report=True)
    data = rng.integers(97, 102, size=30000).astype(np.uint8)
    for algo in ("nonblockingpcgroups", "blockinggroups", "nonblockingallgroups"):
        for tile_mode in ("auto", "global"):
            got, want = run_both(engine, w.text(), data, 5, 6000, group_num=3, depth=3,
                                 algorithm=algo, tile_mode=tile_mode, chunk=700)
            assert len(want) > 100
            assert np.array_equal(got, want), (algo, tile_mode)


def test_dead_windows(engine):
    """Windows whose bytes are all of the tile's dead class (bytes no state
    accepts) skip injection: DNA patterns over a stream of 'x' with ACGT
    islands (planted occurrences included) that straddle window and chunk
    boundaries, matches carried into dead windows among them."""
    anml, dna = W.hamming_set(seed=61, n_patterns=20, input_len=1 << 14, plant_every=1 << 9)
    rng = np.random.default_rng(61)
    data = np.full(1 << 16, ord("x"), dtype=np.uint8)
    for _ in range(200):
        n = int(rng.integers(20, 600))
        at = int(rng.integers(0, len(data) - n))
        src = int(rng.integers(0, len(dna) - n))
        data[at:at + n] = dna[src:src + n]
    for window, chunk in ((64, 0), (0, 700), (97, 300)):
        got, want = run_both(engine, anml, data, 4, len(data) // 4, group_num=2, depth=-1,
                             algorithm="nonblockingpcgroups", window=window, chunk=chunk)
        assert len(want) > 20
        assert np.array_equal(got, want), (window, chunk)


def test_layered_shortcuts(engine):
    """Successors a `.*` enables from its first match on (their edges from the
    `.*`'s predecessors dropped from the layered tile): a reporting successor
    right after the predecessors (gap 0), two predecessors that both lead to
    the successor (a shortcut) or only one of them (none), over several
    segments and chunks."""
    w = W.AnmlWriter()
    # x y .* z (report at z): y leads to .* and to z
    w.ste("a0", [ord("x")], ["a1"], start="all-input")
    w.ste("a1", [ord("y")], ["as", "az"])
    w.ste("as", None, ["as", "az"], symbol_set="*")
    w.ste("az", [ord("z")], [], report=True)
    # (p | q) .* r r, both p and q lead to the first r: a shortcut
    w.ste("b0", [ord("p")], ["bs", "br"], start="all-input")
    w.ste("b1", [ord("q")], ["bs", "br"], start="all-input")
    w.ste("bs", None, ["bs", "br"], symbol_set="*")
    w.ste("br", [ord("r")], ["bt"])
    w.ste("bt", [ord("r")], [], report=True)
    # (p | q) .* z, only p leads to z directly: no shortcut
    w.ste("c0", [ord("p")], ["cs", "cz"], start="all-input")
    w.ste("c1", [ord("q")], ["cs"], start="all-input")
    w.ste("cs", None, ["cs", "cz"], symbol_set="*")
    w.ste("cz", [ord("z")], [], report=True)
    groups = nb.Groups(nb.Nfa.from_string(w.text()), group_num=1)
    lay = [t for t in groups.tiles(precompute_depth=2) if t["phase"] == 2]
    assert sum(t["shortcuts"] for t in lay) == 2  # az of as, br of bs
    rng = np.random.default_rng(8)
    data = rng.choice(np.frombuffer(b"xyzpqr", dtype=np.uint8), size=6000,
                      p=[0.3, 0.3, 0.1, 0.05, 0.05, 0.2])
    for algo in ("nonblockingpcgroups", "blockinggroups", "NAPgroups"):
        for chunk in (0, 97):
            got, want = run_both(engine, w.text(), data, 6, 1000, depth=2, algorithm=algo,
                                 chunk=chunk)
            assert len(want) > 50
            assert np.array_equal(got, want), (algo, chunk)


def test_layered_shortcuts_random(engine):
    """Random star-heavy automata (extra forward edges around `.*` states,
    reporting and always-active stars): every layered tile, with or without
    shortcuts, gives the oracle's reports."""
    from test_tiles_host import _random_star_nfa
    with_shortcuts = 0
    for seed in range(40):
        rng = np.random.default_rng(500 + seed)
        anml = _random_star_nfa(rng, int(rng.integers(2, 12)))
        groups = nb.Groups(nb.Nfa.from_string(anml), group_num=2)
        with_shortcuts += sum(t["shortcuts"] > 0 for t in groups.tiles(precompute_depth=3))
        data = rng.integers(96, 102, size=4000).astype(np.uint8)
        got, want = run_both(engine, anml, data, 4, 1000, group_num=2, depth=3,
                             algorithm=("nonblockingpcgroups", "blockinggroups")[seed % 2],
                             chunk=(0, 150)[(seed // 2) % 2])
        assert np.array_equal(got, want), seed
    assert with_shortcuts > 5


def test_plan_cache_after_tables_freed(engine):
    """Tables created where freed ones were (same address) get their own unit
    plan: the engine keys its plan cache by a serial number."""
    import gc
    anml, data = W.dotstar_set(seed=43, n_patterns=60, input_len=1 << 15, plant_every=1 << 9)
    nfa = nb.Nfa.from_string(anml)
    groups = nb.Groups(nfa, group_num=2)
    want, _ = oracle.match(groups.views(), data, 2, len(data) // 2)
    for i in range(8):
        mode = ("shared", "global", "auto")[i % 3]
        tables = nb.Tables(groups, precompute_depth=(3, -1)[i % 2], tile_mode=mode,
                           tile_states=(0, 300)[(i // 2) % 2])
        got = engine.match(tables, data, 2, len(data) // 2)
        assert np.array_equal(got, want), (i, mode)
        del tables
        gc.collect()
