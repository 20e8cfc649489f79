"""The oracle itself (CPU): pinned to the reference's known-answer test, to an
independent brute-force simulation, and checked for sensitivity."""
import os

import numpy as np
import pytest

import ngap_b200 as nb
from ngap_b200 import workloads as W
from oracle import frontend, oracle

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
APPLE = ["0x400000005", "0x40000002f", "0x400000040", "0x40000004b"]


def _apple():
    nodes, adj = frontend.load_anml(open(os.path.join(GOLD, "apple.anml")).read())
    data = np.fromfile(os.path.join(GOLD, "apple_input.txt"), dtype=np.uint8)
    return frontend.build_groups(nodes, adj, 1), data


@pytest.mark.parametrize("mode", [0, 1])
def test_apple_known_answer(mode):
    groups, data = _apple()
    got, _ = oracle.match(groups, data, 1, len(data), mode=mode)
    assert [hex(x) for x in got] == APPLE


def test_apple_segmented_drops_straddling_matches():
    """Segments start from scratch (ngap.cu:2201-2210): an 'apple' crossing a
    segment boundary is not reported."""
    groups, data = _apple()
    got, _ = oracle.match(groups, data, 3, 27, mode=1)  # boundaries at 27 and 54
    offs = sorted(int(x) & 0xFFFFFFFF for x in got)
    assert offs == [5, 47, 64, 75]
    got2, _ = oracle.match(groups, data, 9, 9, mode=1)  # boundaries 45, 63, 72 cut 3 matches
    assert sorted(int(x) & 0xFFFFFFFF for x in got2) == [5]


def brute(groups, data, num_seg, seg_len, is_dup=False):
    """Set-based NFA simulation written independently of the C oracle."""
    out = set()
    for gi, g in enumerate(groups):
        bits, ro, co = g["symbol_sets"], g["row_offsets"], g["col_indices"]
        for s in range(num_seg):
            lo = s * seg_len
            front = set(int(x) for x in g["always_active"])
            if s == 0 or is_dup:
                front |= set(int(x) for x in g["start_states"])
            for p in range(lo, lo + seg_len):
                b = int(data[p])
                nxt = set()
                for v in front:
                    if (int(bits[v, b >> 5]) >> (b & 31)) & 1:
                        if g["node_attrs"][v] & 2:
                            out.add(((v | (gi << 22)) << 32) | p)
                        nxt |= set(int(x) for x in co[ro[v]:ro[v + 1]])
                front = nxt | set(int(x) for x in g["always_active"])
    keys = sorted(((r & 0xFFFFFFFF) << 32) | (r >> 32) for r in out)
    return np.array([((k & 0xFFFFFFFF) << 32) | (k >> 32) for k in keys], dtype=np.uint64)


@pytest.mark.parametrize("gen,kw,g,nseg", [
    (W.literal_set, dict(seed=31, n_patterns=12, input_len=3000, plant_every=300), 2, 3),
    (W.levenshtein_set, dict(seed=32, n_patterns=3, k=8, input_len=1500, plant_every=200), 2, 2),
    (W.dotstar_set, dict(seed=33, n_patterns=5, input_len=2000, plant_every=300), 3, 2),
    (W.hamming_set, dict(seed=34, n_patterns=3, k=8, input_len=1500, plant_every=150), 2, 3),
])
@pytest.mark.parametrize("is_dup", [False, True])
def test_oracle_vs_brute_force(gen, kw, g, nseg, is_dup):
    anml, data = gen(**kw)
    nodes, adj = frontend.load_anml(anml)
    groups = frontend.build_groups(nodes, adj, g)
    seg = len(data) // nseg
    want = brute(groups, data, nseg, seg, is_dup)
    for mode in (0, 1):
        got, _ = oracle.match(groups, data, nseg, seg, is_dup=is_dup, mode=mode)
        assert np.array_equal(got, want)


def test_unique_flag_same_set():
    anml, data = W.levenshtein_set(seed=35, n_patterns=4, k=8, input_len=4000, plant_every=300)
    nodes, adj = frontend.load_anml(anml)
    groups = frontend.build_groups(nodes, adj, 2)
    a, sa = oracle.match(groups, data, 2, 2000, mode=0, unique=False)
    b, sb = oracle.match(groups, data, 2, 2000, mode=0, unique=True)
    c, sc = oracle.match(groups, data, 2, 2000, mode=1)
    assert np.array_equal(a, b) and np.array_equal(a, c)
    assert sa["reports_raw"] >= sb["reports_raw"] >= sc["reports_raw"]


def test_product_cpu_checker_agrees_and_planted_mistake_is_caught(built):
    """The CLI's CPU checker and the oracle agree; an error planted in the
    oracle's copy of the tables (one report flag cleared) is detected."""
    anml, data = W.literal_set(seed=36, n_patterns=16, input_len=20000, plant_every=500)
    groups = nb.Groups(nb.Nfa.from_string(anml), group_num=2)
    views = groups.views()
    want, _ = oracle.match(views, data, 4, 5000)
    assert np.array_equal(nb.cpu_validate(groups, data, 4, 5000), want)
    planted = [dict(row_offsets=v.row_offsets, col_indices=v.col_indices,
                    symbol_sets=v.symbol_sets, node_attrs=v.node_attrs.copy(),
                    always_active=v.always_active, start_states=v.start_states) for v in views]
    rep_states = np.nonzero(planted[0]["node_attrs"] & 2)[0]
    planted[0]["node_attrs"][rep_states] &= 0xFD
    bad, _ = oracle.match(planted, data, 4, 5000)
    assert len(bad) < len(want)


def test_stats_count_frontier():
    groups, data = _apple()
    _, st = oracle.match(groups, data, 1, len(data), mode=1)
    # 'a' is always active: it matches at every 'a' of the input
    assert st["matched"] >= int(np.sum(data == ord("a")))
    assert st["reports_raw"] == 4
