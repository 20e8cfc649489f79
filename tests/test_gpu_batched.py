"""Batched matching on the GPU: many streams of uneven length, several NFAs,
one launch; every stream's reports bit-exact against the oracle run on that
stream alone (one segment, start-of-data states at its start)."""
import numpy as np
import pytest

import ngap_b200 as nb
from ngap_b200 import workloads as W
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def suite():
    nfas, data, offsets, lengths, nfa_of = W.batched_suite(
        seed=7, n_nfas=5, n_streams=48, min_states=300, max_states=4000, len_lo=1,
        len_hi=1 << 15, sample_len=1 << 14)
    groups = [nb.Groups(nb.Nfa.from_string(n["anml"]), group_num=3) for n in nfas]
    return nfas, data, offsets, lengths, nfa_of, groups


def _expected(suite):
    nfas, data, offsets, lengths, nfa_of, groups = suite
    out = []
    for s in range(len(offsets)):
        seg = data[offsets[s]:offsets[s] + lengths[s]]
        if lengths[s] == 0:
            out.append(np.zeros(0, np.uint64))
            continue
        want, _ = oracle.match(groups[nfa_of[s]].views(), seg, 1, int(lengths[s]))
        out.append(want)
    return out


@pytest.mark.parametrize("depth,algo,graph", [(2, "nonblockingpcgroups", False),
                                              (-1, "nonblockingallgroups", False),
                                              (-1, "nonblockingpcgroups", True),
                                              (0, "NAPgroups", False)])
def test_batched_per_stream_parity(engine, suite, depth, algo, graph):
    import torch
    nfas, data, offsets, lengths, nfa_of, groups = suite
    tables = [nb.Tables(g, precompute_depth=depth) for g in groups]
    ts = nb.TableSet(tables)
    want = _expected(suite)
    assert sum(len(w) for w in want) > 20
    src = torch.from_numpy(data).pin_memory() if graph else data
    for rep in range(2 if graph else 1):  # graph: capture, then replay
        nb.batch_match_async(engine, ts, src.numpy() if graph else src, offsets, lengths, nfa_of,
                             algorithm=algo, use_graph=graph)
        engine.sync()
        reps, sids = nb.batch_results(engine)
        got = nb.split_by_stream(reps, sids, len(offsets))
        for s in range(len(offsets)):
            assert np.array_equal(got[s], want[s]), (rep, s, nfas[nfa_of[s]]["kind"])


def test_batched_device_input_and_mixed_tiles(engine, suite):
    import torch
    nfas, data, offsets, lengths, nfa_of, groups = suite
    tables = [nb.Tables(g, precompute_depth=3, tile_states=200) for g in groups]
    ts = nb.TableSet(tables)
    d = torch.from_numpy(data).cuda()
    nb.batch_match_async(engine, ts, d, offsets, lengths, nfa_of, chunk=700, window=256)
    engine.sync()
    reps, sids = nb.batch_results(engine)
    got = nb.split_by_stream(reps, sids, len(offsets))
    for s, w in enumerate(_expected(suite)):
        assert np.array_equal(got[s], w), s


def test_plain_after_batched(engine, suite):
    """The engine's plan caches switch cleanly between plain and batched runs."""
    nfas, data, offsets, lengths, nfa_of, groups = suite
    t = nb.Tables(groups[0], precompute_depth=2)
    seg = data[:4096]
    got = engine.match(t, seg, 4, 1024)
    want, _ = oracle.match(groups[0].views(), seg, 4, 1024)
    assert np.array_equal(got, want)


def test_batched_global_tiles(engine, suite):
    """Global tiles (several groups per tile) inside a tableset."""
    nfas, data, offsets, lengths, nfa_of, groups = suite
    tables = [nb.Tables(g, precompute_depth=-1, tile_mode="global") for g in groups]
    ts = nb.TableSet(tables)
    nb.batch_match_async(engine, ts, data, offsets, lengths, nfa_of, window=200)
    engine.sync()
    reps, sids = nb.batch_results(engine)
    got = nb.split_by_stream(reps, sids, len(offsets))
    for s, w in enumerate(_expected(suite)):
        assert np.array_equal(got[s], w), s


def test_batched_dense_reports(engine):
    """Tens of thousands of reports over many streams: the radix pipeline."""
    w = W.AnmlWriter()
    w.ste("a", list(range(1, 256)), ["b"], start="all-input", report=True)
    w.ste("b", [ord("x")], [], report=True)
    g = nb.Groups(nb.Nfa.from_string(w.text()), group_num=1)
    ts = nb.TableSet([nb.Tables(g, precompute_depth=2)])
    rng = np.random.default_rng(5)
    lengths = rng.integers(0, 3000, size=40).astype(np.uint64)
    offsets = np.concatenate([[0], np.cumsum(lengths)[:-1]]).astype(np.uint64)
    data = rng.integers(0, 256, size=int(lengths.sum()), dtype=np.uint8)
    nfa_of = np.zeros(len(lengths), np.int32)
    nb.batch_match_async(engine, ts, data, offsets, lengths, nfa_of)
    engine.sync()
    reps, sids = nb.batch_results(engine)
    got = nb.split_by_stream(reps, sids, len(offsets))
    total = 0
    for s in range(len(lengths)):
        seg = data[int(offsets[s]):int(offsets[s] + lengths[s])]
        want = (oracle.match(g.views(), seg, 1, int(lengths[s]))[0] if lengths[s]
                else np.zeros(0, np.uint64))
        total += len(want)
        assert np.array_equal(got[s], want), s
    assert total > 20000
