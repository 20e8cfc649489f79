"""GPU side of the learned scheduler and the serving loop: worklist traces,
the feature kernel, the MLP kernels, and that scheduling knobs and batching
never change a report."""
import numpy as np
import pytest

import ngap_b200 as nb
from ngap_b200 import cost_model as cm
from ngap_b200 import serving as sv
from ngap_b200 import workloads as W
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_suite():
    nfas, data, offsets, lengths, nfa_of = W.batched_suite(
        seed=11, n_nfas=4, n_streams=40, min_states=300, max_states=3000, len_lo=1 << 8,
        len_hi=1 << 16, sample_len=1 << 14)
    groups = [nb.Groups(nb.Nfa.from_string(n["anml"]), group_num=2) for n in nfas]
    tables = [nb.Tables(g, precompute_depth=-1) for g in groups]
    return nfas, data, offsets, lengths, nfa_of, groups, tables, nb.TableSet(tables)


def test_unit_trace_sums_to_engine_work(engine, small_suite):
    nfas, data, offsets, lengths, nfa_of, groups, tables, ts = small_suite
    engine.set_trace(True)
    try:
        nb.batch_match_async(engine, ts, data, offsets, lengths, nfa_of)
        engine.sync()
        tr = engine.unit_trace()
    finally:
        engine.set_trace(False)
    exp, inj = engine.work()
    assert len(tr) > 0 and int(tr["work"].sum()) == exp + inj
    assert np.all(tr["lo"] >= 0) and np.all(tr["hi"] <= lengths[tr["stream"]])
    # plain matching: positions relative to each segment
    engine.set_trace(True)
    try:
        engine.match(tables[0], data[:1 << 14], 4, 1 << 12)
        tp = engine.unit_trace()
    finally:
        engine.set_trace(False)
    exp, inj = engine.work()
    assert int(tp["work"].sum()) == exp + inj and tp["hi"].max() <= 1 << 12


def test_feature_kernel_matches_host_definition(small_suite):
    rng = np.random.default_rng(2)
    data = rng.integers(0, 9, size=100000).astype(np.uint8)
    offs = np.array([0, 5, 1000, 50000, 99999], np.int64)
    lens = np.array([1, 700, 1024, 30001, 1], np.int64)
    got = cm.byte_features(data, offs, np.arange(5), np.zeros(5, np.int64), lens)
    for i in range(5):
        want = sv.host_features(data[offs[i]:offs[i] + lens[i]])
        assert np.allclose(got[i], want, atol=1e-5), i


def test_mlp_trains_and_bf16_follows_fp32():
    rng = np.random.default_rng(3)
    x = rng.standard_normal((4000, 20)).astype(np.float32)
    y = np.abs(x[:, 0] * 2 + x[:, 1] - 0.5 * x[:, 2]) * 3
    m = cm.LearnedModel(0, seed=4, in_dim=20)
    before = np.mean((m.predict_log(x, bf16=False) - np.log2(1 + y)) ** 2)
    m.fit(x, y, epochs=40, batch=256, lr=2e-3)
    f32 = m.predict_log(x, bf16=False)
    b16 = m.predict_log(x, bf16=True)
    after = np.mean((f32 - np.log2(1 + y)) ** 2)
    assert after < 0.02 * before
    assert np.max(np.abs(b16 - f32)) < 0.05 * max(1.0, np.max(np.abs(f32)))
    m2 = cm.LearnedModel(0, seed=9, in_dim=20)
    m2.set_params(m.params())
    m2.mu, m2.sd = m.mu, m.sd
    assert np.array_equal(m2.predict_log(x, bf16=False), f32)


def test_scheduler_knobs_keep_reports(engine, small_suite):
    """Per-stream chunk lengths and a small queue capacity reshape the work
    only; a queue too small fails loudly instead of losing reports."""
    nfas, data, offsets, lengths, nfa_of, groups, tables, ts = small_suite
    nb.batch_match_async(engine, ts, data, offsets, lengths, nfa_of)
    engine.sync()
    base = nb.batch_results(engine)
    rng = np.random.default_rng(5)
    chunks = rng.choice([0, 256, 700, 4096, 9000], size=len(offsets))
    for q in (0, 4096, 1024):
        try:
            nb.batch_match_async(engine, ts, data, offsets, lengths, nfa_of, chunks=chunks,
                                 queue_capacity=q)
            engine.sync()
        except nb.NgapError as ex:
            assert ex.status == 6  # NGAP_E_OVERFLOW_QUEUE
            continue
        got = nb.batch_results(engine)
        assert np.array_equal(got[0], base[0]) and np.array_equal(got[1], base[1]), q


def test_serving_results_same_alone_and_in_the_mix(engine, small_suite):
    """Requests served by continuous batching over two engines report exactly
    what each reports when matched alone, with every scheduler."""
    nfas, data, offsets, lengths, nfa_of, groups, tables, ts = small_suite
    pool = [data[int(o):int(o + l)] for o, l in zip(offsets, lengths) if l > 0]
    pool_nfa = [int(k) for k, l in zip(nfa_of, lengths) if l > 0]
    reqs = sv.make_requests(pool, pool_nfa, len(nfas), rate=20000, duration=0.01,
                            median=4096, max_len=1 << 16, seed=7)
    assert len(reqs) > 50
    reg = cm.region_table(data, offsets, lengths, nfa_of, tables)
    y = cm.collect(engine, ts, data, offsets, lengths, nfa_of, reg)
    lm = cm.LearnedModel(0).fit(reg["x"], y, epochs=20)
    served = {}
    for name, pred in (("default", None), ("static", sv.Predictor("static", tables)),
                       ("learned", sv.Predictor("learned", tables, lm))):
        rs = [sv.Request(r.rid, r.nfa, r.data, r.arrival) for r in reqs]
        srv = sv.Server(ts, predictor=pred, slots=2, budget=1 << 22, max_batch_bytes=1 << 20,
                        queue_capacity=cm.queue_for(4.0) if pred else 0)
        m = srv.run(rs)
        assert m["requests"] == len(reqs) and m["p99_ms"] >= m["p50_ms"] > 0
        served[name] = rs
    for r in reqs:
        want, _ = oracle.match(groups[r.nfa].views(), r.data, 1, len(r.data))
        for name in served:
            assert np.array_equal(served[name][r.rid].reports, want), (name, r.rid)
