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
    # every unit ran: a start clock was replaced by a positive duration (< 2^40)
    assert np.all(tr["cycles"] > 0) and np.all(tr["cycles"] < (1 << 40))
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


H = 64


def _unpack(p, D):
    """W1[D][H], b1[H], W2[H][H], b2[H], w3[H], b3 from the flat parameter
    vector (the layout of ngap_mlp_get_params)."""
    o = 0
    W1 = p[o:o + D * H].reshape(D, H); o += D * H
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    return W1, b1, W2, b2, w3, p[o]


def _np_forward(p, x, D, rnd=lambda a: a):
    W1, b1, W2, b2, w3, b3 = (rnd(a) for a in _unpack(p, D))
    h1 = rnd(np.maximum(rnd(x) @ W1 + b1, 0.0))
    h2 = rnd(np.maximum(h1 @ W2 + b2, 0.0))
    return h2 @ w3 + b3, h1, h2


def _bf16(a):
    """Round float32 values to bfloat16 (round to nearest, ties to even),
    returned as float64."""
    u = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def _model(D, seed):
    m = cm.LearnedModel(0, seed=seed, in_dim=D)
    rng = np.random.default_rng(seed)
    p = (rng.standard_normal(len(m.params())) * 0.2).astype(np.float32)
    m.set_params(p)
    return m, p.astype(np.float64), rng


def _raw_predict(m, x, bf16):
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros(len(x), np.float32)
    nb.lib().ngap_mlp_predict(m._h, x.ctypes.data, len(x), int(bf16), out.ctypes.data)
    return out.astype(np.float64)


def test_mlp_fp32_forward_matches_numpy():
    """mlp_infer_kernel<false> against a float64 numpy forward pass of the
    same parameters: relative tolerance 1e-5 (FP32 accumulation of at most
    266 products in a different order)."""
    D = cm.IN_DIM
    m, p, rng = _model(D, 5)
    x = rng.standard_normal((333, D)).astype(np.float32)  # a partial last block of rows
    want, _, _ = _np_forward(p, x.astype(np.float64), D)
    got = _raw_predict(m, x, bf16=False)
    scale = np.abs(want).max()
    assert np.allclose(got, want, rtol=1e-5, atol=1e-5 * scale)


def test_mlp_bf16_forward_matches_numpy_rounding():
    """mlp_infer_kernel<true> rounds inputs, weights and activations to bfloat16
    and accumulates in FP32: against a numpy forward pass with the same
    roundings (float64 accumulation), tolerance 4e-3 of the largest output
    (an activation whose FP32 sum lies within one bfloat16 step of a rounding
    boundary may round the other way, 2^-8 of it), and within 5 % of the FP32
    result."""
    D = cm.IN_DIM
    m, p, rng = _model(D, 6)
    x = rng.standard_normal((256, D)).astype(np.float32)
    want, _, _ = _np_forward(p, x.astype(np.float64), D, rnd=_bf16)
    got = _raw_predict(m, x, bf16=True)
    scale = np.abs(want).max()
    assert np.allclose(got, want, rtol=4e-3, atol=4e-3 * scale)
    fp32, _, _ = _np_forward(p, x.astype(np.float64), D)
    assert np.abs(got - fp32).max() <= 0.05 * np.abs(fp32).max()


def test_mlp_host_inference_matches_the_kernel():
    """ngap_mlp_predict_host (the serving loop's inference) against the
    inference kernel: the same roundings and accumulation order per unit,
    products not fused, so FP32 within 1e-4 of the largest output and BF16
    within 4e-3 (an activation within one bfloat16 step of a rounding
    boundary may round the other way, as in the BF16 numpy check); it
    follows parameter changes (set_params)."""
    D = cm.IN_DIM
    m, p, rng = _model(D, 9)
    x = rng.standard_normal((77, D)).astype(np.float32)
    for bf16 in (False, True):
        dev = _raw_predict(m, x, bf16)
        host = np.zeros(len(x), np.float32)
        assert nb.lib().ngap_mlp_predict_host(m._h, x.ctypes.data, len(x), int(bf16),
                                              host.ctypes.data) == 0
        tol = 4e-3 if bf16 else 1e-4
        assert np.allclose(host, dev, rtol=tol, atol=tol * np.abs(dev).max()), bf16
    m.set_params((p * 0.5).astype(np.float32))
    dev = _raw_predict(m, x, False)
    host = np.zeros(len(x), np.float32)
    nb.lib().ngap_mlp_predict_host(m._h, x.ctypes.data, len(x), 0, host.ctypes.data)
    assert np.allclose(host, dev, rtol=1e-4, atol=1e-4 * np.abs(dev).max())


def test_mlp_gradient_matches_numpy_backprop():
    """mlp_grad_kernel (the gradient that ngap_mlp_train gives to Adam)
    against float64 numpy backpropagation of the mean squared error:
    relative tolerance 1e-4 of the largest gradient entry (FP32 sums and
    atomic accumulation across blocks in any order)."""
    D = 40
    m, p, rng = _model(D, 7)
    n = 300
    x = rng.standard_normal((n, D)).astype(np.float32)
    t = rng.standard_normal(n).astype(np.float32)
    grad = np.zeros(len(p), np.float32)
    loss = np.zeros(1, np.float32)
    import ctypes
    rc = nb.lib().ngap_mlp_gradient(m._h, x.ctypes.data, t.ctypes.data, n, grad.ctypes.data,
                                     ctypes.cast(loss.ctypes.data, ctypes.POINTER(ctypes.c_float)))
    assert rc == 0
    X = x.astype(np.float64)
    y, h1, h2 = _np_forward(p, X, D)
    W1, b1, W2, b2, w3, b3 = _unpack(p, D)
    dy = 2.0 * (y - t) / n
    d2 = (h2 > 0) * np.outer(dy, w3)
    d1 = (h1 > 0) * (d2 @ W2.T)
    want = np.concatenate([(X.T @ d1).ravel(), d1.sum(0), (h1.T @ d2).ravel(), d2.sum(0),
                           h2.T @ dy, [dy.sum()]])
    g = grad.astype(np.float64)
    assert np.allclose(g, want, rtol=1e-4, atol=1e-4 * np.abs(want).max())
    assert np.isclose(loss[0], np.mean((y - t) ** 2), rtol=1e-4)
    # the parameters are unchanged by the gradient call
    assert np.array_equal(m.params(), p.astype(np.float32))


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
        eng = nb.Engine(0)  # an engine keeps the largest queue it has held
        try:
            nb.batch_match_async(eng, ts, data, offsets, lengths, nfa_of, chunks=chunks,
                                 queue_capacity=q)
            eng.sync()
        except nb.NgapError as ex:
            assert ex.status == 6  # NGAP_E_OVERFLOW_QUEUE
            continue
        got = nb.batch_results(eng)
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
        srv = sv.Server(ts, predictor=pred, slots=2, budget=4 << 30, max_batch_bytes=1 << 20,
                        queue_capacity=cm.queue_for(4.0) if pred else 0)
        m = srv.run(rs)
        assert m["requests"] == len(reqs) and m["p99_ms"] >= m["p50_ms"] > 0
        assert m["rejected"] == 0 and srv.held_bytes() <= srv.budget
        served[name] = rs
    for r in reqs:
        want, _ = oracle.match(groups[r.nfa].views(), r.data, 1, len(r.data))
        for name in served:
            assert np.array_equal(served[name][r.rid].reports, want), (name, r.rid)
