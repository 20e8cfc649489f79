"""Host logic of the learned scheduler and the serving loop (no GPU)."""
import numpy as np
import pytest

from ngap_b200 import cost_model as cm
from ngap_b200 import serving as sv


def test_regions_cover_streams():
    st, a, ln = cm.regions_of(np.array([0, 100, 40000]), np.array([100, 0, 40000]), region=16384)
    assert st.tolist() == [0, 2, 2, 2]
    assert a.tolist() == [0, 0, 16384, 32768]
    assert ln.tolist() == [100, 16384, 16384, 40000 - 32768]


def test_region_density_spreads_unit_work():
    rs, ra, rl = cm.regions_of(np.array([0]), np.array([300]), region=100)
    dt = np.dtype([("stream", np.int32), ("tile", np.int32), ("lo", np.int64), ("hi", np.int64),
                   ("work", np.uint64)])
    tr = np.array([(0, 0, 50, 150, 100), (0, 1, 200, 300, 30)], dtype=dt)
    y = cm.region_density(tr, rs, ra, rl, region=100)
    assert np.allclose(y, [0.5, 0.5, 0.3])


def test_chunks_and_queue():
    c = cm.chunk_for(np.array([0.0, 2.0, 10.0, 1000.0]), 2.0, base_chunk=2048, lo=256, hi=8192)
    assert c.tolist() == [6144, 2048, 559, 256]
    assert cm.queue_for(0.01) == 4096 and cm.queue_for(1000) == 65536
    ch, q = cm.plan(np.array([1.0, 1.0, 4.0]), np.array([100, 100, 10]))
    assert ch[0] == 2048 and ch[2] < 2048 and q == 16384


def test_static_and_mean_models():
    stats = [{"exp_list": 0.5}, {"exp_list": 3.0}]
    s = cm.StaticModel(stats)
    assert np.allclose(s.predict([0, 1, 1]), [1.0, 6.0, 6.0])
    m = cm.NfaMeanModel(2).fit(np.array([0, 0, 1]), np.array([1.0, 3.0, 5.0]),
                               np.array([1.0, 1.0, 2.0]))
    assert np.allclose(m.predict([0, 1]), [2.0, 5.0])
    assert np.allclose(cm.relative_error(np.array([1.0, 0.0]), np.array([2.0, 0.01])), [0.5, 0.2])


def test_host_features_definition():
    rng = np.random.default_rng(0)
    for L in (1, 700, 1024, 5000, 16384):
        d = rng.integers(0, 7, size=L).astype(np.uint8)
        f = sv.host_features(d)
        assert np.allclose(f[:256], np.bincount(d, minlength=256) / L)
        wl = min(L, 1024)
        nwin = max(1, L // 1024)
        hs = []
        for k in range(nwin):
            c = np.bincount(d[k * wl:(k + 1) * wl], minlength=256)
            q = c[c > 0] / wl
            hs.append(-np.sum(q * np.log2(q)))
        assert np.isclose(f[256], np.mean(hs) / 8, atol=1e-6)
        assert np.isclose(f[257], np.max(hs) / 8, atol=1e-6)


def test_library_host_features_agree(built):
    """ngap_features_host (the library's C implementation the serving loop
    predicts with) against host_features, including empty, sub-window and
    ragged regions, and its argument checks."""
    from ngap_b200._lib import lib
    rng = np.random.default_rng(3)
    datas = [rng.integers(0, 256 if i % 2 else 5, size=L).astype(np.uint8)
             for i, L in enumerate((0, 1, 500, 1023, 1024, 1025, 3000, 16384, 16385))]
    datas.append(np.zeros(4096, np.uint8))
    got = sv.features_host(datas)
    want = np.stack([sv.host_features(d) for d in datas])
    assert np.allclose(got, want, rtol=0, atol=1e-6)
    assert sv.features_host([]).shape == (0, 258)
    d = np.zeros(16, np.uint8)
    off = np.array([8], np.uint64)
    ln = np.array([9], np.uint64)  # 8 + 9 > 16
    out = np.zeros(258, np.float32)
    rc = lib().ngap_features_host(d.ctypes.data, 16, off.ctypes.data, ln.ctypes.data, 1, 1024,
                                  out.ctypes.data)
    assert rc != 0
    rc = lib().ngap_features_host(d.ctypes.data, 16, off.ctypes.data, ln.ctypes.data, 1, 0,
                                  out.ctypes.data)
    assert rc != 0


def test_poisson_requests():
    rng = np.random.default_rng(1)
    pool = [rng.integers(0, 256, 4096, dtype=np.uint8) for _ in range(6)]
    reqs = sv.make_requests(pool, [0, 1, 2, 0, 1, 2], 3, rate=2000, duration=1.0, seed=5)
    t = np.array([r.arrival for r in reqs])
    L = np.array([len(r.data) for r in reqs])
    assert 1800 < len(reqs) < 2200 and np.all(np.diff(t) > 0) and t[-1] < 1.0
    assert 50000 < np.median(L) < 80000
    assert set(r.nfa for r in reqs) == {0, 1, 2}


def test_autotune_sample_streams():
    from ngap_b200 import autotune as at
    lengths = np.arange(1, 201, dtype=np.int64) * 100
    idx = at.sample_streams(lengths, frac=0.05, min_streams=8)
    assert np.all(np.diff(idx) > 0) and len(idx) >= 8
    assert lengths[idx].sum() >= 0.05 * lengths.sum()
    assert np.array_equal(idx, at.sample_streams(lengths, frac=0.05, min_streams=8))
    assert len(at.sample_streams(lengths[:5], frac=0.01, min_streams=32)) == 5
    assert len(at.sample_streams(lengths, frac=1.0)) == 200


class FakeSlot:
    """A serving slot without a GPU: memory grows like an engine's (input copy
    to the largest batch, fixed report and scratch parts from the warm-up
    batch) and a batch completes after `polls` done() queries."""

    def __init__(self, fixed=1000, polls=2):
        self.fixed, self.polls = fixed, polls
        self.mem = {"input": 0, "reports": 0, "scratch": 0, "plan": 0}
        self.launched = []
        self.left = 0

    def memory(self):
        return dict(self.mem)

    def launch(self, batch, params):
        n = sum(len(r.data) for r in batch)
        self.mem["input"] = max(self.mem["input"], sv.padded_input(n))
        self.mem["reports"] = self.mem["scratch"] = self.fixed // 2
        self.launched.append([r.rid for r in batch])
        self.left = self.polls

    def done(self):
        self.left -= 1
        return self.left <= 0

    def finish(self, nreq):
        return [np.array([rid], np.int64) for rid in self.launched[-1]], 0.5, 3


def _server(budget, max_bytes, slots=1, fixed=1000, tables=100, chunk_lo=1 << 30):
    made = []

    def factory(i):
        made.append(FakeSlot(fixed))
        return made[-1]
    srv = sv.Server(None, slots=slots, budget=budget, max_batch_bytes=max_bytes, chunk_lo=chunk_lo,
                    slot_factory=factory, tables_bytes=tables)
    return srv, made


def _reqs(sizes):
    return [sv.Request(i, 0, np.zeros(n, np.uint8), 0.0) for i, n in enumerate(sizes)]


def test_serving_warmup_and_request_cap():
    """Each slot is warmed with the largest plan (one max_batch_bytes request
    of the NFA with the most tiles at the shortest chunk) and with the most
    streams (max_batch_requests requests), so that no buffer grows while
    serving; a batch never holds more than max_batch_requests requests."""
    made = []

    def factory(i):
        made.append(FakeSlot(1000))
        return made[-1]
    srv = sv.Server(None, slots=2, budget=1 << 20, max_batch_bytes=1000, chunk_lo=64,
                    slot_factory=factory, tables_bytes=100, max_batch_requests=4)
    for sl in made:
        assert [len(b) for b in sl.launched] == [1, 4]  # the big request, then the many
    q = _reqs([10] * 9)
    assert len(srv._form(q, 0)) == 4 and len(q) == 5


def test_serving_admission_counts_engine_buffers():
    # tables 100 + fixed 1000 + the warm-up batch's input copy of max_batch_bytes
    # (1000 B -> 1072): every engine buffer is allocated at construction
    srv, made = _server(budget=10_000, max_bytes=1000)
    assert srv.held_bytes() == 100 + 1000 + 1072
    q = _reqs([400, 300, 200, 500])  # capped by max_batch_bytes, in arrival order
    assert [r.rid for r in srv._form(q, 0)] == [0, 1, 2] and [r.rid for r in q] == [3]
    # held 100 + 1000 + 10072; a batch of n streams adds a unit plan of 80 B x 2n:
    # two requests add 320 (within 400 of room), three 480
    srv, made = _server(budget=100 + 1000 + 10_072 + 400, max_bytes=10_000)
    q = _reqs([400, 300, 200])
    got = srv._form(q, 0)
    assert [r.rid for r in got] == [0, 1] and len(q) == 1
    with pytest.raises(ValueError):  # the buffers alone exceed the budget
        _server(budget=2000, max_bytes=1000)


def test_serving_rejects_requests_that_never_fit():
    # held 100 + 2 x (1000 + 1072) = 4244, room 500; a lone request of n bytes
    # adds a plan of 80 B x (n // 100 + 2): 900 -> 880 (never fits),
    # 300 -> 400, 200 -> 320, 100 -> 240
    srv, made = _server(budget=4244 + 500, max_bytes=1000, slots=2, chunk_lo=100)
    reqs = _reqs([300, 5000, 200, 900, 100])  # 5000 > max_batch_bytes; 900 > the budget
    m = srv.run(reqs)  # returns instead of waiting forever
    assert m["rejected"] == 2 and m["requests"] == 3
    bad = {r.rid for r in reqs if r.error}
    assert bad == {1, 3} and all("never be admitted" in reqs[i].error for i in bad)
    served = sorted(rid for s in made for b in s.launched for rid in b if rid >= 0)
    assert served == [0, 2, 4]
    for r in reqs:
        if r.error is None:
            assert r.reports is not None and int(r.reports[0]) == r.rid and r.done >= r.arrival
        else:
            assert r.reports is None
    assert srv.held_bytes() <= srv.budget
    # host time per request, split by phase, and the loop's slow passes
    h = m["host_us_per_request"]
    assert set(h) == {"finish", "predict", "launch", "launch_copy", "launch_match_call"}
    assert all(v >= 0.0 for v in h.values()) and h["predict"] == 0.0  # no predictor
    assert len(m["slow_passes"]["longest_ms"]) == min(5, m["slow_passes"]["count"])


def test_autotune_search_with_fake_launches():
    """The search on the host: every grid point on every tile option, queue
    overflows skipped, the fastest candidate kept."""
    from ngap_b200 import autotune as at
    from ngap_b200.engine import NgapError
    lengths = np.full(40, 1000, dtype=np.int64)
    offsets = np.arange(40, dtype=np.int64) * 1000
    data = np.zeros(40000, np.uint8)
    nfa_of = np.zeros(40, np.int32)
    built, calls = [], []

    def make(opts):
        built.append(opts)
        return ("ts", opts["tile_mode"])

    def run(engine, ts, buf, offs, lens, nf, stream, params):
        calls.append((ts, dict(params)))
        assert len(buf) == int(lens.sum()) and len(offs) == len(lens) == len(nf)
        if params["queue_capacity"] == 1024:
            raise NgapError(6, "queue")
        cost = {"shared": 3.0, "global": 1.0}[ts[1]]
        return cost * params["window"] / 1024 + (0.5 if params["queue_capacity"] else 0.0)

    grid = {"window": [512, 1024], "queue_capacity": [0, 1024, 4096]}
    best, table = at.autotune(None, None, data, offsets, lengths, nfa_of, grid=grid, frac=0.1,
                              reps=2, tile_grid=[{"tile_mode": "shared"}, {"tile_mode": "global"}],
                              run=run, make_tableset=make)
    assert built == [{"tile_mode": "shared"}, {"tile_mode": "global"}]
    assert len(table) == 12 and sum(ms is None for _, ms in table) == 4
    assert best == {"window": 512, "queue_capacity": 0, "tiles": {"tile_mode": "global"}}
    # reps + 1 launches per candidate that did not overflow, one for those that did
    assert len(calls) == 8 * 3 + 4
    with pytest.raises(ValueError):
        at.autotune(None, None, data, offsets, lengths, nfa_of, tile_grid=[{}], run=run)



class FakePredictor:
    """Density per request from a table (rid -> entries per byte)."""

    def __init__(self, dens):
        self.dens = dens

    def density(self, reqs):
        return np.array([self.dens[r.rid] for r in reqs], np.float64)


def test_serving_isolation_keeps_heavy_requests_apart():
    """With isolation, requests predicted heavier than heavy_work never share a
    batch with light ones; slot 0 serves only light requests."""
    made = []

    def factory(i):
        made.append(FakeSlot(1000, polls=3))
        return made[-1]
    sizes = [100] * 12
    heavy_ids = {2, 5, 9}
    dens = {i: (50.0 if i in heavy_ids else 1.0) for i in range(12)}
    srv = sv.Server(None, predictor=FakePredictor(dens), slots=2, budget=1 << 30,
                    max_batch_bytes=10_000, chunk_lo=1 << 30, slot_factory=factory,
                    tables_bytes=0, isolate=True, heavy_work=1000.0, adapt_chunks=False)
    reqs = [sv.Request(i, 0, np.zeros(n, np.uint8), 0.0) for i, n in enumerate(sizes)]
    m = srv.run(reqs)
    assert m["requests"] == 12 and m["rejected"] == 0
    batches = [b for s in made for b in s.launched if -1 not in b]
    for b in batches:
        kinds = {rid in heavy_ids for rid in b}
        assert len(kinds) == 1, b  # never mixed
    assert all(not (set(b) & heavy_ids) for b in made[0].launched if -1 not in b)
    assert all(r.reports is not None and int(r.reports[0]) == r.rid for r in reqs)
    assert all(r.chunk == 0 for r in reqs)  # fixed chunks when adapt_chunks is off
