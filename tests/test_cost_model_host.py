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


def _server(budget, max_bytes, held=()):
    s = sv.Server.__new__(sv.Server)  # the admission rule only: no engines or streams
    s.budget, s.max_bytes = budget, max_bytes
    s.busy = [(None, None, h, None) for h in held] + [None]
    return s


def test_serving_admission():
    reqs = [sv.Request(i, 0, np.zeros(n, np.uint8), 0.0) for i, n in enumerate([40, 30, 20, 50])]
    q = list(reqs)
    s = _server(budget=1000, max_bytes=90)  # batch capped by max_batch_bytes, in arrival order
    assert [r.rid for r in s._form(q)] == [0, 1, 2] and [r.rid for r in q] == [3]
    q = list(reqs)
    s = _server(budget=100, max_bytes=1000, held=(35,))  # 65 bytes free under the budget
    assert [r.rid for r in s._form(q)] == [0] and len(q) == 3
    q = list(reqs)
    s = _server(budget=100, max_bytes=1000, held=(80,))  # the first request does not fit: none
    assert s._form(q) == [] and len(q) == 4


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
