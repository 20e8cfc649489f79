"""The allocation-free report sort (ngap_reports_sort_unique_noalloc).

It serves callers that cannot call cudaMalloc (device memory owned by another
allocator, or loops that cannot take cudaMalloc's implicit synchronisation):
its scratch is a static device array. This file is collected last so that a
run stopping at the first failure has run every other test before it.
"""
import ctypes

import numpy as np
import pytest

import ngap_b200 as nb
from ngap_b200._lib import check, lib

pytestmark = pytest.mark.gpu

MAX_REPORTS = 1 << 18


def _reports(seed, n, ids=5000, offsets=1 << 24):
    rng = np.random.default_rng(seed)
    sid = rng.integers(0, ids, size=n, dtype=np.uint64)
    grp = rng.integers(0, 7, size=n, dtype=np.uint64) << np.uint64(22)
    off = rng.integers(0, offsets, size=n, dtype=np.uint64)
    r = ((sid | grp) << np.uint64(32)) | off
    dup = r[rng.integers(0, n, size=n // 3)]
    out = np.concatenate([r, dup])
    rng.shuffle(out)
    return out


def _noalloc(torch, d_in, n, d_out):
    nout = ctypes.c_uint64()
    stream = torch.cuda.current_stream().cuda_stream
    check(lib().ngap_reports_sort_unique_noalloc(ctypes.c_void_p(d_in.data_ptr()), n,
                                                  ctypes.c_void_p(d_out.data_ptr()),
                                                  ctypes.byref(nout), ctypes.c_void_p(stream)))
    return nout.value


def _host_unique(rep):
    """numpy sort by (offset, id) and unique, in the reference encoding."""
    key = ((rep & np.uint64(0xFFFFFFFF)) << np.uint64(32)) | (rep >> np.uint64(32))
    uk = np.unique(key)
    return (uk << np.uint64(32)) | (uk >> np.uint64(32))


def _exact(seed, n):
    """Exactly n reports (about a third of them duplicates)."""
    rep = _reports(seed, max(1, (3 * n) // 4 + 1))
    return np.resize(rep, n)


def test_noalloc_matches_sort_unique(engine):
    import torch
    for seed, n in ((1, 150_000), (2, 60_000)):  # two calls in a row, different sizes
        rep = _reports(seed, n)
        assert len(rep) <= MAX_REPORTS
        d_in = torch.from_numpy(rep.view(np.int64)).cuda()
        d_ref = torch.empty_like(d_in)
        d_new = torch.full_like(d_in, -1)
        n_ref = engine.sort_unique_device(d_in.data_ptr(), len(rep), d_ref.data_ptr(),
                                          stream=torch.cuda.current_stream().cuda_stream)
        n_new = _noalloc(torch, d_in, len(rep), d_new)
        torch.cuda.synchronize()
        assert n_new == n_ref
        got = d_new[:n_new].cpu().numpy().view(np.uint64)
        want = d_ref[:n_ref].cpu().numpy().view(np.uint64)
        assert np.array_equal(got, want)
        # and against a host sort by (offset, id) + unique
        assert np.array_equal(got, _host_unique(rep))


@pytest.mark.parametrize("n", [1, 2047, 2049, MAX_REPORTS])
def test_noalloc_edge_sizes(engine, n):
    """One report, either side of a 2048-key sort tile, and the full scratch."""
    import torch
    rep = _exact(10 + n, n)
    assert len(rep) == n
    d_in = torch.from_numpy(rep.view(np.int64)).cuda()
    d_out = torch.full_like(d_in, -1)
    n_new = _noalloc(torch, d_in, n, d_out)
    d_ref = torch.empty_like(d_in)
    n_ref = engine.sort_unique_device(d_in.data_ptr(), n, d_ref.data_ptr(),
                                      stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    got = d_out[:n_new].cpu().numpy().view(np.uint64)
    assert n_new == n_ref and np.array_equal(got, d_ref[:n_ref].cpu().numpy().view(np.uint64))
    assert np.array_equal(got, _host_unique(rep))


def test_noalloc_in_place(engine):
    """d_out may be d_in: the input is read into the scratch before any pass
    writes the output."""
    import torch
    rep = _reports(21, 90_000)
    d = torch.from_numpy(rep.view(np.int64)).cuda()
    n_new = _noalloc(torch, d, len(rep), d)
    torch.cuda.synchronize()
    assert np.array_equal(d[:n_new].cpu().numpy().view(np.uint64), _host_unique(rep))


def test_noalloc_rejects_oversize(engine):
    import torch
    d = torch.zeros(8, dtype=torch.int64, device="cuda")
    nout = ctypes.c_uint64()
    rc = lib().ngap_reports_sort_unique_noalloc(ctypes.c_void_p(d.data_ptr()), MAX_REPORTS + 1,
                                                ctypes.c_void_p(d.data_ptr()), ctypes.byref(nout),
                                                None)
    assert rc == 1  # NGAP_E_INVALID
    assert "262144" in nb._lib.last_error()
