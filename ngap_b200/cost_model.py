"""Learned scheduler: predicts the worklist work of input regions and sets the
engine's chunk lengths and queue capacity from the prediction.

The reference records the fetched worklist length per round
(--motivate-worklist-length, code/src/ngap/kernel_ngap_OA.cu:366-369,
code/src/ngap/ngap.cu:1843-1866) and sizes its adaptive always-active interval
from the longest prefix-table list (kernel_ngap_OA.cu:180-194). Here:

* the engine records the work (entries expanded + injected) of every unit it
  runs (ngap_engine_set_trace / ngap_trace_copy); traces are aggregated per
  region of REGION bytes of each stream into worklist entries per input byte,
  the "frontier size" the model predicts;
* features of a region: its 256-bin symbol histogram and windowed Shannon
  entropy (computed on the GPU, ngap_features) plus statistics of its NFA's
  tables (states, edges, always-active states, prefix depth, byte classes,
  longest and mean list, expected list length per position);
* StaticModel is the fallback: the tables' expected list length per position
  (all keys equally likely), doubled for the expansions that follow each
  injected state; it never looks at the input. NfaMeanModel is a calibrated
  baseline: the mean traced density of each NFA. LearnedModel is the 2 x 64
  MLP of ngap_mlp_* (FP32 training, BF16 or FP32 inference) on the log of the
  density;
* chunk_for / plan turn per-stream predictions into per-stream chunk lengths
  (shorter for denser streams) and queue_for into a queue capacity. Neither
  changes any report: they only reshape the work.
"""
import ctypes
import math

import numpy as np

from . import _lib
from ._lib import check, lib
from .engine import as_u8, batch_match_async

REGION = 1 << 14          # bytes per feature region
ENTROPY_WINDOW = 1024     # bytes per entropy window
NFA_FEATURES = 8
IN_DIM = _lib.FEAT_BYTES + NFA_FEATURES


def nfa_features(stats):
    """Fixed-size feature vector of one NFA's tables (dict from Tables.stats())."""
    l2 = lambda v: math.log2(1.0 + float(v))
    return np.array([l2(stats["states"]) / 20, l2(stats["edges"]) / 20, l2(stats["aas"]) / 16,
                     stats["depth"] / 12, stats["max_nlive"] / 256, l2(stats["max_list"]) / 16,
                     l2(stats["cutoff"]) / 16, l2(stats["exp_list"]) / 8], dtype=np.float32)


def regions_of(offsets, lengths, region=REGION):
    """Split every stream into regions of `region` bytes (the last one
    shorter). Returns (stream index, start in stream, length) arrays."""
    st, start, ln = [], [], []
    for i, L in enumerate(np.asarray(lengths, dtype=np.int64)):
        for a in range(0, int(L), region):
            st.append(i)
            start.append(a)
            ln.append(min(region, int(L) - a))
    return (np.array(st, dtype=np.int64), np.array(start, dtype=np.int64),
            np.array(ln, dtype=np.int64))


def byte_features(data, offsets, reg_stream, reg_start, reg_len, window=ENTROPY_WINDOW,
                  stream=None):
    """ngap_features over the regions: [n, 258] float32 (data: host uint8 array
    or CUDA tensor)."""
    n = len(reg_stream)
    out = np.zeros((n, _lib.FEAT_BYTES), dtype=np.float32)
    if n == 0:
        return out
    offs = (np.asarray(offsets, dtype=np.uint64)[reg_stream] + reg_start.astype(np.uint64))
    lens = reg_len.astype(np.uint64)
    if hasattr(data, "data_ptr"):
        ptr, on_dev, nbytes = data.data_ptr(), 1, data.numel()
    else:
        arr = as_u8(data)
        ptr, on_dev, nbytes = arr.ctypes.data, 0, arr.nbytes
    check(lib().ngap_features(ctypes.c_void_p(ptr), nbytes, on_dev, offs.ctypes.data,
                              lens.ctypes.data, n, window, out.ctypes.data,
                              ctypes.c_void_p(stream or 0)))
    return out


def region_density(trace, reg_stream, reg_start, reg_len, region=REGION):
    """Worklist entries per input byte of each region, from unit records
    (Engine.unit_trace()): a unit's work is spread over the regions its
    reported positions [lo, hi) overlap, in proportion to the overlap."""
    index = {}
    for k, (s, a) in enumerate(zip(reg_stream.tolist(), reg_start.tolist())):
        index[(s, a // region)] = k
    work = np.zeros(len(reg_stream), dtype=np.float64)
    for u in trace:
        s, lo, hi, w = int(u["stream"]), int(u["lo"]), int(u["hi"]), float(u["work"])
        if hi <= lo:
            continue
        r0, r1 = lo // region, (hi - 1) // region
        for r in range(r0, r1 + 1):
            a, b = max(lo, r * region), min(hi, (r + 1) * region)
            k = index.get((s, r))
            if k is not None and b > a:
                work[k] += w * (b - a) / (hi - lo)
    return work / np.maximum(reg_len, 1)


def relative_error(pred, true, floor=0.05):
    """|pred - true| / max(true, floor), per region."""
    return np.abs(pred - true) / np.maximum(true, floor)


class StaticModel:
    """Density from the tables alone: expected states injected per position
    (deepest prefix table, keys equally likely), times two for the
    expansions that follow them."""
    name = "static"

    def __init__(self, stats_per_nfa):
        self.rho = np.array([2.0 * max(s["exp_list"], 1e-3) for s in stats_per_nfa])

    def predict(self, nfa_of_region, feats=None):
        return self.rho[np.asarray(nfa_of_region)]


class NfaMeanModel:
    """Calibrated baseline: the byte-weighted mean traced density of each NFA."""
    name = "nfa_mean"

    def __init__(self, n_nfas):
        self.rho = np.full(n_nfas, 1.0)

    def fit(self, nfa_of_region, y, weight):
        for k in range(len(self.rho)):
            m = nfa_of_region == k
            if m.any():
                self.rho[k] = float(np.sum(y[m] * weight[m]) / np.sum(weight[m]))
        return self

    def predict(self, nfa_of_region, feats=None):
        return self.rho[np.asarray(nfa_of_region)]


class LearnedModel:
    """2 x 64 MLP (ngap_mlp_*) on standardised features, trained on
    log2(1 + density); predictions in BF16 (bf16=True) or FP32."""
    name = "learned"

    def __init__(self, device=0, seed=1, in_dim=IN_DIM):
        h = ctypes.c_void_p()
        check(lib().ngap_mlp_create(device, in_dim, 64, seed, ctypes.byref(h)))
        self._h = h
        self.in_dim = in_dim
        self.mu = np.zeros(in_dim, np.float32)
        self.sd = np.ones(in_dim, np.float32)
        self.loss = None

    def __del__(self):
        try:
            if self._h.value and _lib._lib is not None:
                _lib._lib.ngap_mlp_destroy(self._h)
                self._h = ctypes.c_void_p()
        except (AttributeError, TypeError):  # interpreter shutdown
            pass

    def _norm(self, x):
        return np.ascontiguousarray((x - self.mu) / self.sd, dtype=np.float32)

    def fit(self, x, density, epochs=60, batch=512, lr=1e-3):
        x = np.asarray(x, np.float32)
        self.mu = x.mean(axis=0)
        self.sd = x.std(axis=0) + 1e-3
        xn = self._norm(x)
        y = np.ascontiguousarray(np.log2(1.0 + np.asarray(density, np.float64)), dtype=np.float32)
        loss = ctypes.c_float()
        check(lib().ngap_mlp_train(self._h, xn.ctypes.data, y.ctypes.data, len(y), epochs, batch,
                                   ctypes.c_float(lr), ctypes.byref(loss)))
        self.loss = loss.value
        return self

    def predict_log(self, x, bf16=True, host=False):
        """log2(1 + density) per row: the inference kernel, or with host=True
        the library's host restatement of it (ngap_mlp_predict_host)."""
        xn = self._norm(np.asarray(x, np.float32))
        out = np.zeros(len(xn), np.float32)
        if len(xn):
            fn = lib().ngap_mlp_predict_host if host else lib().ngap_mlp_predict
            check(fn(self._h, xn.ctypes.data, len(xn), int(bool(bf16)), out.ctypes.data))
        return out

    def predict(self, nfa_of_region, feats, bf16=True, host=False):
        return np.maximum(np.exp2(self.predict_log(feats, bf16, host)) - 1.0, 0.0)

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(lib().ngap_mlp_set_params(self._h, p.ctypes.data, len(p)))

    def params(self):
        n = ctypes.c_int64()
        check(lib().ngap_mlp_get_params(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, np.float32)
        check(lib().ngap_mlp_get_params(self._h, out.ctypes.data, n.value, ctypes.byref(n)))
        return out


def region_table(data, offsets, lengths, nfa_of, tables, region=REGION):
    """Regions of every stream with their features: dict with stream, start,
    len, nfa and x ([n, IN_DIM])."""
    rs, ra, rl = regions_of(offsets, lengths, region)
    nf = np.asarray(nfa_of)[rs]
    bf = byte_features(data, offsets, rs, ra, rl)
    stats = [t.stats() for t in tables]
    nfeat = np.stack([nfa_features(s) for s in stats])
    x = np.concatenate([bf, nfeat[nf]], axis=1).astype(np.float32)
    return {"stream": rs, "start": ra, "len": rl, "nfa": nf, "x": x, "stats": stats}


def collect(engine, tableset, data, offsets, lengths, nfa_of, regions, **params):
    """One traced batched match: the density of every region (entries/byte)."""
    engine.set_trace(True)
    try:
        batch_match_async(engine, tableset, data, offsets, lengths, nfa_of, **params)
        engine.sync()
        trace = engine.unit_trace()
    finally:
        engine.set_trace(False)
    return region_density(trace, regions["stream"], regions["start"], regions["len"])


def stream_density(pred, reg_stream, reg_len, nstreams):
    """Byte-weighted mean predicted density of every stream."""
    num = np.bincount(reg_stream, weights=pred * reg_len, minlength=nstreams)
    den = np.bincount(reg_stream, weights=reg_len, minlength=nstreams)
    return num / np.maximum(den, 1)


def chunk_for(rho, rho_ref, base_chunk=2048, lo=256, hi=8192):
    """Chunk length of a stream of predicted density rho (entries per byte):
    base_chunk at the reference density rho_ref, scaled by
    (1 + rho_ref) / (1 + rho) (a unit's serial time grows with the positions
    it looks up and the entries it expands), clamped to [lo, hi]."""
    rho = np.maximum(np.asarray(rho, np.float64), 0.0)
    return np.clip(np.round(base_chunk * (1.0 + rho_ref) / (1.0 + rho)), lo, hi).astype(np.int64)


def queue_for(rho_max):
    """Overflow entries per warp: four windows of 1024 positions at the
    densest predicted stream, between 4096 and 65536. A run that needs more
    fails with NGAP_E_OVERFLOW_QUEUE and is rerun with the default."""
    need = max(4 * 1024 * float(rho_max), 1.0)
    return int(min(1 << 16, max(1 << 12, 1 << int(math.ceil(math.log2(need))))))


def plan(rho, lengths, base_chunk=2048, lo=256, hi=8192):
    """Per-stream chunk lengths (chunk_for, reference density = the
    byte-weighted median of rho) and a queue capacity (queue_for)."""
    lengths = np.asarray(lengths, np.float64)
    rho = np.maximum(np.asarray(rho, np.float64), 0.0)
    if len(rho) == 0:
        return np.zeros(0, np.int64), 1 << 16
    order = np.argsort(rho)
    cum = np.cumsum(lengths[order])
    ref = rho[order][min(len(order) - 1, int(np.searchsorted(cum, cum[-1] / 2)))]
    return chunk_for(rho, ref, base_chunk, lo, hi), queue_for(rho.max())
