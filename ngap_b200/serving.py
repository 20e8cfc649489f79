"""Serving loop: match requests against resident NFA tables with continuous
batching, device-memory admission and per-request latency.

The reference has no serving path: each run matches one input against one
NFA (code/src/ngap/main.cu:81-131), and its "latency" is the throughput of a
single 1 MB input. Here:

* the tables of every NFA stay on the device in one tableset;
* requests (NFA id, bytes) arrive over time; whenever one of `slots`
  engines (each on its own CUDA stream) is free, the scheduler forms a batch
  from the queued requests and launches it with ngap_batch_match, so that
  requests arriving while others run are admitted as slots and memory free
  up, and batches on different slots overlap on the device;
* admission: a batch is launched only while the input bytes held by
  in-flight batches stay within `budget` bytes of device memory (each
  engine's report buffers are sized once, for `max_batch_bytes`);
* batches take the queue in arrival order; the scheduler sets each
  request's chunk length from its predicted density (cost_model.chunk_for:
  a unit's serial time bounds a batch's latency, so requests predicted
  denser than rho_ref get proportionally shorter chunks, never longer than
  chunk_hi) and the queue capacity from the densest prediction; "default"
  uses the engine's fixed chunks, "static" the table rule's prediction,
  "learned" the MLP's;
* each request's reports are exactly those of matching it alone
  (tests/test_gpu_cost_model.py checks this for every scheduler).
"""
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import cost_model as cm
from .engine import NgapError, batch_match_async, batch_results, split_by_stream


@dataclass
class Request:
    rid: int
    nfa: int
    data: np.ndarray
    arrival: float                  # seconds from the start of the run
    pred_work: float = 0.0          # predicted worklist entries
    chunk: int = 0                  # chunk length for the request's stream (0 = default)
    done: float = -1.0              # completion time (seconds from the start)
    reports: np.ndarray = field(default=None, repr=False)


def make_requests(pool, nfa_of_stream, n_nfas, rate=2000.0, duration=2.0, median=64 << 10,
                  sigma=1.5, max_len=4 << 20, seed=5):
    """Poisson arrivals at `rate` per second for `duration` seconds; the NFA is
    uniform over n_nfas, the length log-normal (median, sigma) capped at
    max_len, the bytes a window of a random stream of that NFA from `pool`
    (a list of per-stream uint8 arrays)."""
    rng = np.random.default_rng(seed)
    by_nfa = [np.nonzero(np.asarray(nfa_of_stream) == k)[0] for k in range(n_nfas)]
    reqs, t, rid = [], 0.0, 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        k = int(rng.integers(n_nfas))
        L = int(min(max_len, max(1, round(median * math.exp(sigma * rng.standard_normal())))))
        src = pool[int(by_nfa[k][rng.integers(len(by_nfa[k]))])]
        rot = int(rng.integers(len(src)))
        reqs.append(Request(rid, k, np.resize(np.roll(src, -rot), L), t))
        rid += 1
    return reqs


def host_features(data, window=cm.ENTROPY_WINDOW):
    """The byte features of ngap_features for one region, computed on the host:
    normalised 256-bin histogram, then mean and largest windowed entropy / 8."""
    L = len(data)
    out = np.zeros(258, np.float32)
    if L == 0:
        return out
    nwin = 1 if L < window else L // window
    wl = L if L < window else window
    c = np.bincount(_window_base(nwin, wl) + data[:nwin * wl], minlength=nwin * 256)
    c = c.reshape(nwin, 256)
    hist = c.sum(axis=0)
    if nwin * wl < L:
        hist = hist + np.bincount(data[nwin * wl:], minlength=256)
    out[:256] = hist / L
    q = c / wl
    h = -np.sum(q * np.log2(np.where(q > 0, q, 1.0)), axis=1)
    out[256] = h.mean() / 8
    out[257] = h.max() / 8
    return out


_bases = {}


def _window_base(nwin, wl):
    """256 * window index of every byte of nwin windows of wl bytes (cached)."""
    k = (nwin, wl)
    if k not in _bases:
        _bases[k] = (np.arange(nwin * wl, dtype=np.int64) // wl) * 256
    return _bases[k]


class Predictor:
    """Predicted worklist entries of a request: density (entries per byte)
    of its first region times its length. kind: "static" (table rule) or
    "learned" (MLP, BF16 inference on host features)."""

    def __init__(self, kind, tables, model=None):
        self.kind = kind
        self.stats = [t.stats() for t in tables]
        self.nfeat = np.stack([cm.nfa_features(s) for s in self.stats])
        self.static = cm.StaticModel(self.stats)
        self.model = model

    def density(self, reqs):
        nf = np.array([r.nfa for r in reqs], dtype=np.int64)
        if self.kind != "learned":
            return self.static.predict(nf)
        x = np.stack([np.concatenate([host_features(r.data[:cm.REGION]), self.nfeat[r.nfa]])
                      for r in reqs]).astype(np.float32)
        return self.model.predict(nf, x, bf16=True)


class Server:
    """Continuous batching over `slots` engines sharing one tableset."""

    def __init__(self, tableset, predictor=None, rho_ref=2.0, slots=2, budget=1 << 30,
                 max_batch_bytes=64 << 20, device=0, queue_capacity=0,
                 algorithm="nonblockingpcgroups", base_chunk=2048, chunk_lo=256, chunk_hi=2048):
        import torch
        from .engine import Engine
        self.torch = torch
        self.ts = tableset
        self.pred = predictor
        self.rho_ref = rho_ref
        self.base_chunk = base_chunk
        self.chunk_lo, self.chunk_hi = chunk_lo, chunk_hi
        self.budget = budget
        self.max_bytes = max_batch_bytes
        self.queue_capacity = queue_capacity
        self.algorithm = algorithm
        self.engines = [Engine(device) for _ in range(slots)]
        self.streams = [torch.cuda.Stream(device) for _ in range(slots)]
        self.pinned = [torch.empty(max_batch_bytes, dtype=torch.uint8).pin_memory()
                       for _ in range(slots)]
        self.rep_cap = max(1 << 16, max_batch_bytes // 4)
        self.busy = [None] * slots      # (batch, event, held bytes, launch arguments)
        self.batches = []               # (size, bytes, predicted work, device ms)
        self.launches = 0               # kernels launched by the served batches

    def _held(self):
        return sum(b[2] for b in self.busy if b is not None)

    def _reserve(self, nbytes):
        """Device bytes a batch holds while in flight: its input (the report
        buffers are sized once per engine, `rep_cap` reports)."""
        return nbytes

    def _launch(self, slot, batch):
        buf = self.pinned[slot].numpy()
        offs = np.zeros(len(batch), np.int64)
        lens = np.array([len(r.data) for r in batch], np.int64)
        pos = 0
        for i, r in enumerate(batch):
            offs[i] = pos
            buf[pos:pos + len(r.data)] = r.data
            pos += len(r.data)
        nfa = np.array([r.nfa for r in batch], np.int32)
        eng, st = self.engines[slot], self.streams[slot]
        kw = dict(algorithm=self.algorithm, result_capacity=self.rep_cap,
                  stream=st.cuda_stream, queue_capacity=self.queue_capacity,
                  chunks=np.array([r.chunk for r in batch], np.int64))
        batch_match_async(eng, self.ts, buf[:pos], offs, lens, nfa, **kw)
        ev = self.torch.cuda.Event()
        ev.record(st)
        self.busy[slot] = (batch, ev, self._reserve(pos), (offs, lens, nfa, kw, pos))

    def _finish(self, slot, now):
        batch, ev, held, (offs, lens, nfa, kw, pos) = self.busy[slot]
        eng = self.engines[slot]
        try:
            eng.sync()
        except NgapError as ex:  # capacity exceeded: rerun with the defaults (same reports)
            if ex.status not in (6, 7):
                raise
            kw = dict(kw, queue_capacity=0, result_capacity=max(kw["result_capacity"] * 8, 8 * pos))
            batch_match_async(eng, self.ts, self.pinned[slot].numpy()[:pos], offs, lens, nfa, **kw)
            eng.sync()
        dev_ms = sum(eng.times_ms())
        self.launches += eng.launches()
        reps, sids = batch_results(eng)
        per = split_by_stream(reps, sids, len(batch))
        t = time.perf_counter() - self._t0
        for r, rep in zip(batch, per):
            r.reports = rep
            r.done = t
        self.batches.append((len(batch), pos, sum(r.pred_work for r in batch), dev_ms))
        self.busy[slot] = None

    def _form(self, queue):
        """Requests for the next batch, in arrival order, while the batch fits
        max_batch_bytes and the in-flight bytes fit the budget (removed from
        queue)."""
        free = self.budget - self._held()
        n, nbytes = 0, 0
        while n < len(queue):
            nb = nbytes + len(queue[n].data)
            if nb > self.max_bytes or self._reserve(nb) > free:
                break
            n, nbytes = n + 1, nb
        chosen = queue[:n]
        del queue[:n]
        return chosen

    def run(self, requests):
        """Serves requests (sorted by arrival) in real time; returns metrics."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        queue, nxt = [], 0
        self._t0 = time.perf_counter()
        while nxt < len(reqs) or queue or any(b is not None for b in self.busy):
            now = time.perf_counter() - self._t0
            first = nxt
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                queue.append(reqs[nxt])
                nxt += 1
            if self.pred is not None and nxt > first:  # predictions at arrival, inside the clock
                rho = self.pred.density(reqs[first:nxt])
                chunks = cm.chunk_for(rho, self.rho_ref, self.base_chunk, self.chunk_lo,
                                      self.chunk_hi)
                for r, d, c in zip(reqs[first:nxt], rho, chunks):
                    r.pred_work = float(d) * len(r.data)
                    r.chunk = int(c)
            for s, b in enumerate(self.busy):
                if b is not None and b[1].query():
                    self._finish(s, now)
            for s in range(len(self.busy)):
                if self.busy[s] is None and queue:
                    batch = self._form(queue)
                    if batch:
                        self._launch(s, batch)
            if not queue and nxt < len(reqs) and all(b is None for b in self.busy):
                time.sleep(max(0.0, min(reqs[nxt].arrival - now, 0.0005)))
        return summarize(reqs, self.batches)


def summarize(reqs, batches):
    lat = np.array([(r.done - r.arrival) * 1e3 for r in reqs])
    nbytes = sum(len(r.data) for r in reqs)
    span = max(r.done for r in reqs) - min(r.arrival for r in reqs) if reqs else 0.0
    return {"requests": len(reqs), "bytes": nbytes,
            "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
            "mean_ms": float(lat.mean()) if len(lat) else None,
            "MBps": nbytes / span / 1e6 if span > 0 else None,
            "batches": len(batches),
            "mean_batch": float(np.mean([b[0] for b in batches])) if batches else 0.0}
