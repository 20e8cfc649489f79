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
* admission: the tables and every engine's buffers (input copy, report
  buffers, per-warp overflow stacks, unit plan) count against `budget` bytes
  of device memory; a batch is launched only when what it adds keeps the
  total within the budget, and a request that can never fit is rejected
  with an error instead of waiting forever;
* batches take the queue in arrival order; with a predictor, each request's
  work is predicted at arrival (density x length; "static" is the table
  rule's density, "learned" the MLP's on the request's own bytes) and can
  set its chunk length (cost_model.chunk_for: requests predicted denser than
  rho_ref get proportionally shorter chunks) and, with `isolate`, its lane:
  predicted-heavy requests are batched apart from the light ones, so a light
  request never waits for a heavy batch (Server.run);
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
    error: str = None               # set when the request can never be admitted


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


def features_host(datas, window=cm.ENTROPY_WINDOW):
    """host_features of several regions through the library's host
    implementation (ngap_features_host): one call, no device work."""
    from ._lib import check, lib
    n = len(datas)
    out = np.zeros((n, 258), np.float32)
    if n == 0:
        return out
    lens = np.array([len(d) for d in datas], np.uint64)
    offs = np.zeros(n, np.uint64)
    offs[1:] = np.cumsum(lens)[:-1]
    cat = np.ascontiguousarray(np.concatenate(datas) if lens.sum() else np.zeros(1, np.uint8),
                               dtype=np.uint8)
    check(lib().ngap_features_host(cat.ctypes.data, int(lens.sum()), offs.ctypes.data,
                                   lens.ctypes.data, n, int(window), out.ctypes.data))
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
    "learned" (the MLP on host features, its BF16 inference run on the host
    by ngap_mlp_predict_host)."""

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
        feats = features_host([r.data[:cm.REGION] for r in reqs])
        x = np.concatenate([feats, self.nfeat[nf]], axis=1).astype(np.float32)
        # on the host: the matching kernels hold every SM's registers while
        # batches run, so an inference kernel would wait for them to end
        return self.model.predict(nf, x, bf16=True, host=True)


class EngineSlot:
    """One engine on its own non-blocking CUDA stream with a pinned staging
    buffer: the unit the server launches batches on."""

    def __init__(self, tableset, device, max_batch_bytes):
        import torch
        from .engine import Engine
        self.torch = torch
        self.ts = tableset
        self.engine = Engine(device)
        self.stream = torch.cuda.Stream(device)
        self.pinned = torch.empty(max_batch_bytes, dtype=torch.uint8).pin_memory()
        self.event = None
        self.args = None
        self.spent = [0.0, 0.0]  # seconds copying requests into the staging buffer, in the match call

    def memory(self):
        return self.engine.memory()

    def launch(self, batch, params):
        t0 = time.perf_counter()
        buf = self.pinned.numpy()
        offs = np.zeros(len(batch), np.int64)
        lens = np.array([len(r.data) for r in batch], np.int64)
        pos = 0
        for i, r in enumerate(batch):
            offs[i] = pos
            buf[pos:pos + len(r.data)] = r.data
            pos += len(r.data)
        nfa = np.array([r.nfa for r in batch], np.int32)
        kw = dict(params, stream=self.stream.cuda_stream,
                  chunks=np.array([r.chunk for r in batch], np.int64))
        t1 = time.perf_counter()
        batch_match_async(self.engine, self.ts, buf[:pos], offs, lens, nfa, **kw)
        self.spent[0] += t1 - t0
        self.spent[1] += time.perf_counter() - t1
        self.event = self.torch.cuda.Event()
        self.event.record(self.stream)
        self.args = (offs, lens, nfa, kw, pos)

    def done(self):
        return self.event.query()

    def finish(self, nreq):
        """Waits for the batch; (per-request reports, device ms, kernel launches)."""
        offs, lens, nfa, kw, pos = self.args
        eng = self.engine
        try:
            eng.sync()
        except NgapError as ex:  # capacity exceeded: rerun with the defaults (same reports)
            if ex.status not in (6, 7):
                raise
            kw = dict(kw, queue_capacity=0, result_capacity=max(kw["result_capacity"] * 8, 8 * pos))
            batch_match_async(eng, self.ts, self.pinned.numpy()[:pos], offs, lens, nfa, **kw)
            eng.sync()
        reps, sids = batch_results(eng)
        return split_by_stream(reps, sids, nreq), sum(eng.times_ms()), eng.launches()


def padded_input(nbytes):
    """Bytes of an engine's input copy for a batch of nbytes (16-byte padded + 64)."""
    return ((int(nbytes) + 15) & ~15) + 64


class Server:
    """Continuous batching over `slots` engines sharing one tableset.

    Device-memory admission: the tables and every engine's buffers count
    against `budget` bytes. Engine buffers only grow (ngap_engine_memory), so
    a batch is launched on a slot only when what it would add to that
    engine (a larger input copy, a larger unit plan) keeps the total within
    the budget. Each engine's buffers (an input copy of max_batch_bytes,
    report buffers for `rep_cap` reports, per-warp overflow stacks) are
    allocated by a one-stream warm-up batch at construction, so they are
    counted from the start and never grow while serving; a budget that
    cannot hold the tables and those buffers raises ValueError. A request that
    can never be admitted (longer than max_batch_bytes, or needing more than
    the budget leaves with every engine as it is) is rejected at arrival:
    its `error` is set and it gets no reports.
    """

    UNIT_BYTES = 80  # device bytes of a unit record plus its share of a task record

    def __init__(self, tableset, predictor=None, rho_ref=2.0, slots=2, budget=1 << 30,
                 max_batch_bytes=64 << 20, device=0, queue_capacity=0,
                 algorithm="nonblockingpcgroups", base_chunk=2048, chunk_lo=256, chunk_hi=2048,
                 slot_factory=None, tables_bytes=None, isolate=False, heavy_work=None,
                 adapt_chunks=True, max_batch_requests=256):
        self.ts = tableset
        self.pred = predictor
        self.isolate = bool(isolate and predictor is not None and len(range(slots)) > 1)
        self.heavy_work = heavy_work
        self.adapt_chunks = adapt_chunks
        self.rho_ref = rho_ref
        self.base_chunk = base_chunk
        self.chunk_lo, self.chunk_hi = chunk_lo, chunk_hi
        self.budget = budget
        self.max_bytes = max_batch_bytes
        self.max_requests = max(1, int(max_batch_requests))
        self.queue_capacity = queue_capacity
        self.algorithm = algorithm
        self.rep_cap = max(1 << 16, max_batch_bytes // 4)
        if tables_bytes is None:
            tables_bytes = sum(t.device_bytes for t in getattr(tableset, "tables", []))
        self.tables_bytes = int(tables_bytes)
        tiles = [t.stats()["tiles"] for t in getattr(tableset, "tables", [])] or [1]
        self.max_tiles = max(tiles)
        make = slot_factory or (lambda i: EngineSlot(tableset, device, max_batch_bytes))
        self.slots = [make(i) for i in range(slots)]
        self.busy = [None] * slots      # (batch, launch time)
        self.batches = []               # (size, bytes, predicted work, device ms)
        self.launches = 0               # kernels launched by the served batches
        self.rejected = []              # requests that can never be admitted
        # allocate each engine's buffers now, for the largest batches: an input
        # copy of max_batch_bytes, report buffers, per-warp overflow stacks,
        # the unit plan of max_batch_bytes of the NFA with the most tiles at
        # the shortest chunk, and per-stream rows for max_batch_requests
        # streams. A buffer that grew while serving would be freed and
        # allocated again, and cudaFree waits for the whole device, that is
        # for the other slots' batches too.
        lo = max(1, int(chunk_lo)) if adapt_chunks else 0
        big = Request(-1, int(np.argmax(tiles)), np.zeros(max(16, max_batch_bytes), np.uint8), 0.0)
        big.chunk = lo
        k = self.max_requests
        each = max(1, max_batch_bytes // k)
        many = [Request(-2 - i, i % len(tiles), np.zeros(each, np.uint8), 0.0) for i in range(k)]
        for r in many:
            r.chunk = lo
        for sl in self.slots:
            for warm in ([big], many):
                sl.launch(warm, self._params())
                sl.finish(len(warm))
        self.mem = [sl.memory() for sl in self.slots]
        if self.tables_bytes + sum(self._held(m) for m in self.mem) > budget:
            raise ValueError(f"a budget of {budget} bytes does not hold the tables "
                             f"({self.tables_bytes}) and the engines' fixed buffers "
                             f"({sum(self._held(m) for m in self.mem)})")

    def _params(self):
        return dict(algorithm=self.algorithm, result_capacity=self.rep_cap,
                    queue_capacity=self.queue_capacity)

    @staticmethod
    def _held(m):
        return m["input"] + m["reports"] + m["scratch"] + m["plan"]

    def held_bytes(self):
        """Device bytes held now: tables plus every engine's buffers."""
        return self.tables_bytes + sum(self._held(m) for m in self.mem)

    def _growth(self, s, nbytes, nreq):
        """Bytes slot s's engine would add for a batch of nbytes in nreq streams:
        a larger input copy, and room for a unit plan at the shortest chunk."""
        m = self.mem[s]
        plan = self.UNIT_BYTES * self.max_tiles * (nbytes // max(1, self.chunk_lo) + 2 * nreq)
        return max(0, padded_input(nbytes) - m["input"]) + max(0, plan - m["plan"])

    def _fits(self, s, nbytes, nreq):
        return self.held_bytes() + self._growth(s, nbytes, nreq) <= self.budget

    def admissible(self, r):
        """Whether request r alone could ever be admitted (engines never shrink)."""
        n = len(r.data)
        return n <= self.max_bytes and any(self._fits(s, n, 1) for s in range(len(self.slots)))

    def _form(self, queue, s):
        """Requests for the next batch on slot s, in arrival order, while the
        batch fits max_batch_bytes and the device-memory budget (removed from
        queue)."""
        n, nbytes = 0, 0
        while n < len(queue) and n < self.max_requests:
            nb = nbytes + len(queue[n].data)
            if nb > self.max_bytes or not self._fits(s, nb, n + 1):
                break
            n, nbytes = n + 1, nb
        chosen = queue[:n]
        del queue[:n]
        return chosen

    def _finish(self, s):
        batch, _ = self.busy[s]
        per, dev_ms, launches = self.slots[s].finish(len(batch))
        self.launches += launches
        self.mem[s] = self.slots[s].memory()
        t = time.perf_counter() - self._t0
        for r, rep in zip(batch, per):
            r.reports = rep
            r.done = t
        self.batches.append((len(batch), sum(len(r.data) for r in batch),
                             sum(r.pred_work for r in batch), dev_ms))
        self.busy[s] = None

    def run(self, requests):
        """Serves requests (sorted by arrival) in real time; returns metrics.

        Requests that arrived since the last pass of the loop are predicted
        together (one model call, inside the clock, while earlier batches may
        still run): their work (density x length) and, with adapt_chunks,
        their chunk length. Without isolation, batches take the queue in arrival order.
        With isolation (a predictor and at least two slots), a request whose
        predicted work exceeds heavy_work goes to the heavy queue: slot 0
        serves only the light queue, the other slots the heavy queue first
        and the light one when it is empty, so that light requests never
        share a batch with (and wait for) a predicted-heavy one."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        pending, light, heavy, nxt = [], [], [], 0
        self._spent0 = [sum(getattr(sl, "spent", [0.0, 0.0])[i] for sl in self.slots)
                        for i in range(2)]
        self._t0 = time.perf_counter()
        slow = []  # passes of the loop longer than 10 ms: (ms, finish, predict, launch ms)
        spent = [0.0, 0.0, 0.0]  # seconds in finish, predict and launch over the run
        while (nxt < len(reqs) or pending or light or heavy
               or any(b is not None for b in self.busy)):
            now = time.perf_counter() - self._t0
            t_fin = t_pred = t_launch = 0.0
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                r = reqs[nxt]
                nxt += 1
                if self.admissible(r):
                    pending.append(r)
                else:
                    r.error = (f"request of {len(r.data)} bytes can never be admitted "
                               f"(max_batch_bytes {self.max_bytes}, budget {self.budget})")
                    r.done = now
                    self.rejected.append(r)
            for s, b in enumerate(self.busy):
                if b is not None and self.slots[s].done():
                    t1 = time.perf_counter()
                    self._finish(s)
                    t_fin += time.perf_counter() - t1
            # predict as soon as requests arrive (while slots may still be busy,
            # so that the model's cost overlaps the device work), all of them
            # in one call
            if pending:
                if self.pred is not None:  # one prediction for everything that arrived
                    t1 = time.perf_counter()
                    rho = self.pred.density(pending)
                    t_pred += time.perf_counter() - t1
                    chunks = cm.chunk_for(rho, self.rho_ref, self.base_chunk, self.chunk_lo,
                                          self.chunk_hi)
                    for r, d, c in zip(pending, rho, chunks):
                        r.pred_work = float(d) * len(r.data)
                        r.chunk = int(c) if self.adapt_chunks else 0
                for r in pending:
                    if (self.isolate and self.heavy_work is not None
                            and r.pred_work > self.heavy_work):
                        heavy.append(r)
                    else:
                        light.append(r)
                pending = []
            for s in range(len(self.busy)):
                if self.busy[s] is not None:
                    continue
                if not self.isolate:
                    q = light if light else heavy
                elif s == 0:
                    q = light
                else:
                    q = heavy if heavy else light
                if q:
                    t1 = time.perf_counter()
                    batch = self._form(q, s)
                    if batch:
                        self.slots[s].launch(batch, self._params())
                        self.mem[s] = self.slots[s].memory()
                        self.busy[s] = (batch, now)
                    t_launch += time.perf_counter() - t1
            dt = time.perf_counter() - self._t0 - now
            spent[0] += t_fin
            spent[1] += t_pred
            spent[2] += t_launch
            if dt > 0.01:
                slow.append((dt * 1e3, t_fin * 1e3, t_pred * 1e3, t_launch * 1e3))
            if (not pending and not light and not heavy and nxt < len(reqs)
                    and all(b is None for b in self.busy)):
                time.sleep(max(0.0, min(reqs[nxt].arrival - now, 0.0005)))
        m = summarize([r for r in reqs if r.error is None], self.batches,
                      rejected=len(self.rejected))
        m["slow_passes"] = {"count": len(slow), "longest_ms": sorted(slow, reverse=True)[:5]}
        nreq = max(1, len(reqs))
        m["host_us_per_request"] = {k: 1e6 * v / nreq
                                    for k, v in zip(("finish", "predict", "launch"), spent)}
        # launch, split: copying requests into the slots' staging buffers and
        # the batched match call itself (plan, copies, kernel launches)
        split = [sum(getattr(sl, "spent", [0.0, 0.0])[i] for sl in self.slots) for i in range(2)]
        m["host_us_per_request"].update({"launch_copy": 1e6 * (split[0] - self._spent0[0]) / nreq,
                                         "launch_match_call": 1e6 * (split[1] - self._spent0[1]) / nreq})
        return m


def summarize(reqs, batches, rejected=0):
    lat = np.array([(r.done - r.arrival) * 1e3 for r in reqs])
    nbytes = sum(len(r.data) for r in reqs)
    span = max(r.done for r in reqs) - min(r.arrival for r in reqs) if reqs else 0.0
    return {"requests": len(reqs), "bytes": nbytes,
            "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
            "mean_ms": float(lat.mean()) if len(lat) else None,
            "MBps": nbytes / span / 1e6 if span > 0 else None,
            "batches": len(batches), "rejected": rejected,
            "mean_batch": float(np.mean([b[0] for b in batches])) if batches else 0.0}
