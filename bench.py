"""Benchmark: input MB/s of the matching path on one B200.

The metric is input MB/s (10^6 bytes per second) with bit-exact reports,
plain vs batched+learned, with p99 latency (the reference's own throughput is
input bytes over the CUDA-event time of its kernels,
code/src/ngap/ngap.cu:1823-1827). The default run prints ONE JSON line:

* headline (value, e2e, roofline, cpu_baseline): the Hamming k-mer set — 1000
  random ACGT 25-mers with <= 3 substitutions (166k STEs), a 16 MiB ACGT stream
  with mutated copies every 64 KiB, 16 segments of 1 MiB (the reference's
  throughput runs use 1 MB segments), 10 groups, prefix memoization as deep as
  the table caps allow, algorithm nonblockingpcgroups. A step is one match of
  the whole stream plus the device sort/unique of its reports.
    value   inputs already in HBM (16 MiB < L2, so L2 is flushed between steps)
    e2e     through the public API with host buffers: every step a pinned H2D
            of the stream, the match and a D2H of the unique reports, as a
            stream of inputs (two engines on two streams take alternate
            steps, so a copy overlaps the other engine's matching); e2e.serial
            is one engine taking one step at a time
  parity_vs_oracle: two whole segments checked against the oracle in the
  same run, plus sortedness and range of the whole result.
* "batched": the batched suite (16 NFAs of 2k-200k STEs, 4096 streams of
  log-uniform length 1 KiB-4 MiB, about 2 GiB) in one persistent launch per
  step with autotuned parameters (CUDA-graph replay among the candidates),
  its e2e, the same streams matched one ngap_match per stream with
  nonblockingallgroups ("plain") against one batched launch, and per-stream
  parity on a random sample of streams (each stream's reports in its first
  64 KiB against the oracle on that prefix).
* "serving": Poisson arrivals at 2000/s over the same 16 NFAs, p50/p99
  latency and served MB/s for the default, static and learned schedulers, the
  frontier-prediction error of each predictor, and every request's reports
  equal across schedulers and, on a sample, to the oracle's.

Under torchrun each rank matches its own copy of the headline workload
(independent segments, no data-path collective): weak scaling; value = all
bytes / the slowest rank's time; the batched and serving parts run at N=1.

`--impl reference` times the reference CPU matcher automataGroupsReference
(code/src/ngap/ngap.cu:2171-2268) on a bounded sample of the same workload:
the reference's own compiled `ngap` command with --validation (oracle/_ref/ngap,
built from the reference sources by oracle/Makefile; it prints "Reference CPU
elapsed time", one OpenMP thread per (group, segment)) when it is present and
runs on this machine, else the oracle's C restatement of that loop over
group graphs made by the reference's own compiled front-end
(oracle/_ref/ref_frontend). The sample is the first S bytes of every one of
the 16 segments (all 160 (group, segment) units), S sized to a few seconds
of CPU work per step. ms_per_step is the mean sample time.

Other workloads (`--workload`): literal_set (plain single stream; its line
also compares blockinggroups with nonblockingallgroups), high_frontier,
batched_suite and serving (each alone).
"""
import argparse
import json
import os
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "input MB/s on 1 B200 (bit-exact reports), plain vs batched+learned; p99 latency"
SEG = 1 << 20
DATA = "synthetic (seeded generators with the benchmark configs' shapes; ANMLZoo is absent)"


def workload_args(name):
    from ngap_b200 import workloads as W
    if name == "hamming_set":
        anml, data = W.hamming_set(seed=2)
        return anml, data, dict(group_num=10, depth=-1, seg_len=SEG, algorithm="nonblockingpcgroups",
                                desc="1000 ACGT 25-mers, Hamming <= 3 (166k STEs), 16 MiB, 16 x 1 MiB segments")
    if name == "literal_set":
        anml, data = W.literal_set(seed=1)
        return anml, data, dict(group_num=1, depth=-1, seg_len=len(data), algorithm="nonblockingpcgroups",
                                desc="64 literals 8-16 B with classes (786 STEs), 1 MiB single segment")
    if name == "high_frontier":
        anml, data = W.high_frontier(seed=3)
        return anml, data, dict(group_num=10, depth=-1, seg_len=SEG, algorithm="nonblockingpcgroups",
                                desc="500 Levenshtein-2 20-mers + 2000 lit.*lit, 32 MiB, 32 x 1 MiB segments")
    raise SystemExit(f"unknown workload {name}")


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled(workload, num_seg):
    """ncu figures of the matching kernel (DRAM and L2 bytes per launch, L2
    throughput) from the committed summary of the same workload and segment
    count, or None."""
    p = os.path.join(ROOT, "profiles", "match_kernel_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    v = d.get(workload)
    if v is None or int(v.get("num_seg", v.get("streams", -1))) != num_seg:
        return None
    return v


def host_info():
    """Host cores and CPU model of the machine the CPU figures ran on."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "cpu_model": model}


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML
    polled every few milliseconds from a thread (the timed regions are short).
    Without NVML the summary says "unsampled"."""
    REASONS = (("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20),
               ("hw_thermal_slowdown", 0x40), ("sw_power_cap", 0x4))

    def __init__(self, index, period_s=0.004):
        self.index = index
        self.period = period_s
        self.samples = []  # (sm_mhz, max_mhz, reasons bitmask)
        self.stop = threading.Event()
        self.t = None
        self.nvml = None

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        self.nvml = pynvml
        try:  # the CUDA device's PCI bus id names the same GPU in NVML
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            return pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _poll(self, h):
        nv = self.nvml
        mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        while True:
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                rs = int(nv.nvmlDeviceGetCurrentClocksThrottleReasons(h))
                self.samples.append((sm, mx, rs))
            except Exception:
                pass
            if self.stop.wait(self.period):
                break

    def __enter__(self):
        try:
            h = self._handle()
            self.t = threading.Thread(target=self._poll, args=(h,), daemon=True)
            self.t.start()
        except Exception:
            self.t = None
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.t:
            self.t.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [x[0] for x in self.samples]
        reasons = sorted({n for _, _, r in self.samples for n, b in self.REASONS if r & b})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(x[1] for x in self.samples),
                "reasons": reasons, "samples": len(sm), "source": "nvml"}


def worklist_bytes(stats, n_in, n_reports, table_bytes):
    """Bytes of the reference's worklist formulation (input + per matched
    state 24 B of queue/CSR traffic + 8 B per successor tested + 8 B per
    report + tables), from unique-frontier counts."""
    return (n_in + stats["matched"] * 24 + stats["matched_deg"] * 8 + n_reports * 8 + table_bytes)


def frontier_stats(views, data, seg_len, nbytes):
    """Unique-frontier counts per input byte on the first nbytes of segment 0
    (oracle mode 1: bitmap-deduplicated frontier)."""
    from oracle import oracle
    n = min(nbytes, seg_len, len(data))
    _, st = oracle.match(views, data[:n], 1, n, mode=1, nthreads=os.cpu_count() or 1)
    return {k: v / n for k, v in st.items()}, n


def has_sticky(views):
    """True when some group has a state that is not always-active, accepts
    every byte and loops on itself (`.*`): the reference CPU loop as written
    re-adds such a state once per predecessor path and position, so its
    frontier grows without bound; the reference's --unique option bounds it."""
    def f(v, k):
        return v[k] if isinstance(v, dict) else getattr(v, k)
    for v in views:
        ro, co = f(v, "row_offsets"), f(v, "col_indices")
        full = np.all(np.asarray(f(v, "symbol_sets")).reshape(-1, 8) == 0xffffffff, axis=1)
        for s in np.nonzero(full & ((np.asarray(f(v, "node_attrs")) & 1) == 0))[0]:
            if s in co[ro[s]:ro[s + 1]]:
                return True
    return False


# ---------------------------------------------------------------------------
# CPU side: the reference's CPU matcher on a bounded sample


def sample_segments(data, seg_len, nseg, s):
    """The first s bytes of each of nseg segments, concatenated (a bounded
    sample that keeps every (group, segment) unit)."""
    return np.concatenate([data[i * seg_len:i * seg_len + s] for i in range(nseg)])


def ref_cpu_sample(anml_path, data, seg_len, nseg, group_num, s, tmpdir, timeout=900):
    """One run of the reference command on the sample of s bytes per segment:
    (reference CPU MB/s, CPU ms, reference GPU MB/s, record)."""
    from oracle import refcli
    smp = sample_segments(data, seg_len, nseg, s)
    ipath = os.path.join(tmpdir, f"sample_{s}.input")
    smp.tofile(ipath)
    args = refcli.command(anml_path, ipath, len(smp), "nonblockingallgroups", group_num, s,
                          depth=3, validation=True)
    rc, out = refcli.run(args, timeout)
    rec = refcli.parse(out)
    if rc != 0 or rec["cpu_ms"] is None:
        raise RuntimeError(f"reference command failed (rc {rc}): {out[-400:]}")
    return rec


def port_cpu_sample(views, data, seg_len, nseg, s, unique):
    """The oracle's restatement of the reference CPU loop (mode 0: as
    written) on the same sample, one thread per (group, segment) unit like
    the reference's OpenMP loop (ngap.cu:2182-2199), all host cores."""
    from oracle import oracle
    smp = sample_segments(data, seg_len, nseg, s)
    t0 = time.time()
    _, st = oracle.match(views, smp, nseg, s, mode=0, unique=unique,
                         nthreads=os.cpu_count() or 1)
    dt = time.time() - t0
    return {"cpu_ms": dt * 1e3, "cpu_mbps": len(smp) / dt / 1e6, "stats": st}


class CpuBaseline:
    """The reference CPU matcher on bounded samples of a plain workload: the
    reference's own command when it runs here, else the oracle port over the
    reference front-end's graphs (else over the product's graphs, said so)."""

    def __init__(self, anml, data, cfg, product_views=None):
        from oracle import refcli
        self.tmp = tempfile.mkdtemp(prefix="ngap_bench_")
        self.anml_path = os.path.join(self.tmp, "workload.anml")
        with open(self.anml_path, "w") as f:
            f.write(anml)
        self.data, self.cfg = data, cfg
        self.seg_len = cfg["seg_len"]
        self.nseg = len(data) // self.seg_len
        self.kind, self.graphs = None, None
        self.note = ""
        if refcli.available():
            try:  # a tiny sample first: the command must run cleanly here
                ref_cpu_sample(self.anml_path, data, self.seg_len, self.nseg, cfg["group_num"],
                               256, self.tmp, timeout=600)
                self.kind = "reference"
            except Exception as ex:
                self.note = f"reference command unusable here ({str(ex)[:120]}); "
        if self.kind is None:
            self.kind = "port"
            try:
                self.views = _ref_views(self.anml_path, cfg["group_num"])
                self.note += "oracle port over the reference front-end's group graphs"
            except Exception:
                self.views = product_views
                self.note += "oracle port over the product's group graphs (reference front-end absent)"
            self.unique = has_sticky(self.views)

    def sample(self, s):
        """(MB/s, seconds, description) of one sample of s bytes per segment."""
        s = int(max(16, min(self.seg_len, s)))
        if self.kind == "reference":
            rec = ref_cpu_sample(self.anml_path, self.data, self.seg_len, self.nseg,
                                 self.cfg["group_num"], s, self.tmp)
            mbps, ms = rec["cpu_mbps"], rec["cpu_ms"]
            extra = {"reference_gpu_mbps": rec["gpu_mbps"], "validation": rec["validation"]}
        else:
            rec = port_cpu_sample(self.views, self.data, self.seg_len, self.nseg, s, self.unique)
            mbps, ms = rec["cpu_mbps"], rec["cpu_ms"]
            extra = {}
        desc = (f"first {s} B of each of the {self.nseg} segments ({s * self.nseg} B), "
                f"{self.cfg['group_num'] * self.nseg} (group, segment) units, one thread each")
        if self.kind == "port" and self.unique:
            desc += "; --unique (.* states)"
        return mbps, ms / 1e3, desc, extra

    def calibrated(self, seconds):
        """Sample size giving about `seconds` of CPU work: a small probe, then
        scaled (the loop's per-byte cost is steady)."""
        s0 = 4096
        _, t0, _, _ = self.sample(s0)
        if t0 < 0.2:  # too short to scale from reliably: one bigger probe
            s0 = int(min(self.seg_len, s0 * max(2.0, 0.5 / max(t0, 1e-3))))
            _, t0, _, _ = self.sample(s0)
        return int(max(256, min(self.seg_len, s0 * seconds / max(t0, 1e-3))))

    def cores(self):
        return min(os.cpu_count() or 1, self.cfg["group_num"] * self.nseg)


def _ref_views(anml_path, group_num):
    """Group graphs from the reference's own compiled front-end
    (oracle/_ref/ref_frontend), as oracle views: nothing of the product."""
    import subprocess
    from oracle import frontend
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_frontend")
    if not os.access(exe, os.X_OK):
        raise FileNotFoundError(exe)
    out = anml_path + f".g{group_num}.txt"
    subprocess.run([exe, anml_path, str(group_num), out], check=True, capture_output=True,
                   timeout=600)
    with open(out) as f:
        return frontend.parse_ref_dump(f.read())


# ---------------------------------------------------------------------------
# GPU side


def _dist_setup(world, local_rank):
    import torch
    torch.cuda.set_device(local_rank)
    if world <= 1:
        return None
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                            device_id=torch.device("cuda", local_rank))
    return dist


def _max_over_ranks(dist, x):
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


M32 = np.uint64(0xFFFFFFFF)
S32 = np.uint64(32)


def segment_parity(got, views, data, num_seg, seg_len, sample):
    """The whole result sorted by (offset, id), unique and inside the input,
    and equal to the oracle on each sampled segment (segments are matched
    independently; first_segment gives a segment the start-of-data rule of
    its place, code/src/ngap/ngap_buffer.cu:613-631)."""
    from oracle import oracle
    got = np.asarray(got, dtype=np.uint64)
    off, ids = got & M32, got >> S32
    key = (off << S32) | ids
    ok_sorted = bool(np.all(key[1:] > key[:-1]))
    ok_range = bool(got.size == 0 or int(off.max()) < num_seg * seg_len)
    per = {}
    t0 = time.time()
    for s in sample:
        lo = s * seg_len
        want, _ = oracle.match(views, data[lo:lo + seg_len], 1, seg_len, first_segment=s,
                               nthreads=os.cpu_count() or 1)
        want = np.asarray(want, dtype=np.uint64)
        want = (want & ~M32) | ((want & M32) + np.uint64(lo))
        mine = got[(off >= lo) & (off < lo + seg_len)]
        per[int(s)] = {"reports": int(len(want)), "equal": bool(np.array_equal(mine, want))}
    return {"bit_exact": ok_sorted and ok_range and all(v["equal"] for v in per.values()),
            "sorted_unique": ok_sorted, "offsets_in_range": ok_range,
            "segments_checked": per, "segments_total": int(num_seg),
            "oracle_seconds": round(time.time() - t0, 1)}


def run_plain(args, warmup, rank, world, local_rank, dist):
    """The plain single-stream line (headline): returns the JSON dict on rank 0."""
    import torch
    import ngap_b200 as nb

    anml, data, cfg = workload_args(args.workload)
    nfa = nb.Nfa.from_string(anml)
    groups = nb.Groups(nfa, group_num=cfg["group_num"])
    tables = nb.Tables(groups, device=local_rank, precompute_depth=cfg["depth"])
    eng = nb.Engine(local_rank)
    seg_len = cfg["seg_len"]
    num_seg = len(data) // seg_len
    if args.segments > 0:
        num_seg = min(num_seg, args.segments)
    n_in = num_seg * seg_len
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    d_in = torch.from_numpy(data[:n_in]).to(f"cuda:{local_rank}")
    h_pinned = torch.from_numpy(data[:n_in].copy()).pin_memory()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local_rank}")
    kw = dict(algorithm=cfg["algorithm"], stream=sh)

    def step_device():
        eng.match_async(tables, d_in, num_seg, seg_len, **kw)

    for _ in range(warmup):
        step_device()
        eng.sync()
    raw, uniq = eng.counts()
    first = eng.results()

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident timed region
    barrier()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    match_ms, launches = [], 0
    with ClockSampler(local_rank) as clk:
        for i in range(args.steps):
            flush.zero_()  # evict the 16 MiB stream from L2 (outside the step's events)
            evs[i][0].record(stream)
            step_device()
            evs[i][1].record(stream)
            eng.sync()
            match_ms.append(eng.times_ms()[0])
            launches += eng.launches()
        barrier()
    t_ms = _max_over_ranks(dist, float(sum(a.elapsed_time(b) for a, b in evs)))
    value = world * n_in * args.steps / (t_ms / 1e3) / 1e6

    # ---- end to end through the public API with host buffers, one step at a
    # time: pinned H2D copy, match, D2H of the unique reports (L2 flushed
    # before each step, outside its events)
    e2e_ms, d2h = [], 0
    barrier()
    res = first
    for i in range(args.steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        eng.match_async(tables, h_pinned.numpy(), num_seg, seg_len, **kw)
        eng.sync()
        res = eng.results()
        b.record(stream)
        torch.cuda.synchronize()
        e2e_ms.append(a.elapsed_time(b))
        d2h = res.nbytes + 40
    e2e_total = _max_over_ranks(dist, float(sum(e2e_ms)))
    e2e_serial = world * n_in * args.steps / (e2e_total / 1e3) / 1e6

    # ---- the same as a stream of inputs: two engines on two streams take
    # alternate steps, so one step's host copy overlaps the other's matching;
    # every step still copies its input from pinned host memory and reads its
    # reports back, and the time is the whole run's (CUDA events bracketing
    # all steps on the launching stream)
    eng2 = nb.Engine(local_rank)
    lanes = [(eng, torch.cuda.Stream(local_rank)), (eng2, torch.cuda.Stream(local_rank))]
    for e_, st_ in lanes:  # warm the second engine's plan and buffers
        e_.match_async(tables, h_pinned.numpy(), num_seg, seg_len, algorithm=cfg["algorithm"],
                       stream=st_.cuda_stream)
        e_.sync()
    barrier()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _, st_ in lanes:
        st_.wait_event(a)
    stream_res = []
    for i in range(args.steps):
        e_, st_ = lanes[i % 2]
        if i >= 2:  # this engine's previous step: wait, read its reports
            e_.sync()
            stream_res.append(e_.results())
        e_.match_async(tables, h_pinned.numpy(), num_seg, seg_len, algorithm=cfg["algorithm"],
                       stream=st_.cuda_stream)
    for i in range(max(0, args.steps - 2), args.steps):
        e_, _ = lanes[i % 2]
        e_.sync()
        stream_res.append(e_.results())
    for _, st_ in lanes:
        ev = torch.cuda.Event()
        ev.record(st_)
        stream.wait_event(ev)
    b.record(stream)
    torch.cuda.synchronize()
    e2e_stream_ms = _max_over_ranks(dist, a.elapsed_time(b))
    e2e_value = world * n_in * args.steps / (e2e_stream_ms / 1e3) / 1e6
    stream_same = all(np.array_equal(r_, first) for r_ in stream_res)

    algo_cmp = None
    if args.workload == "literal_set" and world == 1:
        # the plain single-stream case compares the blocking matcher with the
        # fully optimised non-blocking one (same device timing, outside the steps)
        algo_cmp = {}
        for name in ("blockinggroups", "nonblockingallgroups"):
            kw_a = dict(kw, algorithm=name)
            for _ in range(warmup):
                eng.match_async(tables, d_in, num_seg, seg_len, **kw_a)
                eng.sync()
            ms = []
            for _ in range(args.steps):
                flush.zero_()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                eng.match_async(tables, d_in, num_seg, seg_len, **kw_a)
                b.record(stream)
                eng.sync()
                ms.append(a.elapsed_time(b))
            algo_cmp[name] = {"MBps": n_in * len(ms) / (sum(ms) / 1e3) / 1e6,
                              "ms_per_step": float(np.mean(ms)),
                              "same_reports": bool(np.array_equal(eng.results(), res))}
    if rank != 0:
        return None
    peak, peak_kind = load_peaks()
    mk = float(np.mean(match_ms))
    line = {"metric": METRIC, "value": value, "unit": "MB/s", "n_gpus": world,
            "steps": args.steps, "warmup": warmup, "ms_per_step": t_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": DATA,
            "config": {"workload": args.workload, "desc": cfg["desc"],
                       "algorithm": cfg["algorithm"], "group_num": groups.count,
                       "precompute_depth": cfg["depth"], "num_seg": num_seg, "seg_len": seg_len,
                       "input_bytes": n_in, "l2": "flushed between steps (256 MiB write)"},
            "reports": {"raw": raw, "unique": uniq},
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "e2e": {"value": e2e_value, "unit": "MB/s", "h2d_bytes_per_step": n_in,
                    "d2h_bytes_per_step": d2h,
                    "how": "two engines on two streams take alternate steps (a stream of "
                           "inputs); each step: pinned H2D of the 16 MiB, match, D2H of the "
                           "unique reports; whole-run CUDA-event time",
                    "serial": {"value": e2e_serial, "how": "one engine, one step at a time, "
                               "L2 flushed before each step"}}}
    views = groups.views()
    if not args.no_check:
        rng = np.random.default_rng(12345)
        sample = sorted({0, int(rng.integers(1, num_seg))} if num_seg > 1 else {0})
        par = segment_parity(first, views, data, num_seg, seg_len, sample)
        par["same_every_step"] = bool(np.array_equal(res, first)) and bool(stream_same)
        par["bit_exact"] = par["bit_exact"] and par["same_every_step"]
        line["parity_vs_oracle"] = par
    if algo_cmp is not None:
        line["algorithms"] = algo_cmp
    # roofline of the matching kernel: bytes this design must move per launch
    # (every input byte, table byte and raw report once) over its CUDA-event
    # time; the measured DRAM and L2 bytes of the same launch from ncu; and
    # the reference's worklist formulation for comparison
    alg = n_in + tables.device_bytes + 8 * raw
    roof = {"bound": "hbm", "unit": "GB/s", "peak": peak, "peak_source": peak_kind,
            "kernel": "match_kernel", "kernel_ms": mk,
            "algorithmic_bytes": alg,
            "algorithmic_def": "input bytes + table bytes + 8 B per raw report, per launch",
            "achieved": alg / (mk / 1e3) / 1e9}
    roof["frac"] = roof["achieved"] / peak
    prof = profiled(args.workload, num_seg)
    roof["traffic"] = float(prof["dram_bytes_per_launch"]) if prof else None
    if prof:
        roof["traffic_source"] = prof.get("source")
        roof["dram_gbs"] = roof["traffic"] / (mk / 1e3) / 1e9
        roof["dram_frac"] = roof["dram_gbs"] / peak
        if prof.get("lts_bytes_per_launch"):
            roof["l2"] = {"bytes": prof["lts_bytes_per_launch"],
                          "gbs": prof["lts_bytes_per_launch"] / (mk / 1e3) / 1e9,
                          "lts_throughput_pct_of_peak": prof.get("lts_throughput_pct")}
    per_byte, nfr = frontier_stats(views, data, seg_len, 64 << 10)
    wl = worklist_bytes({k: v * n_in for k, v in per_byte.items()}, n_in, uniq, tables.device_bytes)
    roof["worklist_equivalent"] = {
        "bytes": wl, "bytes_per_input_byte": wl / n_in, "gbs": wl / (mk / 1e3) / 1e9,
        "frontier_sample": f"oracle unique frontier over the first {nfr} B, scaled to {n_in} B",
        "note": "the reference's global-memory worklist traffic (24 B per matched state + 8 B "
                "per successor tested); this kernel keeps the worklist in shared memory and "
                "resolves up to 12 symbols per prefix-table lookup, so it never moves these bytes"}
    line["roofline"] = roof
    if not args.no_cpu_baseline and world == 1:
        cb = CpuBaseline(anml, data[:n_in], dict(cfg, seg_len=seg_len), product_views=views)
        s = cb.calibrated(args.cpu_seconds)
        mbps, sec, desc, extra = cb.sample(s)
        line["cpu_baseline"] = dict({"value": mbps, "unit": "MB/s", "cores": cb.cores(),
                                     "kind": cb.kind, "sample": desc + f", {sec:.1f} s",
                                     "how": cb.note or "reference command, --validation",
                                     "host": host_info()}, **extra)
    return line


BATCH_DESC = ("16 NFAs of 2k-200k STEs (literal, Hamming, Levenshtein and dot-star generators), "
              "4096 streams of log-uniform length 1 KiB-4 MiB (about 2 GiB), one launch")


class Suite:
    """The batched suite's NFAs, streams and device tables, shared by the
    batched and serving parts."""

    def __init__(self, local_rank, n_streams=4096):
        import torch
        import ngap_b200 as nb
        from ngap_b200 import workloads as W
        t0 = time.time()
        self.nfas, self.data, self.offsets, self.lengths, self.nfa_of = W.batched_suite(
            seed=4, n_streams=n_streams)
        self.groups = [nb.Groups(nb.Nfa.from_string(n["anml"]), group_num=1) for n in self.nfas]
        self.tables = [nb.Tables(g, device=local_rank, precompute_depth=-1) for g in self.groups]
        self.ts = nb.TableSet(self.tables)
        self.eng = nb.Engine(local_rank)
        self.total = int(self.lengths.sum())
        self.d = torch.from_numpy(self.data).to(f"cuda:{local_rank}")
        self.setup_s = time.time() - t0


def stream_parity(suite, reps, sids, nsample=32, prefix=32 << 10, seed=0):
    """Per-stream parity on a random sample: each sampled stream's reports at
    offsets below `prefix` against the oracle on the stream's first `prefix`
    bytes (a report at offset q depends only on the stream's bytes up to q)."""
    from ngap_b200.engine import split_by_stream
    from oracle import oracle
    per = split_by_stream(reps, sids, len(suite.offsets))
    rng = np.random.default_rng(seed)
    pick = rng.choice(len(suite.offsets), size=min(nsample, len(suite.offsets)), replace=False)
    ok, nbytes, nrep, t0 = True, 0, 0, time.time()
    bad = []
    for i in sorted(int(x) for x in pick):
        L = int(min(int(suite.lengths[i]), prefix))
        if L == 0:
            continue
        o = int(suite.offsets[i])
        want, _ = oracle.match(suite.groups[int(suite.nfa_of[i])].views(), suite.data[o:o + L], 1, L,
                               nthreads=os.cpu_count() or 1)
        mine = per[i][(per[i] & M32) < np.uint64(L)]
        eq = bool(np.array_equal(mine, want))
        ok &= eq
        if not eq:
            bad.append(i)
        nbytes += L
        nrep += len(want)
    return {"bit_exact": ok, "streams_checked": len(pick), "bytes_checked": nbytes,
            "reports_checked": nrep, "prefix_bytes": prefix, "mismatched_streams": bad[:8],
            "oracle_seconds": round(time.time() - t0, 1)}


def batched_part(args, warmup, suite, local_rank, steps):
    """The batched suite: device-resident MB/s and e2e of one launch per step,
    plain (one ngap_match per stream) against batched on the same streams, and
    per-stream parity on a sample."""
    import torch
    import ngap_b200 as nb
    from ngap_b200 import autotune

    s = suite
    eng, ts = s.eng, s.ts
    t0 = time.time()
    if args.batched_params:  # fixed parameters (profiling): no autotuning launches
        best, tuned = json.loads(args.batched_params), []
    else:
        best, tuned = autotune.autotune(eng, ts, s.data, s.offsets, s.lengths, s.nfa_of,
                                        frac=0.01)
    tune_s = time.time() - t0
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    pinned = torch.from_numpy(s.data).pin_memory()
    for _ in range(warmup):
        nb.batch_match_async(eng, ts, s.d, s.offsets, s.lengths, s.nfa_of, stream=sh, **best)
        eng.sync()
    raw, uniq = eng.counts()
    reps0, sids0 = nb.batch_results(eng)
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(steps)]
    match_ms, launches = [], 0
    with ClockSampler(local_rank) as clk:
        for i in range(steps):
            evs[i][0].record(stream)
            nb.batch_match_async(eng, ts, s.d, s.offsets, s.lengths, s.nfa_of, stream=sh, **best)
            evs[i][1].record(stream)
            eng.sync()
            match_ms.append(eng.times_ms()[0])
            launches += eng.launches()
        torch.cuda.synchronize()
    t_ms = float(sum(a.elapsed_time(b) for a, b in evs))
    value = s.total * steps / (t_ms / 1e3) / 1e6
    # end to end: pinned host input copied in, every stream's reports copied out
    e2e_ms, d2h = [], 0
    for i in range(steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        nb.batch_match_async(eng, ts, pinned.numpy(), s.offsets, s.lengths, s.nfa_of, stream=sh,
                             **best)
        eng.sync()
        reps, sids = nb.batch_results(eng)
        b.record(stream)
        torch.cuda.synchronize()
        e2e_ms.append(a.elapsed_time(b))
        d2h = reps.nbytes + sids.nbytes + 40
    e2e_value = s.total * steps / (float(sum(e2e_ms)) / 1e3) / 1e6
    same = bool(np.array_equal(reps, reps0) and np.array_equal(sids, sids0))
    # plain (one ngap_match per stream, nonblockingallgroups, sequential on one
    # engine) against one batched launch, on the same 512 streams
    sub = np.arange(min(512, len(s.offsets)))
    sub_b = int(s.lengths[sub].sum())
    plain_ms = 0.0
    for i in sub:
        seg = s.d[int(s.offsets[i]):int(s.offsets[i] + s.lengths[i])]
        eng.match_async(s.tables[int(s.nfa_of[i])], seg, 1, int(s.lengths[i]),
                        algorithm="nonblockingallgroups", stream=sh)
        eng.sync()
        plain_ms += sum(eng.times_ms())
    sub_best = None
    for _ in range(3):
        nb.batch_match_async(eng, ts, s.d, s.offsets[sub], s.lengths[sub], s.nfa_of[sub],
                             stream=sh, **dict(best, use_graph=False))
        eng.sync()
        ms = sum(eng.times_ms())
        sub_best = ms if sub_best is None else min(sub_best, ms)
    out = {"value": value, "unit": "MB/s", "steps": steps, "ms_per_step": t_ms / steps,
           "config": {"workload": "batched_suite", "desc": BATCH_DESC, "streams": len(s.offsets),
                      "nfas": len(s.nfas), "input_bytes": s.total, "params": best,
                      "autotune": [[p, round(ms, 3) if ms is not None else None] for p, ms in tuned],
                      "autotune_seconds": round(tune_s, 1),
                      "setup_seconds": round(s.setup_s, 1),
                      "l2": "inputs larger than L2 (2 GiB)"},
           "reports": {"raw": raw, "unique": uniq},
           "gpu_launches": launches, "clocks": clk.summary(),
           "e2e": {"value": e2e_value, "unit": "MB/s", "h2d_bytes_per_step": s.total,
                   "d2h_bytes_per_step": d2h},
           "plain_vs_batched": {"streams": int(len(sub)), "bytes": sub_b,
                                "plain_algorithm": "nonblockingallgroups",
                                "plain_mbps": sub_b / plain_ms / 1e3,
                                "batched_mbps": sub_b / sub_best / 1e3,
                                "speedup": plain_ms / sub_best}}
    if not args.no_check:
        par = stream_parity(s, reps0, sids0)
        par["same_every_step"] = same
        par["bit_exact"] = par["bit_exact"] and same
        out["parity_vs_oracle"] = par
    peak, peak_kind = load_peaks()
    mk = float(np.mean(match_ms))
    tb = sum(t.device_bytes for t in s.tables)
    alg = s.total + tb + 8 * raw
    out["roofline"] = {"bound": "hbm", "unit": "GB/s", "peak": peak, "peak_source": peak_kind,
                       "kernel": "match_kernel", "kernel_ms": mk, "algorithmic_bytes": alg,
                       "algorithmic_def": "input bytes + table bytes + 8 B per raw report",
                       "achieved": alg / (mk / 1e3) / 1e9,
                       "frac": alg / (mk / 1e3) / 1e9 / peak}
    prof = profiled("batched_suite", len(s.offsets))
    out["roofline"]["traffic"] = float(prof["dram_bytes_per_launch"]) if prof else None
    return out


# chunk lengths of the predicting schedulers (cost_model.chunk_for)
SERVE_CHUNKS = dict(adapt_chunks=True, rho_ref=1.0, base_chunk=512, chunk_lo=64, chunk_hi=2048)

SERVE_DESC = ("Poisson requests at 2000/s, NFA uniform over the 16 of the batched suite, "
              "length log-normal (median 64 KiB, sigma 1.5, at most 4 MiB), 2 engine slots, "
              "16 GiB device-memory budget")


def serving_part(args, warmup, suite, steps, step_s=0.25):
    """Serving: p50/p99 latency and served MB/s under the default (arrival
    order), static and learned schedulers (predicted-work isolation lanes),
    the frontier-prediction error of each predictor, and report parity."""
    from ngap_b200 import cost_model as cm, serving as sv
    from oracle import oracle

    s = suite
    t0 = time.time()
    reg = cm.region_table(s.d, s.offsets, s.lengths, s.nfa_of, s.tables)
    y = cm.collect(s.eng, s.ts, s.d, s.offsets, s.lengths, s.nfa_of, reg)
    test = np.random.default_rng(0).random(len(s.offsets)) < 0.3
    te = test[reg["stream"]]
    lm = cm.LearnedModel(0).fit(reg["x"][~te], y[~te], epochs=60)
    mean = cm.NfaMeanModel(len(s.nfas)).fit(reg["nfa"][~te], y[~te], reg["len"][~te])
    stat = cm.StaticModel(reg["stats"])
    err = {}
    for name, pr in (("static", stat.predict(reg["nfa"])), ("nfa_mean", mean.predict(reg["nfa"])),
                     ("learned_fp32", lm.predict(reg["nfa"], reg["x"], bf16=False)),
                     ("learned_bf16", lm.predict(reg["nfa"], reg["x"], bf16=True))):
        e = cm.relative_error(pr[te], y[te])
        err[name] = {"median": float(np.median(e)), "mean": float(np.mean(e))}
    train_s = time.time() - t0
    pool = [s.data[int(o):int(o + l)] for o, l in zip(s.offsets, s.lengths)]
    dur = step_s * steps
    reqs = sv.make_requests(pool, s.nfa_of, len(s.nfas), rate=2000, duration=dur, seed=5)
    warm = sv.make_requests(pool, s.nfa_of, len(s.nfas), rate=2000,
                            duration=step_s * max(2, warmup), seed=6)
    preds = {"default": None, "static": sv.Predictor("static", s.tables),
             "learned": sv.Predictor("learned", s.tables, lm)}
    servers = {}
    for name, pred in preds.items():
        q = 0
        if pred is not None:
            q = cm.queue_for(float(np.max(pred.density(warm))))
        srv = sv.Server(s.ts, predictor=pred, slots=2, budget=16 << 30, queue_capacity=q,
                        **(SERVE_CHUNKS if pred is not None else {}))
        srv.run([sv.Request(r.rid, r.nfa, r.data, r.arrival) for r in warm])
        servers[name] = (srv, q)
    lat = {name: [] for name in preds}
    served, launches, clk_all, dev_ms, d2h, results = {}, 0, None, 0.0, 0, {}
    for rnd in range(2):  # two interleaved rounds of the three schedulers
        for name, (srv, q) in servers.items():
            srv.batches.clear()
            srv.launches = 0
            rs = [sv.Request(r.rid, r.nfa, r.data, r.arrival) for r in reqs]
            with ClockSampler(0) as clk:
                m = srv.run(rs)
            launches += srv.launches
            dev = np.array([b[3] for b in srv.batches]) if srv.batches else np.zeros(1)
            lat[name].append({"p50_ms": m["p50_ms"], "p99_ms": m["p99_ms"],
                              "mean_ms": m["mean_ms"], "batches": m["batches"],
                              "rejected": m["rejected"], "slow_passes": m["slow_passes"],
                              "host_us_per_request": m["host_us_per_request"],
                              "batch_device_ms_p50": float(np.percentile(dev, 50)),
                              "batch_device_ms_p99": float(np.percentile(dev, 99))})
            served.setdefault(name, []).append(m["MBps"])
            if rnd == 1:
                results[name] = rs
            if name == "learned" and rnd == 1:
                clk_all = clk.summary()
                dev_ms = sum(b[3] for b in srv.batches)
                d2h = 12 * sum(len(r.reports) for r in rs)  # u64 report + u32 stream id
    total = sum(len(r.data) for r in reqs)
    # parity: every request's reports identical under the three schedulers,
    # and equal to the oracle on a random sample of requests (prefix of 64 KiB)
    same = all(np.array_equal(results["default"][i].reports, results[k][i].reports)
               for k in ("static", "learned") for i in range(len(reqs)))
    rng = np.random.default_rng(3)
    ok, nchk, t1 = True, 0, time.time()
    for i in sorted(rng.choice(len(reqs), size=min(24, len(reqs)), replace=False)):
        r = results["learned"][int(i)]
        L = min(len(r.data), 16 << 10)
        want, _ = oracle.match(s.groups[r.nfa].views(), r.data[:L], 1, L,
                               nthreads=os.cpu_count() or 1)
        ok &= bool(np.array_equal(r.reports[(r.reports & M32) < np.uint64(L)], want))
        nchk += 1

    def mean_of(name, key):
        return float(np.mean([x[key] for x in lat[name]]))
    summary = {name: {"p50_ms": mean_of(name, "p50_ms"), "p99_ms": mean_of(name, "p99_ms"),
                      "served_mbps": float(np.mean(served[name]))} for name in preds}
    return {"value": summary["learned"]["served_mbps"], "unit": "MB/s",
            "config": {"workload": "serving", "desc": SERVE_DESC, "requests": len(reqs),
                       "seconds_of_arrivals": dur, "bytes": total, "rounds": 2,
                       "timing": "wall clock from arrival to reports on the host",
                       "model_seconds": round(train_s, 1)},
            "latency_ms": summary, "rounds": lat,
            "learned_vs_static": {
                "p99_ratio": summary["learned"]["p99_ms"] / summary["static"]["p99_ms"],
                "p50_ratio": summary["learned"]["p50_ms"] / summary["static"]["p50_ms"]},
            "scheduler": "default: the engine's chunks (about 2 KiB); static / learned: "
                         "each request's density (worklist entries per byte) predicted when a "
                         "slot is free, chunk = 512 x (1 + 1) / (1 + density) clamped to "
                         "[64, 2048] bytes, so that a batch's longest unit stays short; "
                         "batches in arrival order on 2 slots; queue sized from the densest "
                         "warm-up prediction",
            "chunk_policy": SERVE_CHUNKS,
            "frontier_prediction_rel_err": err,
            "gpu_launches": launches, "clocks": clk_all,
            "parity_vs_oracle": {"bit_exact": bool(ok and same), "same_under_every_scheduler":
                                 bool(same), "requests_checked": nchk, "prefix_bytes": 16 << 10,
                                 "oracle_seconds": round(time.time() - t1, 1)},
            "e2e": {"value": summary["learned"]["served_mbps"], "unit": "MB/s",
                    "h2d_bytes_per_step": int(total / max(1, steps)),
                    "d2h_bytes_per_step": int(d2h / max(1, steps))},
            "device_ms_learned": dev_ms}


# ---------------------------------------------------------------------------
# reference arm


def run_reference(args, warmup):
    """The reference CPU matcher on bounded samples of the headline workload
    (see the module docstring); K timed samples after W untimed small ones."""
    anml, data, cfg = workload_args(args.workload)
    n_in = (len(data) // cfg["seg_len"]) * cfg["seg_len"]
    cb = CpuBaseline(anml, data[:n_in], cfg)
    for _ in range(warmup):  # untimed: small samples
        cb.sample(1024)
    per = max(1.0, args.cpu_seconds * 2 / max(1, args.steps))
    s = cb.calibrated(per)
    vals, secs, extra = [], [], {}
    for _ in range(args.steps):
        mbps, sec, desc, extra = cb.sample(s)
        vals.append(mbps)
        secs.append(sec)
    v = float(np.mean(vals))
    line = {"metric": METRIC, "value": v, "unit": "MB/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": warmup, "ms_per_step": float(np.mean(secs)) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": DATA, "impl": "reference",
            "config": {"workload": args.workload, "desc": cfg["desc"],
                       "group_num": cfg["group_num"], "seg_len": cfg["seg_len"]},
            "cpu_baseline": dict({"value": v, "unit": "MB/s", "cores": cb.cores(),
                                  "threads": cfg["group_num"] * cb.nseg, "kind": cb.kind,
                                  "sample": desc + f"; after {warmup} untimed warm-up samples of "
                                                   "1 KiB per segment",
                                  "how": cb.note or "the reference's own ngap command, "
                                                    "--validation (its CPU validator timing line)",
                                  "host": host_info()}, **extra),
            "e2e": {"value": v, "unit": "MB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_suite_reference(args, warmup):
    """Reference arm of the batched suite and of serving: the oracle's
    restatement of the reference CPU loop over bounded samples of the
    streams (the first 16 KiB of random streams, one stream per thread),
    on group graphs from the reference's own front-end where it is built."""
    from concurrent.futures import ThreadPoolExecutor
    from ngap_b200 import workloads as W
    from oracle import oracle
    nfas, data, offsets, lengths, nfa_of = W.batched_suite(seed=4)
    tmp = tempfile.mkdtemp(prefix="ngap_bench_")
    views, how = [], "reference front-end graphs"
    for k, n in enumerate(nfas):
        p = os.path.join(tmp, f"nfa{k}.anml")
        with open(p, "w") as f:
            f.write(n["anml"])
        try:
            views.append(_ref_views(p, 1))
        except Exception:
            import ngap_b200 as nb
            views.append(nb.Groups(nb.Nfa.from_string(n["anml"]), group_num=1).views())
            how = "product front-end graphs (reference front-end absent)"
    uniq = [has_sticky(v) for v in views]
    ncores = os.cpu_count() or 1
    cap = 1 << 14

    def one(i):
        n = int(min(int(lengths[i]), cap))
        k = int(nfa_of[i])
        seg = data[int(offsets[i]):int(offsets[i]) + n]
        oracle.match(views[k], seg, 1, n, mode=0, unique=uniq[k], nthreads=1)
        return n

    def sample(seconds, seed):
        order = np.random.default_rng(seed).permutation(len(offsets))
        t0, done, nbytes = time.time(), 0, 0
        with ThreadPoolExecutor(ncores) as ex:
            while done < len(order) and (done == 0 or time.time() - t0 < seconds):
                part = order[done:done + ncores]
                done += len(part)
                nbytes += sum(ex.map(one, part))
        dt = time.time() - t0
        return nbytes / dt / 1e6, dt, done, nbytes

    for k in range(warmup):
        sample(0.0, 1000 + k)
    per = max(3.0, args.cpu_seconds * 3 / max(1, args.steps))
    vals, secs = [], []
    for k in range(args.steps):
        v, dt, done, nbytes = sample(per, k)
        vals.append(v)
        secs.append(dt)
    v = float(np.mean(vals))
    line = {"metric": METRIC, "value": v, "unit": "MB/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": warmup, "ms_per_step": float(np.mean(secs)) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": DATA, "impl": "reference",
            "config": {"workload": args.workload, "desc": BATCH_DESC, "streams": len(offsets),
                       "nfas": len(nfas)},
            "cpu_baseline": {"value": v, "unit": "MB/s", "cores": min(ncores, len(offsets)),
                             "kind": "port",
                             "sample": f"random streams, first {cap} B of each, one per thread, "
                                       f"about {per:.0f} s per step"
                                       + (f"; --unique for the {sum(uniq)} NFAs with .* states"
                                          if any(uniq) else ""),
                             "how": "oracle port of the reference CPU loop over " + how,
                             "host": host_info()},
            "e2e": {"value": v, "unit": "MB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="hamming_set",
                    choices=["hamming_set", "literal_set", "high_frontier", "batched_suite",
                             "serving"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-check", action="store_true", help="skip the parity checks")
    ap.add_argument("--no-extras", action="store_true",
                    help="headline line only (no batched and serving parts)")
    ap.add_argument("--cpu-seconds", type=float, default=3.0,
                    help="CPU seconds of the cpu_baseline sample (the reference arm takes "
                         "max(1, 2 x this / steps) per step)")
    ap.add_argument("--segments", type=int, default=0,
                    help="match only the first N segments (smaller case for profiling)")
    ap.add_argument("--batched-params", default="",
                    help="JSON parameters of the batched launch instead of autotuning them")
    ap.add_argument("--streams", type=int, default=4096,
                    help="streams of the batched suite (fewer: a smaller case for profiling)")
    args = ap.parse_args()
    warmup = max(3, args.warmup)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:  # the reference arm is one CPU run; other ranks have nothing to do
            return
        if args.workload in ("batched_suite", "serving"):
            run_suite_reference(args, warmup)
        else:
            run_reference(args, warmup)
        return

    if args.workload in ("batched_suite", "serving"):
        if rank != 0:
            return
        import torch
        torch.cuda.set_device(0)
        suite = Suite(0, args.streams)
        part = (batched_part(args, warmup, suite, 0, args.steps) if args.workload == "batched_suite"
                else serving_part(args, warmup, suite, args.steps))
        line = {"metric": METRIC, "value": part.pop("value"), "unit": part.pop("unit"),
                "n_gpus": 1, "steps": args.steps, "warmup": warmup,
                "ms_per_step": part.pop("ms_per_step", 250.0), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": DATA}
        line.update(part)
        print(json.dumps(line), flush=True)
        return

    dist = _dist_setup(world, local_rank)
    t0 = time.time()
    line = run_plain(args, warmup, rank, world, local_rank, dist)
    if rank == 0:
        line["wall_seconds"] = {"plain": round(time.time() - t0, 1)}
    if rank == 0 and world == 1 and args.workload == "hamming_set" and not args.no_extras:
        t1 = time.time()
        suite = Suite(local_rank)
        line["batched"] = batched_part(args, warmup, suite, local_rank, min(args.steps, 5))
        t2 = time.time()
        line["serving"] = serving_part(args, warmup, suite, args.steps)
        line["wall_seconds"].update({"batched": round(t2 - t1, 1),
                                     "serving": round(time.time() - t2, 1)})
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
