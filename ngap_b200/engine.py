"""Python mirror of the reference's `ngap` host interface over the C ABI.

The reference drives matching through `class ngap` (code/src/ngap/ngap.h:27-177):
set_ngap_option, preprocessing, set_nfa_group, add_symbol_stream,
prepare_original_input_streams and one launch_*_groups() per algorithm. The
same flow is offered here by :class:`Ngap`; :class:`Nfa`, :class:`Groups`,
:class:`Tables` and :class:`Engine` wrap the C ABI objects one to one.
"""
import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import ALGORITHMS, NgapError, check, lib


TILE_MODES = {"auto": 0, "shared": 1, "global": 2}


def table_opts(device, precompute_depth, precompute_cutoff, tile_states, max_table_entries,
               tile_mode):
    """ngap_table_opts from Python values; tile_mode is one of TILE_MODES."""
    if tile_mode not in TILE_MODES:
        raise ValueError(f"tile_mode must be one of {sorted(TILE_MODES)}")
    return _lib.TableOpts(device, precompute_depth, precompute_cutoff, tile_states,
                          max_table_entries, TILE_MODES[tile_mode])


def as_u8(data):
    """Host input as a contiguous uint8 array: bytes-like objects (bytes,
    bytearray, memoryview) by their bytes, arrays and sequences as values."""
    if isinstance(data, (bytes, bytearray, memoryview)):
        return np.frombuffer(data, dtype=np.uint8)
    return np.ascontiguousarray(data, dtype=np.uint8)


class Nfa:
    """Parsed ANML (load_nfa_from_anml, code/src/commons/NFALoader.cpp:70)."""

    def __init__(self, handle):
        self._h = ctypes.c_void_p(handle)

    @classmethod
    def from_file(cls, path):
        """Loads an ANML file (load_nfa_from_file, NFALoader.cpp:164-171)."""
        h = ctypes.c_void_p()
        check(lib().ngap_nfa_load_anml(str(path).encode(), ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def from_string(cls, xml):
        """Parses an ANML document held in memory (str or bytes)."""
        data = xml.encode() if isinstance(xml, str) else bytes(xml)
        h = ctypes.c_void_p()
        check(lib().ngap_nfa_parse_anml(data, len(data), ctypes.byref(h)))
        return cls(h.value)

    @property
    def num_states(self):
        return lib().ngap_nfa_num_states(self._h)

    @property
    def num_edges(self):
        return lib().ngap_nfa_num_edges(self._h)

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value and _lib._lib is not None:
            _lib._lib.ngap_nfa_destroy(self._h)
            self._h = ctypes.c_void_p()


@dataclass
class GroupGraph:
    """One group graph as Graph::ReadNFA + Csr::fromCoo lay it out."""
    row_offsets: np.ndarray
    col_indices: np.ndarray
    symbol_sets: np.ndarray  # (V, 8) uint32
    node_attrs: np.ndarray
    always_active: np.ndarray
    start_states: np.ndarray
    cc_begin: np.ndarray
    orig_node: np.ndarray

    @property
    def num_states(self):
        return len(self.node_attrs)


def _np(ptr, n, dtype):
    if n == 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


class Groups:
    """Group graphs after CC split, degree limiting and grouping (ngap.cu:63-91)."""

    def __init__(self, nfa, group_num=10, max_nfa_size=-1, quit_degree=True, remove_degree=False):
        opts = _lib.GroupOpts(group_num, max_nfa_size, int(quit_degree), int(remove_degree))
        h = ctypes.c_void_p()
        check(lib().ngap_groups_build(nfa._h, ctypes.byref(opts), ctypes.byref(h)))
        self._h = h
        self._nfa = nfa

    @property
    def count(self):
        """Number of groups (at most group_num; fewer when there are fewer CCs)."""
        return lib().ngap_groups_count(self._h)

    def cc_stats(self):
        """(CCs, CCs whose out-degree could not be limited, CCs over
        max_nfa_size), as limit_out_degree_on_ccs counts them
        (nfa_utils.cpp:637-680)."""
        t, f, b = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        check(lib().ngap_groups_cc_stats(self._h, ctypes.byref(t), ctypes.byref(f), ctypes.byref(b)))
        return t.value, f.value, b.value

    def view(self, g):
        """Group g's graph as numpy views of the library's arrays (CSR, bitsets,
        attributes, always-active and start lists; graph.cu:169-206)."""
        v = _lib.GroupView()
        check(lib().ngap_group_view_get(self._h, g, ctypes.byref(v)))
        V, E = v.num_states, v.num_edges
        return GroupGraph(
            row_offsets=_np(v.row_offsets, V + 1, np.int32),
            col_indices=_np(v.col_indices, E, np.int32),
            symbol_sets=_np(v.symbol_sets, V * 8, np.uint32).reshape(V, 8),
            node_attrs=_np(v.node_attrs, V, np.uint8),
            always_active=_np(v.always_active, v.num_aas, np.int32),
            start_states=_np(v.start_states, v.num_start, np.int32),
            cc_begin=_np(v.cc_begin, v.num_ccs + 1, np.int32),
            orig_node=_np(v.orig_node, V, np.int32),
        )

    def views(self):
        return [self.view(g) for g in range(self.count)]

    @staticmethod
    def _plan_opts(precompute_depth, tile_states, tile_mode, max_table_entries):
        return table_opts(0, precompute_depth, -1, tile_states, max_table_entries, tile_mode)

    def tiles(self, precompute_depth=0, tile_states=0, tile_mode="auto", max_table_entries=0):
        """The tiles Tables(...) would build, planned on the host (no GPU):
        list of dicts (phase, pair, group, num_states, num_ccs, nact, nsticky,
        global, depth, max_path, nlive, dense_levels, naas, shortcuts,
        table_bytes)."""
        opts = self._plan_opts(precompute_depth, tile_states, tile_mode, max_table_entries)
        n = ctypes.c_int()
        check(lib().ngap_tiles_describe(self._h, ctypes.byref(opts), None, 0, ctypes.byref(n)))
        buf = (_lib.TileDesc * max(1, n.value))()
        check(lib().ngap_tiles_describe(self._h, ctypes.byref(opts), buf, n.value,
                                        ctypes.byref(n)))
        out = []
        for d in buf[:n.value]:
            r = {k: getattr(d, k) for k, _ in _lib.TileDesc._fields_}
            r["global"] = r.pop("global_")
            out.append(r)
        return out

    def table_lookup(self, tile, keys, precompute_depth=0, tile_states=0, tile_mode="auto",
                     max_table_entries=0):
        """Looks up byte strings (uint8 array [n, d]) in prefix table d of a
        tile, planned on the host as tiles() plans it. Returns, per string,
        (ids, report_ids): the report ids (sid | group << 22) of the states
        the table lists and of its report states."""
        keys = np.ascontiguousarray(keys, dtype=np.uint8)
        if keys.ndim != 2:
            raise ValueError("keys must be a 2-D uint8 array [n, length]")
        opts = self._plan_opts(precompute_depth, tile_states, tile_mode, max_table_entries)
        n, d = keys.shape
        off = np.zeros(n + 1, np.int64)
        roff = np.zeros(n + 1, np.int64)
        cap = max(1024, 4 * n)
        while True:
            ids = np.zeros(cap, np.uint32)
            reps = np.zeros(cap, np.uint32)
            rc = lib().ngap_tiles_lookup(self._h, ctypes.byref(opts), tile, keys.ctypes.data, n, d,
                                         ids.ctypes.data, off.ctypes.data, reps.ctypes.data,
                                         roff.ctypes.data, cap)
            need = max(int(off[n]), int(roff[n]))
            if rc != 0 and need > cap:
                cap = need
                continue
            check(rc)
            return [(ids[off[k]:off[k + 1]].copy(), reps[roff[k]:roff[k + 1]].copy())
                    for k in range(n)]

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value and _lib._lib is not None:
            _lib._lib.ngap_groups_destroy(self._h)
            self._h = ctypes.c_void_p()


class Tables:
    """Device-resident matching tables (group_graph.h:6-109, ngap.cu:3086-3111)."""

    def __init__(self, groups, device=0, precompute_depth=0, precompute_cutoff=-1,
                 tile_states=0, max_table_entries=0, tile_mode="auto"):
        opts = table_opts(device, precompute_depth, precompute_cutoff, tile_states,
                          max_table_entries, tile_mode)
        h = ctypes.c_void_p()
        check(lib().ngap_tables_build(groups._h, ctypes.byref(opts), ctypes.byref(h)))
        self._h = h
        self.groups = groups
        self.num_groups = groups.count

    @property
    def device_bytes(self):
        return lib().ngap_tables_device_bytes(self._h)

    def stats(self):
        """Table statistics (dict): tiles, states, edges, aas, depth, max_nlive,
        max_list, cutoff, list_entries, exp_list."""
        st = _lib.TablesStats()
        check(lib().ngap_tables_stats_get(self._h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in _lib.TablesStats._fields_}

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value and _lib._lib is not None:
            _lib._lib.ngap_tables_destroy(self._h)
            self._h = ctypes.c_void_p()


class Engine:
    """Device buffers, kernels and results (ngap_buffer.cu; ngap.cu launch_*)."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        check(lib().ngap_engine_create(device, ctypes.byref(h)))
        self._h = h
        self.device = device

    def match_async(self, tables, data, num_seg, seg_len, algorithm="nonblockingallgroups",
                    is_dup=False, unique=False, active_threshold=20, report_off=False,
                    result_capacity=54619400, window=0, chunk=0, first_segment=0, stream=None):
        """Starts matching `data` (numpy uint8 array in host memory, or a CUDA
        tensor / object exposing data_ptr()) of num_seg * seg_len bytes.
        first_segment: global index of data's first segment when a stream is
        split across GPUs (start-of-data states belong to global segment 0)."""
        algo = ALGORITHMS[algorithm] if isinstance(algorithm, str) else int(algorithm)
        p = _lib.MatchParams(algo, num_seg, seg_len, int(is_dup), int(unique), active_threshold,
                             int(report_off), result_capacity, window, chunk, first_segment)
        if hasattr(data, "data_ptr"):
            ptr, on_dev = data.data_ptr(), int(getattr(data, "is_cuda", True))
            nbytes = data.numel() * data.element_size() if hasattr(data, "numel") else None
        else:
            arr = as_u8(data)
            self._keep = arr
            ptr, on_dev, nbytes = arr.ctypes.data, 0, arr.nbytes
        if num_seg * seg_len > 0 and ptr == 0:
            raise NgapError(1, "empty input")
        if nbytes is not None and nbytes < num_seg * seg_len:
            raise NgapError(1, f"input holds {nbytes} bytes, num_seg * seg_len = "
                               f"{num_seg * seg_len}")
        check(lib().ngap_match(self._h, tables._h, ctypes.c_void_p(ptr), on_dev, ctypes.byref(p),
                               ctypes.c_void_p(stream or 0)))

    def sync(self):
        """Waits for the engine's last match; raises NgapError on its status."""
        return check(lib().ngap_engine_sync(self._h))

    def set_trace(self, enable=True):
        """Records per-unit worklist work in the following matches."""
        check(lib().ngap_engine_set_trace(self._h, int(bool(enable))))

    def unit_trace(self):
        """Records of the last match's units: numpy structured array with
        fields stream, tile, lo, hi (positions relative to the segment or
        stream), work (entries expanded + injected) and cycles (SM clock
        cycles the unit's warp spent on it)."""
        n = ctypes.c_int64()
        check(lib().ngap_trace_copy(self._h, None, 0, ctypes.byref(n)))
        cap = max(1, n.value)
        buf = (_lib.UnitTrace * cap)()
        check(lib().ngap_trace_copy(self._h, buf, cap, ctypes.byref(n)))
        dt = np.dtype([("stream", np.int32), ("tile", np.int32), ("lo", np.int64),
                       ("hi", np.int64), ("work", np.uint64), ("cycles", np.uint64)])
        return np.frombuffer(buf, dtype=dt, count=n.value).copy()

    @property
    def device_bytes(self):
        return lib().ngap_engine_device_bytes(self._h)

    def memory(self):
        """Device bytes the engine holds, by part: dict with input, reports,
        scratch (per-warp worklist scratch) and plan."""
        m = _lib.EngineMem()
        check(lib().ngap_engine_memory(self._h, ctypes.byref(m)))
        return {k: getattr(m, k) for k in ("input", "reports", "scratch", "plan")}

    def match(self, tables, data, num_seg, seg_len, **kw):
        """match_async, sync and results: sorted unique reports (uint64)."""
        self.match_async(tables, data, num_seg, seg_len, **kw)
        self.sync()
        return self.results()

    def counts(self):
        """(raw reports emitted, unique reports) of the last match."""
        raw, uniq = ctypes.c_uint64(), ctypes.c_uint64()
        check(lib().ngap_results_count(self._h, ctypes.byref(raw), ctypes.byref(uniq)))
        return raw.value, uniq.value

    def results(self):
        """Sorted unique reports, reference encoding ((sid|g<<22)<<32 | offset)."""
        _, n = self.counts()
        out = np.zeros(n, dtype=np.uint64)
        if n:
            got = lib().ngap_results_copy(self._h, out.ctypes.data, n)
            if got != n:
                raise NgapError(5, _lib.last_error())
        return out

    def results_device_ptr(self):
        return lib().ngap_results_device(self._h)

    def times_ms(self):
        """(match ms, sort ms) of the last match, from CUDA events."""
        a, b = ctypes.c_float(), ctypes.c_float()
        check(lib().ngap_last_times_ms(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def launches(self):
        """Kernels the last match launched."""
        return lib().ngap_last_launches(self._h)

    def work(self):
        """(worklist entries expanded, entries injected) of the last match."""
        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        check(lib().ngap_engine_work(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def sort_unique_device(self, d_in_ptr, n, d_out_ptr, stream=None):
        """Device radix sort + unique of n reference-encoded reports."""
        nout = ctypes.c_uint64()
        check(lib().ngap_reports_sort_unique(self._h, ctypes.c_void_p(d_in_ptr), n,
                                             ctypes.c_void_p(d_out_ptr), ctypes.byref(nout),
                                             ctypes.c_void_p(stream or 0)))
        return nout.value

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value and _lib._lib is not None:
            _lib._lib.ngap_engine_destroy(self._h)
            self._h = ctypes.c_void_p()


class TableSet:
    """Tables of several NFAs usable in one batched launch."""

    def __init__(self, tables):
        self.tables = list(tables)  # keep them alive
        arr = (ctypes.c_void_p * len(self.tables))(*[t._h.value for t in self.tables])
        h = ctypes.c_void_p()
        check(lib().ngap_tableset_create(arr, len(self.tables), ctypes.byref(h)))
        self._h = h

    def __len__(self):
        return len(self.tables)

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value and _lib._lib is not None:
            _lib._lib.ngap_tableset_destroy(self._h)
            self._h = ctypes.c_void_p()


def batch_match_async(engine, tableset, data, offsets, lengths, nfas,
                      algorithm="nonblockingpcgroups", unique=False, active_threshold=20,
                      report_off=False, result_capacity=54619400, window=0, chunk=0,
                      use_graph=False, stream=None, chunks=None, queue_capacity=0):
    """Starts one launch over all streams: stream i is data[offsets[i] :
    offsets[i] + lengths[i]] matched against tableset NFA nfas[i]. `data` is a
    numpy uint8 array (pinned memory is needed with use_graph) or a CUDA tensor.
    chunks: optional per-stream chunk lengths (0 = `chunk`); queue_capacity:
    overflow-stack entries per warp (0 = the default)."""
    n = len(offsets)
    ss = (_lib.BatchStream * n)()
    for i in range(n):
        ss[i] = _lib.BatchStream(int(offsets[i]), int(lengths[i]), int(nfas[i]),
                                 int(chunks[i]) if chunks is not None else 0)
    engine._keep_streams = ss
    algo = ALGORITHMS[algorithm] if isinstance(algorithm, str) else int(algorithm)
    p = _lib.BatchParams(algo, int(unique), active_threshold, int(report_off), result_capacity,
                         window, chunk, int(use_graph), int(queue_capacity))
    if hasattr(data, "data_ptr"):
        ptr, on_dev, nbytes = data.data_ptr(), int(getattr(data, "is_cuda", True)), data.numel()
    else:
        arr = as_u8(data)
        engine._keep = arr
        ptr, on_dev, nbytes = arr.ctypes.data, 0, arr.nbytes
    check(lib().ngap_batch_match(engine._h, tableset._h, ctypes.c_void_p(ptr), nbytes, on_dev, ss,
                                 n, ctypes.byref(p), ctypes.c_void_p(stream or 0)))


def batch_results(engine):
    """(reports, stream_ids): unique reports sorted by (stream, offset, id);
    offsets are local to each stream."""
    _, n = engine.counts()
    rep = np.zeros(n, dtype=np.uint64)
    sid = np.zeros(n, dtype=np.uint32)
    got = ctypes.c_uint64()
    if n:
        check(lib().ngap_batch_results(engine._h, rep.ctypes.data, sid.ctypes.data, n,
                                       ctypes.byref(got)))
    return rep[:got.value], sid[:got.value]


def split_by_stream(reports, stream_ids, nstreams):
    """List of per-stream report arrays."""
    bounds = np.searchsorted(stream_ids, np.arange(nstreams + 1, dtype=np.uint32))
    return [reports[bounds[i]:bounds[i + 1]] for i in range(nstreams)]


def cpu_validate(groups, data, num_seg, seg_len, is_dup=False):
    """The library's CPU checker (the CLI's --validation): sorted unique reports."""
    arr = as_u8(data)
    if arr.nbytes < num_seg * seg_len:
        raise NgapError(1, f"input holds {arr.nbytes} bytes, num_seg * seg_len = "
                           f"{num_seg * seg_len}")
    cap = 1 << 16
    while True:
        out = np.zeros(cap, dtype=np.uint64)
        ms = ctypes.c_double()
        n = lib().ngap_cpu_validate_reference(groups._h, arr.ctypes.data, num_seg, seg_len,
                                              int(is_dup), out.ctypes.data, cap, ctypes.byref(ms))
        if n >= 0:
            return out[:n]
        cap *= 4


@dataclass
class NgapOption:
    """Fields and defaults of ngap_option + common_gpunfa_options
    (code/src/ngap/ngap_option.h:52-68, code/include/commons/common_func.h:50-58)."""
    algorithm: str = "nonblockingallgroups"
    group_num: int = 10
    max_nfa_size: int = -1
    quit_degree: bool = True
    remove_degree: bool = False
    duplicate_input_stream: int = 1
    input_start_pos: int = 0
    input_len: int = -1
    split_chunk_size: int = -1
    output_capacity: int = 54619400
    report_off: bool = False
    unique: bool = False
    active_threshold: int = 20
    precompute_depth: int = 0
    precompute_cutoff: int = -1
    data_buffer_fetch_size: int = 128
    add_aas_start: int = 0
    add_aas_interval: int = 1
    validation: bool = True
    quick_validation: int = -1
    device: int = 0
    window: int = 0
    chunk: int = 0
    tile_states: int = 0


class Ngap:
    """Reference-shaped driver: the main.cu flow on one GPU."""

    def __init__(self, nfa, opt=None):
        self.nfa = nfa
        self.opt = opt or NgapOption()
        self.groups = None
        self.tables = None
        self.streams = []
        self.original = None
        self.engine = None

    def set_ngap_option(self, opt):
        self.opt = opt

    def preprocessing(self):
        """ngap::preprocessing + group_nfas_by_num (ngap.cu:63-91,
        nfa_utils.cpp:382-424)."""
        o = self.opt
        self.groups = Groups(self.nfa, o.group_num, o.max_nfa_size, o.quit_degree, o.remove_degree)
        self.opt.group_num = self.groups.count
        return self.groups

    def set_nfa_group(self, groups):
        self.groups = groups

    def set_report_off(self, report_off, output_capacity, quick_validation=-1):
        """ngap.h set_report_off (main.cu:105-106): count reports only, the
        result capacity and the expected report count of --quick-validation."""
        self.opt.report_off = bool(report_off)
        self.opt.output_capacity = int(output_capacity)
        self.opt.quick_validation = int(quick_validation)

    def add_symbol_stream(self, seg):
        self.streams.append(as_u8(seg).copy())

    def slice_input(self, data):
        """main.cu:48-51: input_len bytes from input_start_pos (to the end when
        the input is shorter) when both are set (not -1)."""
        o = self.opt
        d = as_u8(data)
        if o.input_start_pos != -1 and o.input_len != -1:
            st = min(max(o.input_start_pos, 0), len(d))
            d = d[st:st + max(o.input_len, 0)]
        return d

    def prepare_segments(self, data):
        """main.cu:48-51 and 81-102: slice the input, duplicate it, cut it into
        equal segments (the whole stream when split_chunk_size <= 0) and keep
        the duplicated stream (prepare_original_input_streams)."""
        o = self.opt
        ss = np.tile(self.slice_input(data), o.duplicate_input_stream)
        chunk = o.split_chunk_size if o.split_chunk_size > 0 else len(ss)
        num_seg = len(ss) // chunk if chunk > 0 else 0
        self.streams = [ss[i * chunk:(i + 1) * chunk] for i in range(num_seg)]
        self.prepare_original_input_streams(ss)
        return num_seg, chunk

    def prepare_original_input_streams(self, ss):
        self.original = as_u8(ss)

    def automata_validation(self, results):
        """ngap::automataValidation (ngap.cu:2270-2344): the reports equal the
        CPU checker's on the same segments (automataGroupsReference,
        ngap.cu:2171-2268)."""
        if self.groups is None:
            self.preprocessing()
        data = np.concatenate(self.streams) if self.streams else np.zeros(0, np.uint8)
        seg_len = len(self.streams[0]) if self.streams else 0
        want = cpu_validate(self.groups, data, len(self.streams), seg_len, self.is_dup())
        return bool(np.array_equal(np.asarray(results, dtype=np.uint64), want))

    def is_dup(self):
        """Start-of-data states in every segment (ngap_buffer.cu:479-484)."""
        o = self.opt
        return o.duplicate_input_stream > 1 and (o.split_chunk_size in (-1, o.input_len))

    def launch(self, algorithm=None):
        """Builds tables and an engine once, matches the segments and returns
        the sorted unique reports (the launch_*_groups bodies, ngap.cu:115-2078)."""
        o = self.opt
        if self.groups is None:
            self.preprocessing()
        if self.tables is None:
            self.tables = Tables(self.groups, o.device, o.precompute_depth, o.precompute_cutoff,
                                 o.tile_states)
        if self.engine is None:
            self.engine = Engine(o.device)
        data = np.concatenate(self.streams) if self.streams else np.zeros(0, np.uint8)
        seg_len = len(self.streams[0]) if self.streams else 0
        return self.engine.match(self.tables, data, len(self.streams), seg_len,
                                 algorithm=algorithm or o.algorithm, is_dup=self.is_dup(),
                                 unique=o.unique, active_threshold=o.active_threshold,
                                 report_off=o.report_off, result_capacity=o.output_capacity,
                                 window=o.window, chunk=o.chunk)

    # one entry point per reference launcher (main.cu:114-127)
    def launch_blocking_groups(self):
        return self.launch("blockinggroups")

    def launch_non_blocking_nap_groups(self):
        return self.launch("NAPgroups")

    def launch_non_blocking_groups(self):
        return self.launch("nonblockinggroups")

    def launch_non_blocking_r1_groups(self):
        return self.launch("nonblockingr1groups")

    def launch_non_blocking_r2_groups(self):
        return self.launch("nonblockingr2groups")

    def launch_non_blocking_prec_groups(self):
        return self.launch("nonblockingpcgroups")

    def launch_non_blocking_all_groups(self):
        return self.launch("nonblockingallgroups")


def decode_reports(reports):
    """Splits reference-encoded reports into (ids, offsets)."""
    r = np.asarray(reports, dtype=np.uint64)
    return (r >> np.uint64(32)).astype(np.uint32), (r & np.uint64(0xFFFFFFFF)).astype(np.uint32)
