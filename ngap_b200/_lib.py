"""ctypes binding of the C ABI declared in include/ngap_b200.h.

The shared library is built in-tree (ngap_b200/libngap_b200.so) by
``__graft_entry__.build()`` or ``make -C ngap_b200/csrc``. There is no CPU
fallback: if the library cannot be loaded, every entry point raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# NGAP_B200_LIB names another build of the same library (A/B measurements of
# kernel variants); by default the in-tree build is loaded
LIB_PATH = os.environ.get("NGAP_B200_LIB") or os.path.join(_HERE, "libngap_b200.so")

NGAP_OK = 0
STATUS_NAMES = {
    0: "NGAP_OK", 1: "NGAP_E_INVALID", 2: "NGAP_E_PARSE", 3: "NGAP_E_UNSUPPORTED",
    4: "NGAP_E_DEGREE", 5: "NGAP_E_CUDA", 6: "NGAP_E_OVERFLOW_QUEUE",
    7: "NGAP_E_OVERFLOW_RESULTS", 8: "NGAP_E_TIMEOUT", 9: "NGAP_E_NOMEM", 10: "NGAP_E_IO",
}

ALGORITHMS = {
    "blockinggroups": 0, "NAPgroups": 1, "nonblockinggroups": 2, "nonblockingr1groups": 3,
    "nonblockingr2groups": 4, "nonblockingpcgroups": 5, "nonblockingallgroups": 6,
}


class NgapError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class GroupOpts(ctypes.Structure):
    _fields_ = [("group_num", ctypes.c_int), ("max_nfa_size", ctypes.c_int),
                ("quit_degree", ctypes.c_int), ("remove_degree", ctypes.c_int)]


class GroupView(ctypes.Structure):
    _fields_ = [("num_states", ctypes.c_int32), ("num_edges", ctypes.c_int32),
                ("num_aas", ctypes.c_int32), ("num_start", ctypes.c_int32),
                ("num_ccs", ctypes.c_int32),
                ("row_offsets", ctypes.POINTER(ctypes.c_int32)),
                ("col_indices", ctypes.POINTER(ctypes.c_int32)),
                ("symbol_sets", ctypes.POINTER(ctypes.c_uint32)),
                ("node_attrs", ctypes.POINTER(ctypes.c_uint8)),
                ("always_active", ctypes.POINTER(ctypes.c_int32)),
                ("start_states", ctypes.POINTER(ctypes.c_int32)),
                ("cc_begin", ctypes.POINTER(ctypes.c_int32)),
                ("orig_node", ctypes.POINTER(ctypes.c_int32))]


class TableOpts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("precompute_depth", ctypes.c_int),
                ("precompute_cutoff", ctypes.c_int), ("tile_states", ctypes.c_int),
                ("max_table_entries", ctypes.c_int64), ("tile_mode", ctypes.c_int)]


class TileDesc(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int32) for k in (
        "phase", "pair", "group", "num_states", "num_ccs", "nact", "nsticky", "global_",
        "depth", "max_path", "nlive", "dense_levels", "naas", "shortcuts")] + \
        [("table_bytes", ctypes.c_int64)]


class MatchParams(ctypes.Structure):
    _fields_ = [("algorithm", ctypes.c_int), ("num_seg", ctypes.c_int64),
                ("seg_len", ctypes.c_int64), ("is_dup", ctypes.c_int), ("unique", ctypes.c_int),
                ("active_threshold", ctypes.c_int), ("report_off", ctypes.c_int),
                ("result_capacity", ctypes.c_uint64), ("window", ctypes.c_int),
                ("chunk", ctypes.c_int), ("first_segment", ctypes.c_int64)]


class BatchStream(ctypes.Structure):
    _fields_ = [("offset", ctypes.c_uint64), ("length", ctypes.c_uint64),
                ("nfa", ctypes.c_int32), ("chunk", ctypes.c_int32)]


class BatchParams(ctypes.Structure):
    _fields_ = [("algorithm", ctypes.c_int), ("unique", ctypes.c_int),
                ("active_threshold", ctypes.c_int), ("report_off", ctypes.c_int),
                ("result_capacity", ctypes.c_uint64), ("window", ctypes.c_int),
                ("chunk", ctypes.c_int), ("use_graph", ctypes.c_int),
                ("queue_capacity", ctypes.c_int)]


class EngineMem(ctypes.Structure):
    _fields_ = [("input", ctypes.c_int64), ("reports", ctypes.c_int64),
                ("scratch", ctypes.c_int64), ("plan", ctypes.c_int64)]


class UnitTrace(ctypes.Structure):
    _fields_ = [("stream", ctypes.c_int32), ("tile", ctypes.c_int32), ("lo", ctypes.c_int64),
                ("hi", ctypes.c_int64), ("work", ctypes.c_uint64), ("cycles", ctypes.c_uint64)]


class TablesStats(ctypes.Structure):
    _fields_ = [("tiles", ctypes.c_int32), ("states", ctypes.c_int32), ("edges", ctypes.c_int32),
                ("aas", ctypes.c_int32), ("depth", ctypes.c_int32), ("max_nlive", ctypes.c_int32),
                ("max_list", ctypes.c_int32), ("cutoff", ctypes.c_int32),
                ("list_entries", ctypes.c_int64), ("exp_list", ctypes.c_double)]


FEAT_BYTES = 258  # NGAP_FEAT_BYTES


# name -> (restype, argtypes); exactly the functions include/ngap_b200.h declares
SIGNATURES = {
    "ngap_nfa_load_anml": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)]),
    "ngap_nfa_parse_anml": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t,
                                           ctypes.POINTER(ctypes.c_void_p)]),
    "ngap_nfa_destroy": (None, [ctypes.c_void_p]),
    "ngap_nfa_num_states": (ctypes.c_int64, [ctypes.c_void_p]),
    "ngap_nfa_num_edges": (ctypes.c_int64, [ctypes.c_void_p]),
    "ngap_groups_build": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(GroupOpts),
                                         ctypes.POINTER(ctypes.c_void_p)]),
    "ngap_groups_count": (ctypes.c_int, [ctypes.c_void_p]),
    "ngap_groups_cc_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64),
                                            ctypes.POINTER(ctypes.c_int64),
                                            ctypes.POINTER(ctypes.c_int64)]),
    "ngap_group_view_get": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                           ctypes.POINTER(GroupView)]),
    "ngap_groups_destroy": (None, [ctypes.c_void_p]),
    "ngap_tables_build": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(TableOpts),
                                         ctypes.POINTER(ctypes.c_void_p)]),
    "ngap_tables_destroy": (None, [ctypes.c_void_p]),
    "ngap_tiles_lookup": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(TableOpts), ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_int64]),
    "ngap_tiles_describe": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(TableOpts),
                                           ctypes.POINTER(TileDesc), ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_int)]),
    "ngap_tables_device_bytes": (ctypes.c_int64, [ctypes.c_void_p]),
    "ngap_engine_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "ngap_engine_destroy": (None, [ctypes.c_void_p]),
    "ngap_match": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                  ctypes.POINTER(MatchParams), ctypes.c_void_p]),
    "ngap_engine_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "ngap_results_count": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64),
                                          ctypes.POINTER(ctypes.c_uint64)]),
    "ngap_results_device": (ctypes.c_void_p, [ctypes.c_void_p]),
    "ngap_results_copy": (ctypes.c_int64, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64]),
    "ngap_last_times_ms": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float),
                                          ctypes.POINTER(ctypes.c_float)]),
    "ngap_last_launches": (ctypes.c_int, [ctypes.c_void_p]),
    "ngap_engine_work": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64),
                                        ctypes.POINTER(ctypes.c_uint64)]),
    "ngap_engine_device_bytes": (ctypes.c_int64, [ctypes.c_void_p]),
    "ngap_engine_memory": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(EngineMem)]),
    "ngap_engine_set_trace": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "ngap_engine_test_wait_timeout": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32,
                                                     ctypes.c_int32]),
    "ngap_trace_copy": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(UnitTrace), ctypes.c_int64,
                                       ctypes.POINTER(ctypes.c_int64)]),
    "ngap_tables_stats_get": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(TablesStats)]),
    "ngap_features": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_void_p, ctypes.c_void_p]),
    "ngap_features_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_void_p]),
    "ngap_mlp_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                       ctypes.POINTER(ctypes.c_void_p)]),
    "ngap_mlp_destroy": (None, [ctypes.c_void_p]),
    "ngap_mlp_train": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                      ctypes.POINTER(ctypes.c_float)]),
    "ngap_mlp_gradient": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_int64, ctypes.c_void_p,
                                         ctypes.POINTER(ctypes.c_float)]),
    "ngap_mlp_predict": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                        ctypes.c_int, ctypes.c_void_p]),
    "ngap_mlp_predict_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                             ctypes.c_int, ctypes.c_void_p]),
    "ngap_mlp_get_params": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                           ctypes.POINTER(ctypes.c_int64)]),
    "ngap_mlp_set_params": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]),
    "ngap_tableset_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_void_p)]),
    "ngap_tableset_destroy": (None, [ctypes.c_void_p]),
    "ngap_batch_match": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_uint64, ctypes.c_int,
                                        ctypes.POINTER(BatchStream), ctypes.c_int,
                                        ctypes.POINTER(BatchParams), ctypes.c_void_p]),
    "ngap_batch_results": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    "ngap_reports_sort_unique": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                                ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64),
                                                ctypes.c_void_p]),
    "ngap_reports_sort_unique_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64,
                                                        ctypes.c_void_p,
                                                        ctypes.POINTER(ctypes.c_uint64),
                                                        ctypes.c_void_p]),
    "ngap_cpu_validate_reference": (ctypes.c_int64, [ctypes.c_void_p, ctypes.c_void_p,
                                                     ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                                     ctypes.c_void_p, ctypes.c_int64,
                                                     ctypes.POINTER(ctypes.c_double)]),
    "ngap_last_error": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t]),
    "ngap_version": (ctypes.c_char_p, []),
}

_lib = None


def lib():
    """Loads libngap_b200.so once; raises if it is missing (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is not built; run __graft_entry__.build() or make -C ngap_b200/csrc")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error():
    buf = ctypes.create_string_buffer(2048)
    lib().ngap_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status):
    if status != NGAP_OK:
        raise NgapError(status, last_error())
    return status
