"""Test infrastructure (oracle), not product code.

ctypes front for liboracle.so (oracle/ngap_oracle.c), the C restatement of the
reference CPU matcher automataGroupsReference (code/src/ngap/ngap.cu:2171-2268)
and of its sort/unique validation (ngap.cu:2270-2344). Used only by tests, the
smoke check and the CPU-baseline leg of bench.py.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


class OracleGroup(ctypes.Structure):
    _fields_ = [("V", ctypes.c_int32),
                ("row_offsets", ctypes.c_void_p), ("cols", ctypes.c_void_p),
                ("bits", ctypes.c_void_p), ("attrs", ctypes.c_void_p),
                ("naas", ctypes.c_int32), ("aas", ctypes.c_void_p),
                ("nstart", ctypes.c_int32), ("starts", ctypes.c_void_p)]


class OracleStats(ctypes.Structure):
    _fields_ = [("matched", ctypes.c_uint64), ("matched_deg", ctypes.c_uint64),
                ("reports_raw", ctypes.c_uint64), ("frontier", ctypes.c_uint64)]


_L = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def lib():
    global _L
    if _L is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.oracle_match.restype = ctypes.c_int64
        L.oracle_match.argtypes = [ctypes.POINTER(OracleGroup), ctypes.c_int, ctypes.c_void_p,
                                   ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_int64,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(OracleStats)]
        L.oracle_last_needed.restype = ctypes.c_int64
        _L = L
    return _L


def _field(g, name):
    if isinstance(g, dict):
        return g[name]
    return getattr(g, name)


def match(groups, data, num_seg, seg_len, is_dup=False, mode=1, unique=False, nthreads=0,
          first_segment=0, validator_quirk=False):
    """Returns (sorted unique reports as uint64 in the reference encoding, stats dict).
    `groups` items expose row_offsets, col_indices, symbol_sets, node_attrs,
    always_active, start_states (dicts or objects). validator_quirk reproduces
    the reference CPU validator's odd-start rule (ngap_oracle.h): segments
    that start at an odd position report nothing."""
    keep = []
    arr = (OracleGroup * max(1, len(groups)))()
    for i, g in enumerate(groups):
        ro = np.ascontiguousarray(_field(g, "row_offsets"), dtype=np.int32)
        co = np.ascontiguousarray(_field(g, "col_indices"), dtype=np.int32)
        bi = np.ascontiguousarray(_field(g, "symbol_sets"), dtype=np.uint32)
        at = np.ascontiguousarray(_field(g, "node_attrs"), dtype=np.uint8)
        aa = np.ascontiguousarray(_field(g, "always_active"), dtype=np.int32)
        st = np.ascontiguousarray(_field(g, "start_states"), dtype=np.int32)
        keep += [ro, co, bi, at, aa, st]
        arr[i] = OracleGroup(len(at), ro.ctypes.data, co.ctypes.data, bi.ctypes.data,
                             at.ctypes.data, len(aa), aa.ctypes.data, len(st), st.ctypes.data)
    d = np.ascontiguousarray(data, dtype=np.uint8)
    cap = 1 << 16
    stats = OracleStats()
    while True:
        out = np.zeros(cap, dtype=np.uint64)
        n = lib().oracle_match(arr, len(groups), d.ctypes.data, num_seg, seg_len, int(is_dup),
                               first_segment, mode, int(unique), int(bool(validator_quirk)),
                               nthreads, out.ctypes.data, cap, ctypes.byref(stats))
        if n >= 0:
            break
        cap = max(cap * 2, int(lib().oracle_last_needed()) + 1)
    return out[:n], {"matched": stats.matched, "matched_deg": stats.matched_deg,
                     "reports_raw": stats.reports_raw, "frontier": stats.frontier}
