"""ngap_b200: B200-native automata processing (drop-in for ngAP's matching path).

Host API over the C ABI in include/ngap_b200.h; kernels are hand-written CUDA
for sm_100a in ngap_b200/csrc.
"""
from ._lib import ALGORITHMS, LIB_PATH, NgapError, lib  # noqa: F401
from .engine import (Engine, GroupGraph, Groups, Ngap, NgapOption, Nfa, Tables,  # noqa: F401
                     TableSet, batch_match_async, batch_results, cpu_validate, decode_reports,
                     split_by_stream)

__all__ = ["ALGORITHMS", "Engine", "GroupGraph", "Groups", "Ngap", "NgapOption", "Nfa", "Tables",
           "TableSet", "NgapError", "batch_match_async", "batch_results", "cpu_validate",
           "decode_reports", "lib", "LIB_PATH", "split_by_stream"]
