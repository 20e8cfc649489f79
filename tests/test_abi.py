"""The C-ABI library (CPU): loads, exports every declared symbol, and its
host-only entry points work without a GPU. Also the CLI's argument handling."""
import ctypes
import os
import re
import subprocess

import ngap_b200 as nb
from ngap_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ngap_b200.h")
CLI = os.path.join(ROOT, "ngap_b200", "bin", "ngap")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b(ngap_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_api():
    names = declared_functions()
    assert "ngap_match" in names and "ngap_reports_sort_unique_noalloc" in names
    assert len(names) >= 25


def test_library_exports_every_declared_symbol(built):
    L = nb.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert missing == []


def test_binding_covers_header(built):
    assert sorted(_lib.SIGNATURES) == declared_functions()


def test_host_entry_points_without_gpu(built):
    nfa = nb.Nfa.from_string(open(os.path.join(ROOT, "tests", "golden", "apple.anml")).read())
    assert (nfa.num_states, nfa.num_edges) == (5, 4)
    g = nb.Groups(nfa, group_num=3)
    assert g.count == 1 and g.cc_stats() == (1, 0, 0)
    assert nb.lib().ngap_version().startswith(b"ngap_b200")


def test_null_arguments_are_errors(built):
    L = nb.lib()
    assert L.ngap_nfa_load_anml(None, None) == 1
    assert L.ngap_groups_build(None, None, None) == 1
    assert L.ngap_match(None, None, None, 0, None, None) == 1
    assert "null" in _lib.last_error()


def test_cli_bad_args():
    r = subprocess.run([CLI, "--bogus", "1"], capture_output=True, text=True)
    assert r.returncode == 1 and "Error in command line" in r.stderr
    r = subprocess.run([CLI, "-a", "x.anml"], capture_output=True, text=True)
    assert r.returncode == 1


def test_cli_unknown_algorithm(tmp_path):
    inp = tmp_path / "in.txt"
    inp.write_bytes(b"apple" * 10)
    r = subprocess.run([CLI, "-a", os.path.join(ROOT, "tests", "golden", "apple.anml"), "-i",
                        str(inp), "--algorithm=nosuch", "--group-num=1"],
                       capture_output=True, text=True)
    assert r.returncode == 0
    assert "not supported algoritm nosuch" in r.stdout and "FINISHED!" in r.stdout


def test_scheduler_entry_points_reject_bad_arguments(built):
    L = nb.lib()
    assert L.ngap_engine_set_trace(None, 1) == 1
    assert L.ngap_trace_copy(None, None, 0, None) == 1
    assert L.ngap_tables_stats_get(None, None) == 1
    assert L.ngap_features(None, 0, 0, None, None, 1, 1024, None, None) == 1
    # a region whose offset + length wraps past 2^64 is out of range, not accepted
    data = (ctypes.c_uint8 * 16)()
    offs, lens = (ctypes.c_uint64 * 1)(2**64 - 1), (ctypes.c_uint64 * 1)(2)
    out = (ctypes.c_float * _lib.FEAT_BYTES)()
    assert L.ngap_features(data, 16, 0, offs, lens, 1, 1024, out, None) == 1
    assert "out of range" in _lib.last_error()
    assert L.ngap_mlp_train(None, None, None, 0, 1, 1, ctypes.c_float(0.1), None) == 1
    assert L.ngap_mlp_predict(None, None, 0, 0, None) == 1
    assert L.ngap_mlp_set_params(None, None, 0) == 1
    assert L.ngap_engine_device_bytes(None) == 0
    n = ctypes.c_int(-5)
    assert L.ngap_tiles_describe(None, None, None, 0, ctypes.byref(n)) == 1
    g = nb.Groups(nb.Nfa.from_string(open(os.path.join(ROOT, "tests", "golden",
                                                       "apple.anml")).read()), group_num=1)
    assert L.ngap_tiles_describe(g._h, None, None, 4, ctypes.byref(n)) == 1  # cap > 0, no out
    assert L.ngap_tiles_describe(g._h, None, None, 0, ctypes.byref(n)) == 0 and n.value == 1


def test_cli_help_and_new_flags():
    r = subprocess.run([CLI, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "--tile-mode" in r.stdout and "usage: ngap" in r.stdout
    r = subprocess.run([CLI, "--tile-mode", "x"], capture_output=True, text=True)
    assert r.returncode == 1 and "Unable to convert" in r.stderr


def test_cli_host_flow_before_the_device():
    """main.cu:45-102 before any device work: input slicing (shorter input
    sliced to its end), duplication, segment count, CC statistics. Without a
    GPU the command stops at the first device call with 255; with one it runs on."""
    apple = os.path.join(ROOT, "tests", "golden", "apple.anml")
    inp = os.path.join(ROOT, "tests", "golden", "apple_input.txt")
    r = subprocess.run([CLI, "-a", apple, "-i", inp, "--algorithm", "nonblockinggroups",
                        "--group-num=1", "--input-start-pos=70", "--input-len=50",
                        "--duplicate-input-stream=3", "--split-entire-inputstream-to-chunk-size=4",
                        "--unique=yes", "--validation=0"], capture_output=True, text=True, timeout=120)
    out = r.stdout
    assert r.returncode in (0, 255), r.stdout + r.stderr
    assert "input_stream_size = 81" in out
    assert "the input is shorter than the length specified, just slice to end" in out
    assert "total_state_number = 5" in out and "num_succeed 1, num_fail 0" in out
    assert "grouped_nfas.size = 1 pl.num_seg=8" in out  # 3 x 11 bytes in 4-byte segments
    assert "dup_input_stream = 3" in out and "split_entire_inputstream_to_chunk_size = 4" in out
    r = subprocess.run([CLI, "-a", apple, "-i", inp, "--unique=maybe"], capture_output=True,
                       text=True)
    assert r.returncode == 1 and "Unable to convert 'maybe'" in r.stderr
    r = subprocess.run([CLI, "-a", apple, "-i", os.path.join(ROOT, "no_such_input")],
                       capture_output=True, text=True)
    assert r.returncode == 255 and "no such input file" in r.stdout
