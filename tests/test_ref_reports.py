"""Golden reports of the reference's own `ngap` command, built from the
reference sources by oracle/Makefile and run on a B200 by
tests/golden/make_ref_reports.py (fixtures under tests/golden/ref_reports/).

Every record holds the sorted unique reports of the reference's GPU run
("Result(N):") and of its CPU validator automataGroupsReference ("Reference
result(N):", code/src/ngap/ngap.cu:2171-2344).

* Small cases (complete lists, seven algorithms each): the oracle, the
  library's CPU checker (CPU) and the engine (GPU) must give exactly the
  reference GPU run's reports; the oracle with validator_quirk must give
  exactly the reference CPU validator's, which differ where a segment starts
  at an odd position (ngap.cu:2212: the validator then tests the empty
  frontiers[1] and reports nothing for that segment; apple_3seg, 27-byte
  segments, and apple_dup2, two 81-byte segments, show it).
* Benchmark cases at the benchmark's sizes (the literal set 1 MiB; the first
  3 MiB of the Hamming set as 3 x 1 MiB segments with 1 and 10 groups): the
  unique count and the first 40 sorted reports printed by the reference,
  against the engine at full size (GPU) and, where the oracle finishes in
  seconds, the oracle (CPU).
"""
import glob
import json
import os

import numpy as np
import pytest

import ngap_b200 as nb
from ngap_b200 import workloads as W
from ngap_b200.engine import cpu_validate
from oracle import oracle

from golden.make_ref_reports import parse

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "ref_reports")
SMALL = sorted(p for p in glob.glob(os.path.join(GOLD, "*.json"))
               if not os.path.basename(p).startswith("bench."))
BENCH = sorted(glob.glob(os.path.join(GOLD, "bench.*.json")))


def test_parser_reads_the_reference_lines():
    out = ("Results number: 9\nUnique results number: 4\nvalidation start.\n"
           "Reference CPU elapsed time: 52573 ms, 0.0598354 MB/s\n"
           "Validation PASS!\nResult(4): \n0x400000005, 0x40000002f, 0x400000040, "
           "0x40000004b, \nReference result(4): \n0x400000005, 0x40000002f, 0x400000040, "
           "0x40000004b, \n\nngap elapsed time: 0.1 seconds, throughput = 1 MB/s \n")
    rec = parse(out)
    assert rec["raw"] == 9 and rec["unique"] == rec["cpu_unique"] == 4 and rec["validation"]
    assert rec["gpu"] == rec["cpu"] == [0x400000005, 0x40000002F, 0x400000040, 0x40000004B]
    assert rec["cpu_ms"] == 52573 and rec["cpu_mbps"] == 0.0598354 and rec["gpu_mbps"] == 1.0
    empty = parse("Result(0): \n\nReference result(0): \n\n")
    assert empty["gpu"] == [] and empty["cpu"] == [] and not empty["validation"]


def test_fixtures_present():
    """Seven small cases x seven algorithms, and the benchmark-size records."""
    assert len(SMALL) == 49
    assert len(BENCH) == 4
    for p in SMALL + BENCH:
        rec = json.load(open(p))
        assert rec["returncode"] == 0, p


def _case(path):
    rec = json.load(open(path))
    base = os.path.join(os.path.dirname(path), rec["case"])
    anml = open(base + ".anml").read()
    data = np.fromfile(base + ".input", dtype=np.uint8)
    o = rec["options"]
    ss = np.tile(data, o["dup"])
    split = o["split"] if o["split"] > 0 else len(ss)
    nseg = len(ss) // split
    is_dup = o["dup"] > 1 and o["split"] in (-1, o["input_len"])  # main.cu via ngap_buffer.cu:479-484
    groups = nb.Groups(nb.Nfa.from_string(anml), group_num=o["group_num"])
    return rec, groups, ss[:nseg * split], nseg, split, is_dup


def _odd_start(nseg, split):
    return any((s * split) % 2 for s in range(nseg))


@pytest.mark.parametrize("path", SMALL, ids=[os.path.basename(p) for p in SMALL])
def test_oracle_and_checker_reproduce_the_reference(built, path):
    rec, groups, ss, nseg, split, is_dup = _case(path)
    assert rec["complete"]
    gpu = np.array(rec["gpu"], dtype=np.uint64)
    cpu = np.array(rec["cpu"], dtype=np.uint64)
    # the reference agrees with itself except through the validator's odd-start rule
    assert rec["validation"] == (not _odd_start(nseg, split) or np.array_equal(gpu, cpu))
    got, _ = oracle.match(groups.views(), ss, nseg, split, is_dup=is_dup,
                          unique=bool(rec["options"].get("unique")))
    assert np.array_equal(got, gpu)
    quirk, _ = oracle.match(groups.views(), ss, nseg, split, is_dup=is_dup, validator_quirk=True,
                            unique=bool(rec["options"].get("unique")))
    assert np.array_equal(quirk, cpu)
    assert np.array_equal(cpu_validate(groups, ss, nseg, split, is_dup), gpu)


def test_the_odd_start_cases_are_covered():
    """At least one fixture where the reference's validator and its GPU run
    disagree, so the quirk above is exercised."""
    diff = [p for p in SMALL if not json.load(open(p))["validation"]]
    assert any("apple_3seg" in p for p in diff) and any("apple_dup2" in p for p in diff)


@pytest.mark.gpu
@pytest.mark.parametrize("path", SMALL, ids=[os.path.basename(p) for p in SMALL])
def test_engine_reproduces_the_reference(engine, path):
    rec, groups, ss, nseg, split, is_dup = _case(path)
    want = np.array(rec["gpu"], dtype=np.uint64)
    tables = nb.Tables(groups, precompute_depth=rec["options"]["precompute_depth"])
    got = engine.match(tables, ss, nseg, split, algorithm=rec["algorithm"], is_dup=is_dup,
                       unique=bool(rec["options"].get("unique")))
    assert np.array_equal(got, want)


def _bench_case(path):
    rec = json.load(open(path))
    wl = rec["workload"]
    anml, data = getattr(W, wl["generator"])(seed=wl["seed"])
    data = data[:wl["input_bytes"]]
    o = rec["options"]
    groups = nb.Groups(nb.Nfa.from_string(anml), group_num=o["group_num"])
    return rec, groups, data, len(data) // o["split"], o["split"]


def test_bench_records_agree_with_themselves():
    for p in BENCH:
        rec = json.load(open(p))
        assert rec["validation"] and rec["unique"] == rec["cpu_unique"] and rec["gpu"] == rec["cpu"]
        assert len(rec["gpu"]) == min(40, rec["unique"])


@pytest.mark.parametrize("path", [p for p in BENCH if "literal" in p],
                         ids=lambda p: os.path.basename(p))
def test_oracle_reproduces_the_reference_at_benchmark_size(built, path):
    rec, groups, data, nseg, split = _bench_case(path)
    got, _ = oracle.match(groups.views(), data, nseg, split, nthreads=os.cpu_count() or 1)
    assert len(got) == rec["unique"]
    assert [int(x) for x in got[:40]] == rec["gpu"]


@pytest.mark.gpu
@pytest.mark.parametrize("path", BENCH, ids=lambda p: os.path.basename(p))
def test_engine_reproduces_the_reference_at_benchmark_size(engine, path):
    rec, groups, data, nseg, split = _bench_case(path)
    tables = nb.Tables(groups, precompute_depth=-1)
    got = engine.match(tables, data, nseg, split, algorithm=rec["algorithm"])
    assert len(got) == rec["unique"]
    assert [int(x) for x in got[:40]] == rec["gpu"]
