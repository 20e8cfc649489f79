"""Golden reports of the reference's own `ngap` command (fixtures under
tests/golden/ref_reports/, made by tests/golden/make_ref_reports.py, which
runs the reference built by oracle/Makefile on a GPU machine): the oracle
and the library's CPU checker (CPU) and the engine (GPU) must give exactly
the reports the reference printed for its GPU run and its CPU validator.
The fixture tests are skipped while no fixtures exist."""
import glob
import json
import os

import numpy as np
import pytest

import ngap_b200 as nb
from ngap_b200.engine import cpu_validate
from oracle import oracle

from golden.make_ref_reports import parse

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "ref_reports", "*.json")))


def test_parser_reads_the_reference_lines():
    out = ("Results number: 9\nUnique results number: 4\nvalidation start.\n"
           "Validation PASS!\nResult(4): \n0x400000005, 0x40000002f, 0x400000040, "
           "0x40000004b, \nReference result(4): \n0x400000005, 0x40000002f, 0x400000040, "
           "0x40000004b, \n\nngap elapsed time: 0.1 seconds, throughput = 1 MB/s \n")
    rec = parse(out)
    assert rec["raw"] == 9 and rec["unique"] == rec["cpu_unique"] == 4 and rec["validation"]
    assert rec["gpu"] == rec["cpu"] == [0x400000005, 0x40000002F, 0x400000040, 0x40000004B]
    empty = parse("Result(0): \n\nReference result(0): \n\n")
    assert empty["gpu"] == [] and empty["cpu"] == [] and not empty["validation"]


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


def _want(rec):
    if not (rec["complete"] and rec["returncode"] == 0):
        pytest.skip(f"{rec['case']} {rec['algorithm']}: the reference's output is incomplete")
    return np.array(rec["gpu"], dtype=np.uint64)


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_oracle_and_checker_reproduce_the_reference(built, path):
    rec, groups, ss, nseg, split, is_dup = _case(path)
    want = _want(rec)
    assert rec["validation"] and rec["cpu"] == rec["gpu"]  # the reference agreed with itself
    got, _ = oracle.match(groups.views(), ss, nseg, split, is_dup=is_dup)
    assert np.array_equal(got, want)
    assert np.array_equal(cpu_validate(groups, ss, nseg, split, is_dup), want)


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_engine_reproduces_the_reference(engine, path):
    rec, groups, ss, nseg, split, is_dup = _case(path)
    want = _want(rec)
    tables = nb.Tables(groups, precompute_depth=rec["options"]["precompute_depth"])
    got = engine.match(tables, ss, nseg, split, algorithm=rec["algorithm"], is_dup=is_dup,
                       unique=bool(rec["options"].get("unique")))
    assert np.array_equal(got, want)
