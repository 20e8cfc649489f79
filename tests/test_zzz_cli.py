"""The reference-compatible command line on the GPU (the drop-in boundary):
the apple example (README.md:156-186 of the reference) through every
--algorithm, with the stdout lines the reference's experiment scripts parse
(code/scripts/launch_exps.py:443-458), --validation against the library's
CPU checker, the binary report dump, and --report-off with
--quick-validation."""
import os
import re
import subprocess

import numpy as np
import pytest

import ngap_b200 as nb

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "ngap_b200", "bin", "ngap")
GOLD = os.path.join(ROOT, "tests", "golden")
KAT = [0x400000005, 0x40000002F, 0x400000040, 0x40000004B]


def _run(*args):
    return subprocess.run([CLI, "-a", os.path.join(GOLD, "apple.anml"), "-i",
                           os.path.join(GOLD, "apple_input.txt"), "--group-num=1", *args],
                          capture_output=True, text=True, timeout=300)


@pytest.mark.parametrize("algo", list(nb.ALGORITHMS))
def test_cli_apple(engine, tmp_path, algo):
    dump = tmp_path / "reports.bin"
    r = _run(f"--algorithm={algo}", "--precompute-depth=3", "--dump-reports", str(dump))
    assert r.returncode == 0, r.stdout + r.stderr
    out = r.stdout
    assert "Unique results number: 4" in out and "Validation PASS!" in out, out
    assert "0x400000005, 0x40000002f, 0x400000040, 0x40000004b" in out
    m = re.search(r"ngap elapsed time: (\S+) seconds, throughput = (\S+) MB/s", out)
    assert m and float(m.group(1)) > 0 and float(m.group(2)) > 0, out
    assert out.rstrip().endswith("FINISHED!")
    assert np.fromfile(dump, dtype=np.uint64).tolist() == KAT


def test_cli_report_off_quick_validation(engine):
    r = _run("--algorithm=nonblockingallgroups", "--report-off=true", "--quick-validation=4")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Quick Validation PASS! (report off)" in r.stdout, r.stdout
    assert int(re.search(r"Results number: (\d+)", r.stdout).group(1)) >= 4
