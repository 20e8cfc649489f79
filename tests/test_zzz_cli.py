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


def test_cli_tuning_picks_a_choice_then_runs_it(engine):
    """--tuning (ngap.cu:1995-2056): a grid of the engine's knobs, every
    choice checked against the first one's reports, then the run with the
    best choice and its usual lines."""
    r = _run("--algorithm=nonblockingallgroups", "--precompute-depth=3", "--tuning=true")
    assert r.returncode == 0, r.stdout + r.stderr
    out = r.stdout
    tries = re.findall(r"\[Tuning\] Try choice:", out)
    assert len(tries) == 5 * 5 * 3, len(tries)
    m = re.search(r"\[Tuning\] Tuning completed: the best choice is\n\s+window=(\d+), "
                  r"chunk=(\d+), active_threshold=(\d+)", out)
    assert m, out[-2000:]
    assert "Validation PASS!" in out and "0x400000005, 0x40000002f, 0x400000040, 0x40000004b" in out
    assert out.rstrip().endswith("FINISHED!")


def test_cli_motivate_worklist_length(engine, tmp_path):
    """--motivate-worklist-length (ngap.cu:1843-1866): the worklist work of
    every unit written to <app-name>.worklist.txt."""
    r = subprocess.run([CLI, "-a", os.path.join(GOLD, "apple.anml"), "-i",
                        os.path.join(GOLD, "apple_input.txt"), "--group-num=1",
                        "--algorithm=nonblockingpcgroups", "--precompute-depth=2",
                        "--split-entire-inputstream-to-chunk-size=27",
                        "--motivate-worklist-length=true", "--app-name=apple"],
                       capture_output=True, text=True, timeout=300, cwd=tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Save froniter length file to apple.worklist.txt" in r.stdout
    rows = [list(map(int, ln.split())) for ln in (tmp_path / "apple.worklist.txt").read_text()
            .splitlines()]
    assert rows and {row[0] for row in rows} == {0, 1, 2}  # three segments of 27 bytes
    assert all(0 <= row[2] < row[3] <= 27 and row[4] >= 0 for row in rows)
    assert sum(row[4] for row in rows) > 0
