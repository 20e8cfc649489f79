"""Test infrastructure (oracle), not product code.

Runs the reference's own `ngap` command, built from the reference sources by
`make -C oracle ref-ngap` into oracle/_ref/ngap (when the reference checkout
was present at build time), and reads the lines it prints:

* "Results number: N" and "Unique results number: N" (code/src/ngap/ngap.cu:
  1841, 1928);
* "Result(N):" / "Reference result(N):" followed by the first 40 sorted unique
  reports of its GPU run and of its CPU validator (ngap.cu:2270-2292);
* "Validation PASS!" (ngap.cu:2335);
* "ngap elapsed time: S seconds, throughput = X MB/s" (ngap.cu:1981-1989);
* "Reference CPU elapsed time: T ms, Y MB/s" (ngap.cu:2261-2267), the timing
  of the reference CPU matcher automataGroupsReference (ngap.cu:2171-2268),
  one OpenMP thread per (group, segment).

Used by tests/golden/make_ref_reports.py (golden fixtures) and by bench.py's
reference arm and CPU baseline. The command needs a GPU even for its CPU
validator (its buffers come from cudaMalloc, code/include/commons/array2.h:
42-48).
"""
import os
import re
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REF_NGAP = os.path.join(HERE, "_ref", "ngap")


def available():
    return os.access(REF_NGAP, os.X_OK)


def parse(out):
    """The reference's stdout lines as a dict (None where a line is absent)."""
    def hexes(label):
        m = re.search(r"(?m)^" + re.escape(label) + r"\((\d+)\):\s*\n([^\n]*)", out)
        if not m:
            return None, None
        vals = [int(x, 16) for x in re.findall(r"0x[0-9a-f]+", m.group(2))]
        return int(m.group(1)), vals
    raw = re.search(r"Results number: (\d+)", out)
    uq = re.search(r"Unique results number: (\d+)", out)
    n_gpu, gpu = hexes("Result")
    n_cpu, cpu = hexes("Reference result")
    gt = re.search(r"ngap elapsed time: ([0-9.e+-]+) seconds, (?:throughput = |WRONGTHRPUT\()"
                   r"([0-9.e+-]+)", out)
    ct = re.search(r"Reference CPU elapsed time: (\d+) ms, ([0-9.e+-]+) MB/s", out)
    return {"raw": int(raw.group(1)) if raw else None,
            "unique": n_gpu if n_gpu is not None else (int(uq.group(1)) if uq else None),
            "gpu": gpu, "cpu_unique": n_cpu, "cpu": cpu,
            "validation": "Validation PASS!" in out,
            "gpu_seconds": float(gt.group(1)) if gt else None,
            "gpu_mbps": float(gt.group(2)) if gt else None,
            "cpu_ms": int(ct.group(1)) if ct else None,
            "cpu_mbps": float(ct.group(2)) if ct else None}


def command(anml_path, input_path, n, algorithm, group_num, split, depth=0, dup=1,
            validation=True, unique=False, extra=()):
    return [REF_NGAP, "-a", anml_path, "-i", input_path, f"--algorithm={algorithm}",
            f"--group-num={group_num}", "--input-start-pos=0", f"--input-len={n}",
            f"--split-entire-inputstream-to-chunk-size={split}",
            f"--duplicate-input-stream={dup}", f"--validation={'true' if validation else 'false'}",
            f"--precompute-depth={depth}", f"--unique={'true' if unique else 'false'}",
            *extra]


def run(args, timeout, env=None):
    """(return code, stdout) of one run of the reference command."""
    r = subprocess.run(args, capture_output=True, text=True, timeout=timeout, env=env)
    return r.returncode, r.stdout
