"""Golden reports from the reference's own `ngap` command, run on a GPU machine.

The reference writes no report file, but with --validation it prints the
sorted unique reports of its GPU run ("Result(N):") and of its CPU validator
("Reference result(N):", code/src/ngap/ngap.cu:2270-2344) in full when there
are at most 40. The cases below are small enough for that. For each case and
algorithm this writes tests/golden/ref_reports/<case>.<algorithm>.json with the
command's options, both report lists, the raw count and the validation
verdict, and the case's ANML and input next to them.

Build the reference first (outputs only in oracle/_ref/):
    make -C oracle -j8 ref-ngap
then, on a machine with a GPU, from the repo root:
    python tests/golden/make_ref_reports.py
"""
import json
import os
import re
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from ngap_b200 import workloads as W  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "ref_reports")
REF = os.path.join(ROOT, "oracle", "_ref", "ngap")
ALGOS = ["blockinggroups", "NAPgroups", "nonblockinggroups", "nonblockingr1groups",
         "nonblockingr2groups", "nonblockingpcgroups", "nonblockingallgroups"]


def cases():
    """(name, anml, input bytes, options). Group counts never exceed the CC
    count; NFAs with start-of-data states use one group (the reference's
    non-blocking seeding drops the group bits of their reports,
    ngap_buffer.cu:626-629)."""
    apple = open(os.path.join(ROOT, "tests", "golden", "apple.anml")).read()
    apple_in = open(os.path.join(ROOT, "tests", "golden", "apple_input.txt"), "rb").read()
    yield "apple_1seg", apple, apple_in, dict(group_num=1, split=81)
    yield "apple_3seg", apple, apple_in, dict(group_num=1, split=27)
    yield "apple_dup2", apple, apple_in, dict(group_num=1, split=81, dup=2)
    a, d = W.literal_set(seed=21, n_patterns=20, input_len=4096, plant_every=256)
    yield "literal_g3", a, d.tobytes(), dict(group_num=3, split=1024)
    a, d = W.hamming_set(seed=22, n_patterns=2, k=12, input_len=2048, plant_every=512)
    yield "hamming_g2", a, d.tobytes(), dict(group_num=2, split=1024)
    a, d = W.levenshtein_set(seed=23, n_patterns=2, k=10, input_len=1024, plant_every=512)
    yield "levenshtein_g2", a, d.tobytes(), dict(group_num=2, split=1024)
    a, d = W.dotstar_set(seed=24, n_patterns=6, input_len=1024, plant_every=256)
    yield "dotstar_g2", a, d.tobytes(), dict(group_num=2, split=512, unique=True)


def parse(out):
    def hexes(label):
        m = re.search(re.escape(label) + r"\((\d+)\):\s*\n([^\n]*)", out)
        if not m:
            return None, None
        vals = [int(x, 16) for x in re.findall(r"0x[0-9a-f]+", m.group(2))]
        return int(m.group(1)), vals
    raw = re.search(r"Results number: (\d+)", out)
    n_gpu, gpu = hexes("Result")
    n_cpu, cpu = hexes("Reference result")
    return {"raw": int(raw.group(1)) if raw else None, "unique": n_gpu, "gpu": gpu,
            "cpu_unique": n_cpu, "cpu": cpu, "validation": "Validation PASS!" in out}


def main():
    if not os.path.exists(REF):
        raise SystemExit("build the reference first: make -C oracle -j8 ref-ngap")
    os.makedirs(OUT, exist_ok=True)
    for name, anml, data, o in cases():
        a_path = os.path.join(OUT, name + ".anml")
        i_path = os.path.join(OUT, name + ".input")
        open(a_path, "w").write(anml)
        open(i_path, "wb").write(data)
        dup = o.get("dup", 1)
        for algo in ALGOS:
            args = [REF, "-a", a_path, "-i", i_path, f"--algorithm={algo}",
                    f"--group-num={o['group_num']}", "--input-start-pos=0",
                    f"--input-len={len(data)}",
                    f"--split-entire-inputstream-to-chunk-size={o['split']}",
                    f"--duplicate-input-stream={dup}", "--validation=true",
                    "--precompute-depth=2", f"--unique={'true' if o.get('unique') else 'false'}"]
            r = subprocess.run(args, capture_output=True, text=True, timeout=120)
            rec = parse(r.stdout)
            rec.update({"case": name, "algorithm": algo, "returncode": r.returncode,
                        "options": dict(o, dup=dup, input_len=len(data), precompute_depth=2),
                        "command": " ".join(os.path.relpath(x, ROOT) if x.startswith(ROOT) else x
                                            for x in args)})
            complete = rec["unique"] is not None and rec["unique"] <= 40 and rec["gpu"] is not None
            rec["complete"] = bool(complete and len(rec["gpu"]) == rec["unique"])
            with open(os.path.join(OUT, f"{name}.{algo}.json"), "w") as f:
                json.dump(rec, f, indent=1)
            print(name, algo, "rc", r.returncode, "unique", rec["unique"], "validation",
                  rec["validation"], "complete", rec["complete"])


if __name__ == "__main__":
    main()
