"""Golden reports from the reference's own `ngap` command, run on a GPU machine.

The reference writes no report file, but with --validation it prints the
sorted unique reports of its GPU run ("Result(N):") and of its CPU validator
("Reference result(N):", code/src/ngap/ngap.cu:2270-2344): in full when there
are at most 40, else the first 40.

Two sets of fixtures:

* small cases (at most 40 reports, so both lists are complete) x the seven
  algorithms: <case>.<algorithm>.json with the command's options, both report
  lists, the raw count and the validation verdict, and the case's ANML and
  input next to them;
* benchmark cases at the benchmark's own sizes (the literal set, 1 MiB, one
  segment; the first 3 MiB of the Hamming set as 3 x 1 MiB segments, with 1
  and 10 groups): bench.<case>.<algorithm>.json with the unique count, the
  first 40 sorted reports of both runs, the verdict and the two elapsed-time
  lines. Their inputs are regenerated from the seeded generators named in the
  record, so only the record is committed.

Build the reference first (outputs only in oracle/_ref/):
    make -C oracle -j8 ref-ngap
then, on a machine with a GPU, from the repo root:
    python tests/golden/make_ref_reports.py [--out DIR] [--only small|bench|all]
"""
import argparse
import json
import os
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from ngap_b200 import workloads as W  # noqa: E402
from oracle import refcli  # noqa: E402
from oracle.refcli import parse  # noqa: E402,F401

OUT = os.path.join(ROOT, "tests", "golden", "ref_reports")
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


# benchmark-size cases: (name, generator, seed, input bytes used, options, algorithms)
BENCH = [
    ("literal_c1", "literal_set", 1, 1 << 20, dict(group_num=1, split=1 << 20),
     ["blockinggroups", "nonblockingallgroups"]),
    ("hamming_c2_g1", "hamming_set", 2, 3 << 20, dict(group_num=1, split=1 << 20),
     ["nonblockingallgroups"]),
    ("hamming_c2_g10", "hamming_set", 2, 3 << 20, dict(group_num=10, split=1 << 20),
     ["nonblockingallgroups"]),
]


def bench_input(gen, seed, n):
    """The ANML and the first n input bytes of a benchmark workload."""
    anml, data = getattr(W, gen)(seed=seed)
    return anml, data[:n].tobytes()


def command(a_path, i_path, n, algo, o, depth):
    return refcli.command(a_path, i_path, n, algo, o["group_num"], o["split"], depth=depth,
                          dup=o.get("dup", 1), unique=bool(o.get("unique")))


def rel(args):
    return " ".join(os.path.relpath(x, ROOT) if x.startswith(ROOT) else x for x in args)


def small(out):
    for name, anml, data, o in cases():
        a_path = os.path.join(out, name + ".anml")
        i_path = os.path.join(out, name + ".input")
        open(a_path, "w").write(anml)
        open(i_path, "wb").write(data)
        dup = o.get("dup", 1)
        for algo in ALGOS:
            args = command(a_path, i_path, len(data), algo, o, 2)
            rc, text = refcli.run(args, 120)
            rec = parse(text)
            rec.update({"case": name, "algorithm": algo, "returncode": rc,
                        "options": dict(o, dup=dup, input_len=len(data), precompute_depth=2),
                        "command": rel(args)})
            complete = rec["unique"] is not None and rec["unique"] <= 40 and rec["gpu"] is not None
            rec["complete"] = bool(complete and len(rec["gpu"]) == rec["unique"])
            with open(os.path.join(out, f"{name}.{algo}.json"), "w") as f:
                json.dump(rec, f, indent=1)
            print(name, algo, "rc", rc, "unique", rec["unique"], "validation",
                  rec["validation"], "complete", rec["complete"], flush=True)


def bench(out, depth=3):
    tmp = tempfile.mkdtemp(prefix="ngap_ref_")
    for name, gen, seed, n, o, algos in BENCH:
        anml, data = bench_input(gen, seed, n)
        a_path = os.path.join(tmp, name + ".anml")
        i_path = os.path.join(tmp, name + ".input")
        open(a_path, "w").write(anml)
        open(i_path, "wb").write(data)
        for algo in algos:
            args = command(a_path, i_path, n, algo, o, depth)
            rc, text = refcli.run(args, 1500)
            rec = parse(text)
            rec.update({"case": name, "algorithm": algo, "returncode": rc,
                        "workload": {"generator": gen, "seed": seed, "input_bytes": n},
                        "options": dict(o, dup=1, input_len=n, precompute_depth=depth),
                        "command": rel(args).replace(tmp, "<tmp>")})
            with open(os.path.join(out, f"bench.{name}.{algo}.json"), "w") as f:
                json.dump(rec, f, indent=1)
            print(name, algo, "rc", rc, "unique", rec["unique"], "cpu_unique",
                  rec["cpu_unique"], "validation", rec["validation"], "gpu MB/s",
                  rec["gpu_mbps"], "cpu MB/s", rec["cpu_mbps"], flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=OUT)
    ap.add_argument("--only", default="all", choices=["small", "bench", "all"])
    a = ap.parse_args()
    if not refcli.available():
        raise SystemExit("build the reference first: make -C oracle -j8 ref-ngap")
    os.makedirs(a.out, exist_ok=True)
    if a.only in ("small", "all"):
        small(a.out)
    if a.only in ("bench", "all"):
        bench(a.out)


if __name__ == "__main__":
    main()
