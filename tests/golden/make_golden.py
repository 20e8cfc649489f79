"""Generates the golden group-graph fixtures from the reference's own front-end.

Writes tests/golden/cases/<name>.anml (seeded synthetic automata plus
hand-written syntax cases) and, for each group count, the dump of
oracle/_ref/ref_frontend — the reference's NFALoader / NFA / nfa_utils sources
compiled by oracle/Makefile — as tests/golden/cases/<name>.g<k>.ref.txt.
Run from the repo root where the reference checkout exists:

    make -C oracle ref && python tests/golden/make_golden.py
"""
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from ngap_b200 import workloads as W  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "cases")
REF = os.path.join(ROOT, "oracle", "_ref", "ref_frontend")


def syntax_cases():
    """STEs exercising the VASim symbol-set grammar and XML attribute rules."""
    sets = ["*", ".", "[a-z]", "[^abc]", "\\x41", "[\\x41-\\x5a]", "\\n", "[\\t\\r]", "[\\[\\]]",
            "[a-]", "[-a]", "\\d", "\\w", "\\s", "[\\^]", "&lt;", "&amp;&gt;", "&#65;", "&#200;",
            "[{}]", "\\{", "[\\x7f-\\xff]", "a-c", "[^\\x00-\\x1f]", "\\\\", "[\\-]", "\\q",
            "[\\a\\b\\f\\v]", "[&quot;']", "[&#9;]", "x", "[abc\n]", "^", "[]"]
    w = W.AnmlWriter("syntax")
    n = len(sets)
    for i, s in enumerate(sets):
        tg = [f"s{i + 1}"] if i + 1 < n else []
        start = "all-input" if i % 5 == 0 else ("start-of-data" if i % 7 == 3 else None)
        w.ste(f"s{i}", None, tg, start=start, report=(i % 3 == 2), symbol_set=s)
    return w.text()


def degree_stress(seed, nccs, p_dense):
    """Several small CCs with out-degrees above 4: fan-out hubs (with and
    without self-loops, chained hubs sharing targets) that the limiter splits
    into "_dup_" clones, and dense CCs that it cannot limit and the reference
    drops. Nodes of different CCs are interleaved in the file to exercise the
    CC numbering."""
    rng = np.random.default_rng(seed)
    ccs = []
    for c in range(nccs):
        n = int(rng.integers(5, 14))
        adj = [set() for _ in range(n)]
        if rng.random() < p_dense:
            for i in range(n):
                for j in range(n):
                    if rng.random() < 0.6:
                        adj[i].add(j)
        else:
            for i in range(n - 1):
                adj[i].add(i + 1)
            for h in rng.choice(n, size=int(rng.integers(1, 3)), replace=False):
                for j in rng.choice(n, size=int(rng.integers(5, min(n, 10) + 1)), replace=False):
                    adj[h].add(int(j))
                if rng.random() < 0.5:
                    adj[h].add(int(h))
        ccs.append((n, adj))
    order = [(c, i) for c, (n, _) in enumerate(ccs) for i in range(n)]
    rng.shuffle(order)
    w = W.AnmlWriter("degree")
    for c, i in order:
        n, adj = ccs[c]
        tg = [f"c{c}v{j}" for j in adj[i]]
        rng.shuffle(tg)
        syms = rng.choice(np.arange(97, 103), size=int(rng.integers(1, 4)), replace=False)
        start = "all-input" if rng.random() < 0.3 else ("start-of-data" if rng.random() < 0.2 else None)
        w.ste(f"c{c}v{i}", syms, tg, start=start, report=rng.random() < 0.3)
    return w.text()


def cases():
    yield "apple", open(os.path.join(ROOT, "tests", "golden", "apple.anml")).read(), [1]
    yield "literal", W.literal_set(seed=21, n_patterns=20, input_len=64)[0], [1, 3]
    yield "hamming", W.hamming_set(seed=22, n_patterns=2, k=12, input_len=64)[0], [2]
    yield "levenshtein", W.levenshtein_set(seed=23, n_patterns=2, k=10, input_len=64)[0], [2]
    yield "dotstar", W.dotstar_set(seed=24, n_patterns=6, input_len=256)[0], [4]
    yield "syntax", syntax_cases(), [1, 2]
    for k, (nccs, pd) in enumerate([(6, 0.0), (8, 0.3), (10, 0.2), (5, 0.5)]):
        yield f"degree{k}", degree_stress(100 + k, nccs, pd), [1, 3]


def main():
    if not os.path.exists(REF):
        raise SystemExit("build the reference front-end first: make -C oracle ref")
    os.makedirs(OUT, exist_ok=True)
    for name, anml, gnums in cases():
        path = os.path.join(OUT, name + ".anml")
        with open(path, "w") as f:
            f.write(anml)
        for g in gnums:
            dump = os.path.join(OUT, f"{name}.g{g}.ref.txt")
            subprocess.run([REF, path, str(g), dump], check=True, stdout=subprocess.DEVNULL)
            print("wrote", os.path.relpath(dump, ROOT))


if __name__ == "__main__":
    main()
