"""Seeded synthetic workloads with the shapes of the benchmark configurations.

The reference measures on ANMLZoo/AutomataZoo files that are not available
here; these generators stand in for them with the same kinds of automata and
inputs. Every generator is deterministic in its seed and returns the ANML
text plus the input bytes.

  literal_set       64 literals of 8-16 printable bytes, 10% of positions
                    widened to classes of 2-20 symbols, all-input starts;
                    1 MiB uniform printable input, one planted occurrence per
                    16 KiB.                   (786 STEs; the config estimates ~1.2k)
  hamming_set       1000 random ACGT 25-mers, <= 3 substitutions; 16 MiB of
                    uniform ACGT with mutated copies every 64 KiB. Each 25-mer
                    has a matched and a mismatched STE per (position, errors),
                    166 STEs per pattern.                        (~166k STEs)
  levenshtein_set   ACGT 20-mers, edit distance <= 2 (substitution, insertion,
                    deletion), all-input starts.
  dotstar_set       literal(6-10) .* literal(6-10) over printable ASCII drawn
                    from a Zipf(1.1) symbol law; a fraction of the .* states is
                    always active.
  high_frontier     500 Levenshtein + 2000 dot-star regexes; 16 MiB ACGT +
                    16 MiB Zipf ASCII.   (101k STEs: 135 per Levenshtein 20-mer,
                    17 per dot-star regex; the config estimates ~250k)
"""
import numpy as np

ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)
PRINTABLE = np.arange(0x20, 0x7F, dtype=np.uint8)


def _cls(symbols):
    """VASim symbol set for a set of byte values, every byte hex-escaped."""
    syms = sorted(set(int(s) for s in symbols))
    return "[" + "".join("\\x%02x" % s for s in syms) + "]"


class AnmlWriter:
    def __init__(self, name="synthetic"):
        self.name = name
        self.parts = []
        self.count = 0

    def ste(self, sid, symbols, targets=(), start=None, report=False, symbol_set=None):
        ss = symbol_set if symbol_set is not None else _cls(symbols)
        attrs = f'id="{sid}" symbol-set="{ss}"'
        if start:
            attrs += f' start="{start}"'
        body = "".join(f'<activate-on-match element="{t}"/>' for t in targets)
        if report:
            body += '<report-on-match reportcode="1"/>'
        self.parts.append(f"<state-transition-element {attrs}>{body}</state-transition-element>\n")
        self.count += 1

    def text(self):
        return ('<anml version="1.0">\n<automata-network id="%s">\n' % self.name
                + "".join(self.parts) + "</automata-network>\n</anml>\n")


def _sample_from(rng, cls, n):
    return rng.choice(np.asarray(sorted(cls), dtype=np.uint8), size=n)


def literal_set(seed=1, n_patterns=64, len_lo=8, len_hi=16, class_frac=0.10, class_lo=2,
                class_hi=20, input_len=1 << 20, plant_every=16 << 10):
    """Literals with a few widened positions (the plain single-stream shape):
    (ANML, uniform printable input with occurrences planted every
    plant_every bytes)."""
    rng = np.random.default_rng(seed)
    w = AnmlWriter("literal_set")
    pats = []
    for p in range(n_patterns):
        L = int(rng.integers(len_lo, len_hi + 1))
        classes = []
        for _ in range(L):
            if rng.random() < class_frac:
                k = int(rng.integers(class_lo, class_hi + 1))
                classes.append(set(rng.choice(PRINTABLE, size=k, replace=False).tolist()))
            else:
                classes.append({int(rng.choice(PRINTABLE))})
        pats.append(classes)
        for i, c in enumerate(classes):
            w.ste(f"p{p}_{i}", c, targets=[f"p{p}_{i + 1}"] if i + 1 < L else [],
                  start="all-input" if i == 0 else None, report=(i == L - 1))
    data = rng.choice(PRINTABLE, size=input_len).astype(np.uint8)
    for pos in range(plant_every // 2, input_len, plant_every):
        classes = pats[int(rng.integers(len(pats)))]
        occ = [int(rng.choice(sorted(c))) for c in classes]
        if pos + len(occ) <= input_len:
            data[pos:pos + len(occ)] = occ
    return w.text(), data


def _hamming_pattern(w, tag, pat, d):
    L = len(pat)
    nm = lambda k, i, e: f"{tag}{k}{i}_{e}"  # noqa: E731
    for i in range(L):
        c = int(pat[i])
        other = [int(x) for x in ACGT if x != c]
        for e in range(0, min(i, d) + 1):  # matched p[i] with e errors so far
            tg = []
            if i + 1 < L:
                tg.append(nm("m", i + 1, e))
                if e + 1 <= d:
                    tg.append(nm("x", i + 1, e + 1))
            w.ste(nm("m", i, e), [c], tg, start="all-input" if (i == 0 and e == 0) else None,
                  report=(i == L - 1))
        for e in range(1, min(i + 1, d) + 1):  # mismatched p[i]; e errors including it
            tg = []
            if i + 1 < L:
                tg.append(nm("m", i + 1, e))
                if e + 1 <= d:
                    tg.append(nm("x", i + 1, e + 1))
            w.ste(nm("x", i, e), other, tg, start="all-input" if (i == 0 and e == 1) else None,
                  report=(i == L - 1))


def hamming_set(seed=2, n_patterns=1000, k=25, d=3, input_len=16 << 20, plant_every=64 << 10):
    """Hamming-distance k-mer automata (<= d substitutions): (ANML, uniform
    ACGT input with copies carrying 0..d substitutions every plant_every)."""
    rng = np.random.default_rng(seed)
    w = AnmlWriter("hamming_set")
    pats = rng.choice(ACGT, size=(n_patterns, k))
    for p in range(n_patterns):
        _hamming_pattern(w, f"h{p}", pats[p], d)
    data = rng.choice(ACGT, size=input_len).astype(np.uint8)
    for pos in range(plant_every // 2, input_len - k, plant_every):
        occ = pats[int(rng.integers(n_patterns))].copy()
        nsub = int(rng.integers(0, d + 1))
        for j in rng.choice(k, size=nsub, replace=False):
            occ[j] = rng.choice([x for x in ACGT if x != occ[j]])
        data[pos:pos + k] = occ
    return w.text(), data


def _levenshtein_pattern(w, tag, pat, d):
    """Homogeneous Levenshtein automaton: STE kinds by the symbol consumed on
    entry: M (matches p[i-1], advances), S (any other ACGT, advances, +1),
    I (any ACGT, insertion, +1). Deletions (+1, no symbol) are folded into the
    successor lists (up to the remaining budget)."""
    L = len(pat)
    states = {}

    def sid(kind, i, e):
        return f"{tag}{kind}{i}_{e}"

    def succ(i, e):
        out = []
        for k in range(0, d - e + 1):  # k deletions before the next symbol
            j, ee = i + k, e + k
            if j < L:
                out.append(("M", j + 1, ee))
                if ee + 1 <= d:
                    out.append(("S", j + 1, ee + 1))
            if ee + 1 <= d and 1 <= j < L:
                out.append(("I", j, ee + 1))
        return out

    # enumerate reachable states from the virtual start (0, 0)
    todo = succ(0, 0)
    starts = set(todo)
    seen = set()
    order = []
    while todo:
        s = todo.pop(0)
        if s in seen:
            continue
        seen.add(s)
        order.append(s)
        todo.extend(x for x in succ(s[1], s[2]) if x not in seen)
    for (kind, i, e) in sorted(order, key=lambda x: (x[1], x[2], x[0])):
        if kind == "M":
            syms = [int(pat[i - 1])]
        elif kind == "S":
            syms = [int(x) for x in ACGT if x != pat[i - 1]]
        else:
            syms = [int(x) for x in ACGT]
        rep = e + (L - i) <= d
        w.ste(sid(kind, i, e), syms, [sid(*t) for t in succ(i, e)],
              start="all-input" if (kind, i, e) in starts else None, report=rep)
        states[(kind, i, e)] = True
    return len(states)


def levenshtein_set(seed=3, n_patterns=500, k=20, d=2, input_len=16 << 20, plant_every=64 << 10,
                    writer=None, rng=None):
    """Edit-distance (<= d) automata on ACGT k-mers: (ANML, uniform ACGT input
    with edited copies every plant_every). With `writer` the STEs go into
    that writer and the ANML returned is None."""
    rng = rng if rng is not None else np.random.default_rng(seed)
    w = writer if writer is not None else AnmlWriter("levenshtein_set")
    pats = rng.choice(ACGT, size=(n_patterns, k))
    for p in range(n_patterns):
        _levenshtein_pattern(w, f"l{p}", pats[p], d)
    data = rng.choice(ACGT, size=input_len).astype(np.uint8)
    for pos in range(plant_every // 2, input_len - k - d, plant_every):
        occ = list(pats[int(rng.integers(n_patterns))])
        for _ in range(int(rng.integers(0, d + 1))):
            op = int(rng.integers(3))
            j = int(rng.integers(len(occ)))
            if op == 0:
                occ[j] = rng.choice([x for x in ACGT if x != occ[j]])
            elif op == 1:
                occ.insert(j, rng.choice(ACGT))
            elif len(occ) > 1:
                del occ[j]
        data[pos:pos + len(occ)] = occ
    return (w.text() if writer is None else None), data


def zipf_ascii(rng, n, s=1.1):
    """(symbol order, probabilities, n bytes) of a Zipf(s) law over printable
    ASCII in a random symbol order."""
    ranks = np.arange(1, len(PRINTABLE) + 1, dtype=np.float64)
    prob = ranks ** (-s)
    prob /= prob.sum()
    perm = rng.permutation(PRINTABLE)
    return perm, prob, rng.choice(perm, size=n, p=prob).astype(np.uint8)


def dotstar_set(seed=4, n_patterns=2000, lit_lo=6, lit_hi=10, aas_frac=0.30, input_len=16 << 20,
                plant_every=64 << 10, writer=None, rng=None, zipf_s=1.1):
    """literal .* literal regexes over Zipf ASCII, the .* always active in a
    fraction aas_frac of them: (ANML, Zipf input with both literals planted
    every plant_every, up to 15 bytes apart). With `writer` as in
    levenshtein_set."""
    rng = rng if rng is not None else np.random.default_rng(seed)
    w = writer if writer is not None else AnmlWriter("dotstar_set")
    perm, prob, data = zipf_ascii(rng, input_len, zipf_s)
    pats = []
    for p in range(n_patterns):
        a = rng.choice(perm, size=int(rng.integers(lit_lo, lit_hi + 1)), p=prob)
        b = rng.choice(perm, size=int(rng.integers(lit_lo, lit_hi + 1)), p=prob)
        pats.append((a, b))
        star = f"d{p}s"
        for i, c in enumerate(a):
            if i + 1 < len(a):
                tg = [f"d{p}a{i + 1}"]
            else:
                tg = [star, f"d{p}b0"]
            w.ste(f"d{p}a{i}", [int(c)], tg, start="all-input" if i == 0 else None)
        w.ste(star, None, [star, f"d{p}b0"], symbol_set="*",
              start="all-input" if rng.random() < aas_frac else None)
        for i, c in enumerate(b):
            w.ste(f"d{p}b{i}", [int(c)], [f"d{p}b{i + 1}"] if i + 1 < len(b) else [],
                  report=(i == len(b) - 1))
    for pos in range(plant_every // 2, input_len - 64, plant_every):
        a, b = pats[int(rng.integers(n_patterns))]
        gap = int(rng.integers(0, 16))
        occ = np.concatenate([a, data[pos:pos + gap], b])
        data[pos:pos + len(occ)] = occ
    return (w.text() if writer is None else None), data


def high_frontier(seed=3, n_lev=500, n_dot=2000, half=16 << 20):
    """The high-frontier mix: Levenshtein automata over the first half of the
    input (ACGT) and dot-star regexes over the second (Zipf ASCII)."""
    rng = np.random.default_rng(seed)
    w = AnmlWriter("high_frontier")
    _, dna = levenshtein_set(n_patterns=n_lev, input_len=half, writer=w, rng=rng)
    _, asc = dotstar_set(n_patterns=n_dot, input_len=half, writer=w, rng=rng)
    return w.text(), np.concatenate([dna, asc])


def batched_suite(seed=4, n_nfas=16, n_streams=4096, min_states=2000, max_states=200000,
                  len_lo=1 << 10, len_hi=4 << 20, sample_len=1 << 16):
    """Several NFAs and many streams of uneven length.

    NFA i has a size drawn log-uniformly in [min_states, max_states] STEs and
    comes from the literal, Hamming, Levenshtein and dot-star generators in
    turn. Stream lengths are log-uniform in [len_lo, len_hi]; each stream gets
    an NFA uniformly at random and, by seed, either the NFA generator's own
    input law with planted occurrences (a random rotation of a sample), or
    fresh bytes over the NFA's alphabet (ACGT or printable ASCII) drawn
    uniformly or from a Zipf(1.1) law.

    Returns (nfas, data, offsets, lengths, nfa_of): nfas is a list of dicts
    (kind, anml, states_hint), data the concatenated streams.
    """
    rng = np.random.default_rng(seed)
    per_pattern = {"literal": 12, "hamming": 166, "levenshtein": 135, "dotstar": 17}
    kinds = ["literal", "hamming", "levenshtein", "dotstar"]
    nfas, samples = [], []
    for i in range(n_nfas):
        kind = kinds[i % 4]
        target = int(np.exp(rng.uniform(np.log(min_states), np.log(max_states))))
        n = max(1, target // per_pattern[kind])
        sub = int(rng.integers(1 << 30))
        if kind == "literal":
            anml, sample = literal_set(seed=sub, n_patterns=n, input_len=sample_len,
                                       plant_every=1 << 9)
        elif kind == "hamming":
            anml, sample = hamming_set(seed=sub, n_patterns=n, input_len=sample_len,
                                       plant_every=1 << 10)
        elif kind == "levenshtein":
            anml, sample = levenshtein_set(seed=sub, n_patterns=n, input_len=sample_len,
                                           plant_every=1 << 10)
        else:
            anml, sample = dotstar_set(seed=sub, n_patterns=n, input_len=sample_len,
                                       plant_every=1 << 10)
        nfas.append({"kind": kind, "anml": anml, "states_hint": n * per_pattern[kind]})
        samples.append(sample)
    lengths = np.exp(rng.uniform(np.log(len_lo), np.log(len_hi), size=n_streams)).astype(np.int64)
    nfa_of = rng.integers(0, n_nfas, size=n_streams)
    law = rng.integers(0, 3, size=n_streams)  # 0 generator sample, 1 uniform, 2 Zipf
    offsets = np.zeros(n_streams, dtype=np.int64)
    offsets[1:] = np.cumsum(lengths)[:-1]
    data = np.empty(int(lengths.sum()), dtype=np.uint8)
    for s in range(n_streams):
        L, k = int(lengths[s]), int(nfa_of[s])
        out = data[offsets[s]:offsets[s] + L]
        dna = nfas[k]["kind"] in ("hamming", "levenshtein")
        alpha = ACGT if dna else PRINTABLE
        if law[s] == 0:
            smp = samples[k]
            rot = int(rng.integers(len(smp)))
            out[:] = np.resize(np.roll(smp, -rot), L)
        elif law[s] == 1:
            out[:] = alpha[rng.integers(0, len(alpha), size=L)]
        else:
            ranks = np.arange(1, len(alpha) + 1, dtype=np.float64) ** -1.1
            cdf = np.cumsum(ranks / ranks.sum())
            perm = rng.permutation(alpha)
            out[:] = perm[np.minimum(np.searchsorted(cdf, rng.random(L)), len(alpha) - 1)]
    return nfas, data, offsets, lengths, nfa_of


CONFIGS = {
    "literal_set": literal_set,
    "hamming_set": hamming_set,
    "high_frontier": high_frontier,
}
