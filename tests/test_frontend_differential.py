"""Seeded differential test of the front-end (CPU): random automata and random
symbol sets through the product's ANML loader and preprocessing, through the
oracle's pure-Python restatement (oracle/frontend.py) and through the
reference's own front-end sources compiled into oracle/_ref/ref_frontend
(NFALoader / NFA / nfa_utils / vasim_helper, code/src/commons). Group graphs
must be identical, and an input that the reference rejects must be an error
in both. Skipped where oracle/_ref was not built (it needs the reference
sources at build time)."""
import functools
import os
import random
import subprocess
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import ngap_b200 as nb
from ngap_b200 import workloads as W
from oracle import frontend

from golden.make_golden import degree_stress

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "ref_frontend")
KEYS = ("row_offsets", "col_indices", "symbol_sets", "node_attrs", "always_active",
        "start_states")

pytestmark = pytest.mark.skipif(not os.path.exists(REF), reason="oracle/_ref not built")


def _reference(tmp_path, anml, g):
    """Group graphs of the reference front-end, or None when it rejects the file."""
    src, dump = tmp_path / "case.anml", tmp_path / "case.txt"
    src.write_text(anml)
    if dump.exists():
        dump.unlink()
    r = subprocess.run([REF, str(src), str(g), str(dump)], stdout=subprocess.DEVNULL,
                       stderr=subprocess.DEVNULL, timeout=60)
    if r.returncode != 0 or not dump.exists():
        return None
    return frontend.parse_ref_dump(dump.read_text())


def _product(anml, g):
    try:
        return nb.Groups(nb.Nfa.from_string(anml), group_num=g)
    except nb.NgapError:
        return None


def _python(anml, g):
    """Group graphs of the oracle's restatement, or None when it rejects the file."""
    try:
        nodes, adj = frontend.load_anml(anml)
        return frontend.build_groups(nodes, adj, g)
    except (frontend.ParseError, ET.ParseError, ValueError):
        return None


NOT_CHECKED = object()  # the Python restatement is for small cases only


def _assert_same(prod, ref, py):
    check_py = py is not NOT_CHECKED
    if ref is None or len(ref) == 0:  # rejected, or every CC dropped: an error here
        assert prod is None
        assert not check_py or py is None or len(py) == 0
        return
    assert prod is not None and prod.count == len(ref)
    assert not check_py or (py is not None and len(py) == len(ref))
    for gi in range(prod.count):
        v = prod.view(gi)
        for k in KEYS:
            assert np.array_equal(np.asarray(getattr(v, k)), np.asarray(ref[gi][k])), (gi, k)
            if check_py:
                assert np.array_equal(np.asarray(py[gi][k]), np.asarray(ref[gi][k])), (gi, k, "py")


@pytest.mark.parametrize("seed", range(40))
def test_random_degree_automata(built, tmp_path, seed):
    """Fan-out hubs, self-loops and dense CCs: CC numbering, out-degree
    limiting with clones, dropped CCs and grouping."""
    rng = np.random.default_rng(1000 + seed)
    anml = degree_stress(1000 + seed, int(rng.integers(1, 12)), float(rng.random() * 0.6))
    for g in (1, 2, 5):
        _assert_same(_product(anml, g), _reference(tmp_path, anml, g), _python(anml, g))


TOKENS = ["a", "z", "-", "^", "[", "]", "\\x41", "\\x7f", "\\xff", "\\n", "\\t", "\\d", "\\w",
          "\\s", "\\\\", "\\-", "\\]", "\\[", "\\^", ".", "*", "&amp;", "&lt;", "&#65;", "0", "9",
          "\\r", "\\0"]


@pytest.mark.parametrize("seed", range(12))
def test_random_symbol_sets(built, tmp_path, seed):
    """Random symbol-set strings of the VASim grammar's tokens (classes,
    ranges, negation, escapes, entities): same bitsets, same rejections."""
    rng = random.Random(seed)
    valid = 0
    for _ in range(25):
        w = W.AnmlWriter("sets")
        for i in range(8):
            body = "".join(rng.choice(TOKENS) for _ in range(rng.randint(1, 3)))
            w.ste(f"s{i}", None, [f"s{i + 1}"] if i < 7 else [],
                  start="all-input" if i == 0 else None, report=(i == 7),
                  symbol_set=("[" + body + "]") if rng.random() < 0.7 else body)
        anml = w.text()
        ref = _reference(tmp_path, anml, 1)
        _assert_same(_product(anml, 1), ref, _python(anml, 1))
        valid += ref is not None
    assert valid > 0


@functools.lru_cache(maxsize=1)
def _batched_nfas():
    """The batched suite's NFAs (the suite makes them before any stream)."""
    return [n["anml"] for n in W.batched_suite(seed=4, n_streams=1, len_hi=1 << 10)[0]]


def _full_size_cases():
    """The benchmark's automata at full size, with the group counts it uses."""
    yield "hamming_set", lambda: W.hamming_set(seed=2, input_len=1 << 10)[0], 10
    yield "high_frontier", lambda: W.high_frontier(seed=3, half=1 << 10)[0], 10
    yield "literal_set", lambda: W.literal_set(seed=1, input_len=1 << 10)[0], 1
    for k in range(16):
        yield f"batched_nfa{k}", (lambda k=k: _batched_nfas()[k]), 1


FULL = list(_full_size_cases())


@pytest.mark.parametrize("name,gen,g", FULL, ids=[c[0] for c in FULL])
def test_full_size_automata(built, tmp_path, name, gen, g):
    """Front-end parity at the benchmark's sizes (up to about 200k STEs)."""
    anml = gen()
    ref = _reference(tmp_path, anml, g)
    assert ref is not None and len(ref) > 0
    _assert_same(_product(anml, g), ref, NOT_CHECKED)
