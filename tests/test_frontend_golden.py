"""Front-end parity (CPU): the product's ANML loader and preprocessing, and the
oracle's Python restatement, against group graphs dumped by the reference's
own front-end sources (oracle/_ref/ref_frontend; fixtures made by
tests/golden/make_golden.py)."""
import glob
import os

import numpy as np
import pytest

import ngap_b200 as nb
from oracle import frontend

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(glob.glob(os.path.join(GOLD, "cases", "*.ref.txt")))


def _case(path):
    base = os.path.basename(path)
    name, g = base.split(".")[0], int(base.split(".")[1][1:])
    anml = os.path.join(GOLD, "cases", name + ".anml")
    return name, g, anml


def _same(a, b):
    for k in ("row_offsets", "col_indices", "symbol_sets", "node_attrs", "always_active",
              "start_states"):
        x = a[k] if isinstance(a, dict) else getattr(a, k)
        y = b[k] if isinstance(b, dict) else getattr(b, k)
        assert np.array_equal(np.asarray(x), np.asarray(y)), k


def test_fixtures_present():
    assert len(CASES) >= 14


@pytest.mark.parametrize("dump", CASES, ids=[os.path.basename(c) for c in CASES])
def test_product_frontend_matches_reference(built, dump):
    name, g, anml = _case(dump)
    ref = frontend.parse_ref_dump(open(dump).read())
    nfa = nb.Nfa.from_file(anml)
    if len(ref) == 0:  # the reference drops every CC: the product reports an error
        with pytest.raises(nb.NgapError):
            nb.Groups(nfa, group_num=g)
        return
    groups = nb.Groups(nfa, group_num=g)
    assert groups.count == len(ref)
    for gi in range(groups.count):
        _same(groups.view(gi), ref[gi])


@pytest.mark.parametrize("dump", CASES, ids=[os.path.basename(c) for c in CASES])
def test_python_frontend_matches_reference(dump):
    name, g, anml = _case(dump)
    ref = frontend.parse_ref_dump(open(dump).read())
    nodes, adj = frontend.load_anml(open(anml, encoding="utf-8").read())
    mine = frontend.build_groups(nodes, adj, g)
    assert len(mine) == len(ref)
    for a, b in zip(mine, ref):
        _same(a, b)


def test_degree_limiter_clones_and_drops(built):
    """Clones keep the '_dup_' naming of the reference and failing CCs are dropped."""
    ref = frontend.parse_ref_dump(open(os.path.join(GOLD, "cases", "degree1.g1.ref.txt")).read())
    names = ref[0]["names"]
    assert any("_dup_" in n for n in names)
    nfa = nb.Nfa.from_file(os.path.join(GOLD, "cases", "degree1.anml"))
    groups = nb.Groups(nfa, group_num=1)
    total, failed, _ = groups.cc_stats()
    assert (total, failed) == (8, 2)
    assert groups.view(0).num_states == len(names)


BAD = {
    "malformed_hex": ('<anml><automata-network><state-transition-element id="a" '
                      'symbol-set="[\\x4]"/></automata-network></anml>'),
    "curly": ('<anml><automata-network><state-transition-element id="a" symbol-set="{ab}"/>'
              '</automata-network></anml>'),
    "or_element": '<anml><automata-network><or id="x"/></automata-network></anml>',
    "unknown_target": ('<anml><automata-network><state-transition-element id="a" symbol-set="a">'
                       '<activate-on-match element="b"/></state-transition-element>'
                       '</automata-network></anml>'),
    "duplicate_id": ('<anml><automata-network><state-transition-element id="a" symbol-set="a"/>'
                     '<state-transition-element id="a" symbol-set="b"/></automata-network></anml>'),
    "no_network": "<anml></anml>",
    "bad_xml": "<anml><automata-network>",
}


@pytest.mark.parametrize("case", sorted(BAD))
def test_parse_errors(built, case):
    with pytest.raises(nb.NgapError) as ei:
        nb.Nfa.from_string(BAD[case])
    assert ei.value.status == 2  # NGAP_E_PARSE


def test_file_errors(built, tmp_path):
    with pytest.raises(nb.NgapError) as ei:
        nb.Nfa.from_file(str(tmp_path / "x.mnrl"))
    assert ei.value.status == 3
    with pytest.raises(nb.NgapError) as ei:
        nb.Nfa.from_file(str(tmp_path / "missing.anml"))
    assert ei.value.status == 10


def test_automata_network_at_root_and_description(built):
    xml = ('<automata-network id="n"><description>x</description>'
           '<state-transition-element id="a" symbol-set="[ab]" start="all-input">'
           '<report-on-match reportcode="7"/></state-transition-element></automata-network>')
    g = nb.Groups(nb.Nfa.from_string(xml), group_num=4)
    v = g.view(0)
    assert g.count == 1 and v.num_states == 1 and list(v.node_attrs) == [3]
    assert v.symbol_sets[0, 3] == (1 << 1) | (1 << 2)  # bytes 'a' (97) and 'b' (98)


def test_group_num_float_bound(built):
    """group_nfas_by_num's float bound arithmetic: 7 CCs into 3 groups."""
    w = ['<anml><automata-network>']
    for i in range(7):
        w.append(f'<state-transition-element id="s{i}" symbol-set="a" start="all-input"/>')
    w.append('</automata-network></anml>')
    g = nb.Groups(nb.Nfa.from_string("".join(w)), group_num=3)
    sizes = [g.view(i).num_states for i in range(g.count)]
    nodes, adj = frontend.load_anml("".join(w))
    py = [len(x["node_attrs"]) for x in frontend.build_groups(nodes, adj, 3)]
    assert sizes == py and sum(sizes) == 7
