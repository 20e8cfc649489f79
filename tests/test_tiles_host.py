"""Tile planning on the host (ngap_tiles_describe, no GPU): every CC lands in
exactly one plain or layered tile, dot-star CCs become activation/layered
pairs, large acyclic sets become global tiles, and CCs with a sticky state
reachable from another stay cyclic."""
import numpy as np
import pytest

import ngap_b200 as nb
from ngap_b200 import workloads as W


def _groups(anml, g):
    return nb.Groups(nb.Nfa.from_string(anml), group_num=g)


def _total_ccs_and_states(groups):
    vs = groups.views()
    return sum(len(v.cc_begin) - 1 for v in vs), sum(len(v.node_attrs) for v in vs)


def _check_cover(groups, tiles):
    ccs, states = _total_ccs_and_states(groups)
    main = [t for t in tiles if t["phase"] != 1]  # activation tiles repeat part of a pair
    assert sum(t["num_ccs"] for t in main) == ccs
    assert sum(t["num_states"] for t in main) == states


@pytest.mark.parametrize("mode", ["auto", "shared", "global"])
def test_dotstar_pairs(mode):
    anml, _ = W.dotstar_set(seed=9, n_patterns=150, input_len=1 << 12, plant_every=1 << 10)
    g = _groups(anml, 3)
    tiles = g.tiles(precompute_depth=3, tile_mode=mode)
    _check_cover(g, tiles)
    act = {t["pair"]: t for t in tiles if t["phase"] == 1}
    lay = {t["pair"]: t for t in tiles if t["phase"] == 2}
    assert act and set(act) == set(lay)
    for k in act:
        a, l = act[k], lay[k]
        assert a["nact"] == l["nact"] == l["nsticky"] == a["num_ccs"] == l["num_ccs"]
        assert a["nsticky"] == 0 and a["max_path"] > 0 and l["max_path"] > 0
        assert a["num_states"] < l["num_states"]
    # one star per layered CC; the always-active stars make their CCs plain acyclic ones
    non_aas_stars = anml.count('symbol-set="*">')
    assert sum(t["nact"] for t in act.values()) == non_aas_stars
    assert all(t["max_path"] > 0 for t in tiles if t["phase"] == 0)
    if mode == "shared":
        assert not any(t["global"] for t in tiles)


def test_hamming_global_and_cap():
    # 200 CCs over one alphabet: more than two shared tiles' worth, so auto
    # mode makes one global tile; 80 fit in one shared tile per group
    anml, _ = W.hamming_set(seed=31, n_patterns=80, input_len=1 << 12, plant_every=1 << 10)
    small = _groups(anml, 4).tiles(precompute_depth=4)
    assert len(small) == 4 and not any(t["global"] for t in small)
    anml, _ = W.hamming_set(seed=31, n_patterns=200, input_len=1 << 12, plant_every=1 << 10)
    g = _groups(anml, 4)
    auto = g.tiles(precompute_depth=4)
    assert len(auto) == 1 and auto[0]["global"] == 1 and auto[0]["num_ccs"] == 200
    shared = g.tiles(precompute_depth=4, tile_mode="shared")
    assert len(shared) >= 4 and not any(t["global"] for t in shared)
    assert len({t["group"] for t in shared}) == 4
    capped = g.tiles(precompute_depth=4, tile_mode="global", tile_states=10000)
    assert len(capped) > 1 and all(t["global"] and t["num_states"] <= 10000 for t in capped)
    for tiles in (auto, shared, capped):
        _check_cover(g, tiles)
        assert all(t["phase"] == 0 and t["max_path"] == 25 for t in tiles)


def test_two_stars_stay_cyclic():
    w = W.AnmlWriter()
    for p in range(6):  # x .* y .* z: the second star is reachable from the first
        w.ste(f"x{p}", [97 + p], [f"s{p}", f"y{p}"], start="all-input")
        w.ste(f"s{p}", None, [f"s{p}", f"y{p}"], symbol_set="*")
        w.ste(f"y{p}", [98 + p], [f"t{p}", f"z{p}"])
        w.ste(f"t{p}", None, [f"t{p}", f"z{p}"], symbol_set="*")
        w.ste(f"z{p}", [99 + p], [], report=True)
    g = _groups(w.text(), 2)
    tiles = g.tiles(precompute_depth=2)
    _check_cover(g, tiles)
    assert all(t["phase"] == 0 for t in tiles)
    assert all(t["max_path"] == -1 and t["nsticky"] == 2 * t["num_ccs"] for t in tiles)


def test_bad_options_are_errors():
    anml, _ = W.literal_set(seed=1, n_patterns=4, input_len=1 << 10, plant_every=1 << 8)
    g = _groups(anml, 1)
    with pytest.raises(nb.NgapError):
        g.tiles(precompute_depth=13)
    assert g.tiles(precompute_depth=-1)[0]["depth"] >= 1
