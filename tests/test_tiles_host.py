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


def _shortcuts(v, nodes, sticky):
    """Layered tile of a layered CC, restated: for a sticky state s that is
    not a start-of-data state, with predecessors P (other than s), the
    successors D of s (not s, not always-active, not sticky) that every state
    of P leads to; the edges P -> D are dropped (s enables D from its first
    match on) and the tile keeps the sticky states and the states that reach
    a report state through the remaining edges (none into always-active or
    sticky states). Returns (kept states, dropped edges, D per sticky state)."""
    ro, co = np.asarray(v.row_offsets), np.asarray(v.col_indices)
    at = np.asarray(v.node_attrs)
    starts = {int(x) for x in np.asarray(v.start_states)}

    def succ(u):
        return [int(x) for x in co[ro[u]:ro[u + 1]]]
    pred = {s: [u for u in nodes if u != s and s in succ(u)] for s in sticky}
    dropped, dsets = set(), {}
    for s in sticky:
        d = set()
        if pred[s] and s not in starts:
            d = {u for u in succ(s) if u != s and not at[u] & 1 and u not in sticky
                 and all(u in succ(x) for x in pred[s])}
        dsets[s] = d
        dropped |= {(x, u) for x in pred[s] for u in succ(x) if u in d}

    def kept_edge(x, u):
        return not at[u] & 1 and u not in sticky and (x, u) not in dropped
    keep = {u for u in nodes if at[u] & 2}
    grew = True
    while grew:
        grew = False
        for x in nodes:
            if x not in keep and any(kept_edge(x, u) and u in keep for u in succ(x)):
                keep.add(x)
                grew = True
    return keep | set(sticky), dropped, dsets


def _sticky_of(v, nodes):
    ro, co = np.asarray(v.row_offsets), np.asarray(v.col_indices)
    at = np.asarray(v.node_attrs)
    bits = np.asarray(v.symbol_sets).reshape(-1, 8)
    return {u for u in nodes if not at[u] & 1 and np.all(bits[u] == 0xFFFFFFFF)
            and u in co[ro[u]:ro[u + 1]]}


def _check_cover(groups, tiles):
    """Every CC lands in one plain tile or one layered pair; plain tiles hold
    all of a CC's states, layered tiles the states _shortcuts keeps."""
    ccs, _ = _total_ccs_and_states(groups)
    main = [t for t in tiles if t["phase"] != 1]  # activation tiles repeat part of a pair
    assert sum(t["num_ccs"] for t in main) == ccs
    vs = groups.views()
    kinds = iter(_classify(vs))
    plain = layered = shortcuts = aas = 0
    for v in vs:
        cb = np.asarray(v.cc_begin)
        at = np.asarray(v.node_attrs)
        for c in range(len(cb) - 1):
            nodes = range(int(cb[c]), int(cb[c + 1]))
            if next(kinds)[0] == "layered":
                kept, _, dsets = _shortcuts(v, nodes, _sticky_of(v, nodes))
                layered += len(kept)
                shortcuts += sum(len(d & kept) for d in dsets.values())
                aas += sum(1 for u in kept if at[u] & 1)
            else:
                plain += len(nodes)
    lay = [t for t in main if t["phase"] == 2]
    assert sum(t["num_states"] for t in main if t["phase"] == 0) == plain
    assert sum(t["num_states"] for t in lay) == layered
    assert sum(t["shortcuts"] for t in lay) == shortcuts
    assert sum(t["naas"] for t in lay) == aas


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
        # lit1 . * lit2: lit1's last state leads to the star and to lit2's first
        # state, a shortcut of the star; lit1's states then leave the layered tile
        assert l["shortcuts"] == l["nact"] and l["naas"] == 0 and a["naas"] > 0
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
    for bad in (lambda: g.tiles(tile_mode="tiles"), lambda: nb.Tables(g, tile_mode="tiles")):
        with pytest.raises(ValueError):  # checked before any device work
            bad()
    assert g.tiles(precompute_depth=-1)[0]["depth"] >= 1


def _expected_lists(views, groups_of_tile, keys):
    """Prefix-table semantics restated on the group graphs: table d maps d
    bytes to the states reached after them, starting from the always-active
    states that accept the first byte and following successor edges whose
    target accepts the next byte (edges into always-active states are not
    followed: those states are injected at every position anyway). Returns
    per key (sorted ids, sorted report ids), ids = state | group << 22."""
    out = []
    for key in keys:
        ids, reps = set(), set()
        for gi in groups_of_tile:
            v = views[gi]
            bits = np.asarray(v.symbol_sets).reshape(-1, 8)
            row, col = np.asarray(v.row_offsets), np.asarray(v.col_indices)
            attrs, aas = np.asarray(v.node_attrs), np.asarray(v.always_active)
            aas_set = set(aas.tolist())
            acc = lambda s, b: (int(bits[s, b >> 5]) >> (b & 31)) & 1
            cur = {int(a) for a in aas if acc(a, int(key[0]))}
            for b in key[1:]:
                cur = {int(u) for s in cur for u in col[row[s]:row[s + 1]]
                       if int(u) not in aas_set and acc(u, int(b))}
            ids |= {s | gi << 22 for s in cur}
            reps |= {s | gi << 22 for s in cur if attrs[s] & 2}
        out.append((sorted(ids), sorted(reps)))
    return out


def _keys(data, rng, depth, n=120, plant_every=1 << 9):
    """Substrings of the input at the planted matches and at random places
    (lists mostly non-empty) and random bytes (mostly dead classes), of every
    length 1..depth."""
    out = []
    planted = list(range(plant_every // 2, len(data) - depth, plant_every))
    for d in range(1, depth + 1):
        ks = [data[p:p + d] for p in planted]
        ks += [data[p:p + d] for p in rng.integers(0, len(data) - d, size=n // 2)]
        ks += [rng.integers(0, 256, size=d, dtype=np.uint8) for _ in range(n // 2)]
        out.append(np.stack(ks).astype(np.uint8))
    return out


@pytest.mark.parametrize("case", ["hamming", "literal", "levenshtein", "global3"])
def test_prefix_tables_match_restated_semantics(case):
    rng = np.random.default_rng(5)
    if case == "hamming":
        anml, data = W.hamming_set(seed=2, n_patterns=3, k=8, input_len=1 << 12, plant_every=1 << 9)
        g, kw = 1, dict(precompute_depth=5, tile_mode="shared")
    elif case == "literal":  # 95 live classes (8 mask words): keys base 95, level 4 hashed
        anml, data = W.literal_set(seed=1, input_len=1 << 12, plant_every=1 << 9)
        g, kw = 1, dict(precompute_depth=4, tile_mode="shared")
    elif case == "levenshtein":
        anml, data = W.levenshtein_set(seed=3, n_patterns=2, k=8, input_len=1 << 12,
                                       plant_every=1 << 9)
        g, kw = 1, dict(precompute_depth=4, tile_mode="shared")
    else:  # one global tile over three groups: ids carry the group bits
        anml, data = W.hamming_set(seed=4, n_patterns=6, k=8, input_len=1 << 12, plant_every=1 << 9)
        g, kw = 3, dict(precompute_depth=4, tile_mode="global")
    groups = _groups(anml, g)
    tiles = groups.tiles(**kw)
    views = groups.views()
    assert len(tiles) == 1 and tiles[0]["num_ccs"] == sum(len(v.cc_begin) - 1 for v in views)
    t = tiles[0]
    if case == "literal":
        assert t["nlive"] == 95 and t["depth"] == 4 and t["dense_levels"] & 8 == 0
    else:
        assert t["dense_levels"] == (1 << t["depth"]) - 1
    nonempty = 0
    for d, keys in enumerate(_keys(np.asarray(data), rng, t["depth"]), start=1):
        got = groups.table_lookup(0, keys, **kw)
        want = _expected_lists(views, range(len(views)), keys)
        for (ids, reps), (wi, wr) in zip(got, want):
            assert sorted(ids.tolist()) == wi and sorted(reps.tolist()) == wr
            nonempty += len(wi) > 0
    assert nonempty > 50


def test_table_lookup_arguments():
    anml, _ = W.literal_set(seed=1, n_patterns=4, input_len=1 << 10, plant_every=1 << 8)
    g = _groups(anml, 1)
    depth = g.tiles(precompute_depth=2)[0]["depth"]
    with pytest.raises(nb.NgapError):
        g.table_lookup(0, np.zeros((1, depth + 1), np.uint8), precompute_depth=2)
    with pytest.raises(nb.NgapError):
        g.table_lookup(5, np.zeros((1, 1), np.uint8), precompute_depth=2)
    with pytest.raises(ValueError):
        g.table_lookup(0, np.zeros(3, np.uint8))
    assert g.table_lookup(0, np.zeros((0, 1), np.uint8), precompute_depth=2) == []


@pytest.mark.parametrize("seed", range(100))
def test_prefix_tables_random_automata(seed):
    """Random automata with fan-out hubs, self-loops and dense CCs (no sticky
    states, so every tile is a plain one): the union over all tiles of one
    key's lists equals the definition restated on the whole group set, for
    every tile mode and every depth the tiles have."""
    from golden.make_golden import degree_stress
    rng = np.random.default_rng(seed)
    anml = degree_stress(seed, int(rng.integers(1, 12)), float(rng.random() * 0.5))
    try:
        groups = _groups(anml, int(rng.integers(1, 4)))
    except nb.NgapError:  # every CC dropped by the degree limiter
        return
    views = groups.views()
    for mode in ("shared", "global", "auto"):
        kw = dict(precompute_depth=int(rng.integers(1, 6)), tile_mode=mode)
        tiles = groups.tiles(**kw)
        assert all(t["phase"] == 0 for t in tiles)
        for d in range(1, min(t["depth"] for t in tiles) + 1):
            keys = rng.integers(97, 104, size=(40, d)).astype(np.uint8)  # 'g' is never accepted
            got = [(set(), set()) for _ in keys]
            for ti in range(len(tiles)):
                for k, (ids, reps) in enumerate(groups.table_lookup(ti, keys, **kw)):
                    got[k][0].update(ids.tolist())
                    got[k][1].update(reps.tolist())
            want = _expected_lists(views, range(len(views)), keys)
            assert [(sorted(a), sorted(b)) for a, b in got] == want, (mode, d)


def _random_star_nfa(rng, nccs):
    """CCs of literal chains with `.*` states (some always active, some
    reporting), extra forward edges and, now and then, a back edge."""
    w = W.AnmlWriter("stars")
    for c in range(nccs):
        n = int(rng.integers(3, 9))
        kinds = ["lit"] * n
        for i in range(1, n - 1):
            if rng.random() < 0.35:
                kinds[i] = "aas" if rng.random() < 0.25 else "star"
        edges = {i: set() for i in range(n)}
        for i in range(n - 1):
            edges[i].add(i + 1)
            if kinds[i] in ("star", "aas"):
                edges[i].add(i)
        for _ in range(int(rng.integers(0, 3))):  # extra forward edges
            a = int(rng.integers(0, n - 1))
            edges[a].add(int(rng.integers(a + 1, n)))
        if rng.random() < 0.2:  # a back edge: a cycle through non-sticky states
            a = int(rng.integers(1, n))
            edges[a].add(int(rng.integers(0, a)))
        for i in range(n):
            nm = f"c{c}v{i}"
            tg = [f"c{c}v{j}" for j in sorted(edges[i])]
            if kinds[i] == "lit":
                w.ste(nm, [int(rng.integers(97, 101))], tg, start="all-input" if i == 0 else None,
                      report=(i == n - 1) or rng.random() < 0.1)
            else:
                w.ste(nm, None, tg, symbol_set="*", start="all-input" if kinds[i] == "aas" else None,
                      report=rng.random() < 0.3)
    return w.text()

def _classify(views):
    """The CC classification restated on the group graphs: bounded when the
    graph without edges into always-active states is acyclic; layered when it
    is not, it has sticky states (not always-active, every byte, a self-loop),
    it becomes acyclic without their self-loops and no sticky state reaches
    another; cyclic otherwise. Per CC: (kind, sticky states)."""
    out = []
    for v in views:
        ro, co = np.asarray(v.row_offsets), np.asarray(v.col_indices)
        at = np.asarray(v.node_attrs)
        bits = np.asarray(v.symbol_sets).reshape(-1, 8)
        cb = np.asarray(v.cc_begin)
        for c in range(len(cb) - 1):
            b, e = int(cb[c]), int(cb[c + 1])
            nodes = range(b, e)
            aas = lambda u: bool(at[u] & 1)
            sticky = {u for u in nodes if not aas(u) and np.all(bits[u] == 0xFFFFFFFF) and u in co[ro[u]:ro[u + 1]]}
            def acyclic(keep):
                indeg = {u: 0 for u in nodes}
                for u in nodes:
                    for x in co[ro[u]:ro[u + 1]]:
                        if keep(u, int(x)): indeg[int(x)] += 1
                q = [u for u in nodes if indeg[u] == 0]
                seen = 0
                while q:
                    u = q.pop()
                    seen += 1
                    for x in co[ro[u]:ro[u + 1]]:
                        if keep(u, int(x)):
                            indeg[int(x)] -= 1
                            if indeg[int(x)] == 0: q.append(int(x))
                return seen == len(nodes)
            if acyclic(lambda u, x: not aas(x)):
                out.append(("bounded", len(sticky)))
                continue
            keep = lambda u, x: not aas(x) and not (u == x and u in sticky)
            ok = bool(sticky) and acyclic(keep)
            if ok:  # no sticky state reachable from another
                for s in sticky:
                    stack, seen = [s], {s}
                    while stack and ok:
                        u = stack.pop()
                        for x in co[ro[u]:ro[u + 1]]:
                            x = int(x)
                            if keep(u, x) and x not in seen:
                                if x in sticky:
                                    ok = False
                                    break
                                seen.add(x)
                                stack.append(x)
            out.append(("layered" if ok else "cyclic", len(sticky)))
    return out



@pytest.mark.parametrize("seed", range(60))
def test_layered_classification_random(seed):
    """Tile counts per kind match the restated classification in every tile
    mode: bounded CCs in plain tiles, cyclic ones in cyclic tiles (with their
    sticky states), layered ones in activation/layered pairs (one activation
    slot per sticky state)."""
    rng = np.random.default_rng(seed)
    anml = _random_star_nfa(rng, int(rng.integers(1, 10)))
    groups = _groups(anml, int(rng.integers(1, 4)))
    cl = _classify(groups.views())
    want = (sum(k == "bounded" for k, _ in cl), sum(k == "cyclic" for k, _ in cl),
            sum(k == "layered" for k, _ in cl), sum(s for k, s in cl if k == "layered"),
            sum(s for k, s in cl if k == "cyclic"))
    for mode in ("auto", "shared", "global"):
        tiles = groups.tiles(precompute_depth=2, tile_mode=mode)
        got = (sum(t["num_ccs"] for t in tiles if t["phase"] == 0 and t["max_path"] >= 0),
               sum(t["num_ccs"] for t in tiles if t["phase"] == 0 and t["max_path"] < 0),
               sum(t["num_ccs"] for t in tiles if t["phase"] == 2),
               sum(t["nact"] for t in tiles if t["phase"] == 1),
               sum(t["nsticky"] for t in tiles if t["phase"] == 0 and t["max_path"] < 0))
        assert got == want, mode


def _layered_lists(views, keys):
    """Prefix-table lists of the layered pairs restated on the group graphs,
    per key over all layered CCs: (non-sticky states of the activation
    tables, sticky states they reach, states of the layered tables, their
    report states). Activation tables start from the always-active states
    among the states with a path to a sticky state (through non-sticky
    states) and stop at sticky states; layered tables start from the
    always-active states the layered tile keeps (_shortcuts), never enter a
    sticky state and never take a dropped edge."""
    out = [[set(), 0, set(), set()] for _ in keys]
    for gi, v in enumerate(views):
        ro, co = np.asarray(v.row_offsets), np.asarray(v.col_indices)
        at = np.asarray(v.node_attrs)
        bits = np.asarray(v.symbol_sets).reshape(-1, 8)
        cb = np.asarray(v.cc_begin)
        kinds = _classify([v])

        def succ(u):
            return [int(x) for x in co[ro[u]:ro[u + 1]] if not at[int(x)] & 1]

        def acc(s, b):
            return (int(bits[s, b >> 5]) >> (b & 31)) & 1

        for c in range(len(cb) - 1):
            if kinds[c][0] != "layered":
                continue
            nodes = range(int(cb[c]), int(cb[c + 1]))
            sticky = {u for u in nodes if not at[u] & 1 and np.all(bits[u] == 0xFFFFFFFF)
                      and u in co[ro[u]:ro[u + 1]]}
            kept, dropped, _ = _shortcuts(v, nodes, sticky)
            pre, grew = set(sticky), True
            while grew:
                grew = False
                for u in nodes:
                    if u not in pre and any(x in pre for x in succ(u)):
                        pre.add(u)
                        grew = True
            for k, key in enumerate(keys):
                cur = {u for u in nodes if at[u] & 1 and u in pre and acc(u, int(key[0]))}
                for b in key[1:]:
                    cur = {x for u in cur if u not in sticky for x in succ(u)
                           if x in pre and acc(x, int(b))}
                out[k][0] |= {u | gi << 22 for u in cur if u not in sticky}
                out[k][1] += len(cur & sticky)
                cur = {u for u in nodes if at[u] & 1 and u in kept and acc(u, int(key[0]))}
                for b in key[1:]:
                    cur = {x for u in cur for x in succ(u) if x not in sticky and x in kept
                           and (u, x) not in dropped and acc(x, int(b))}
                out[k][2] |= {u | gi << 22 for u in cur}
                out[k][3] |= {u | gi << 22 for u in cur if at[u] & 2}
    return out


@pytest.mark.parametrize("seed", range(30))
def test_layered_pair_tables_random(seed):
    """The activation and layered tiles' prefix tables on random star-heavy
    automata equal the restated lists (in activation tiles the sticky states
    are the only reports and their ids are activation slots, so they are
    compared by count)."""
    from collections import Counter
    rng = np.random.default_rng(seed)
    groups = _groups(_random_star_nfa(rng, int(rng.integers(1, 10))), int(rng.integers(1, 4)))
    views = groups.views()
    for mode in ("shared", "global"):
        kw = dict(precompute_depth=3, tile_mode=mode)
        tiles = groups.tiles(**kw)
        act = [i for i, t in enumerate(tiles) if t["phase"] == 1]
        lay = [i for i, t in enumerate(tiles) if t["phase"] == 2]
        if not act:
            continue
        for d in range(1, min(tiles[i]["depth"] for i in act + lay) + 1):
            keys = rng.integers(96, 102, size=(30, d)).astype(np.uint8)  # '`' only stars accept
            got = [[Counter(), 0, set(), set()] for _ in keys]
            for i in act:
                for k, (ids, reps) in enumerate(groups.table_lookup(i, keys, **kw)):
                    got[k][0].update(ids.tolist())
                    got[k][0].subtract(reps.tolist())
                    got[k][1] += len(reps)
            for i in lay:
                for k, (ids, reps) in enumerate(groups.table_lookup(i, keys, **kw)):
                    got[k][2] |= set(ids.tolist())
                    got[k][3] |= set(reps.tolist())
            want = _layered_lists(views, keys)
            for k in range(len(keys)):
                nonsticky = {x for x, n in got[k][0].items() if n > 0}
                assert (nonsticky, got[k][1], got[k][2], got[k][3]) == tuple(want[k]), (mode, d, k)
