"""Test infrastructure (oracle), not product code.

Pure-Python restatement of the reference front-end, for small cases:
  * ANML loading          code/src/commons/NFALoader.cpp:37-171 (pugixml parse:
                          entities expanded, tab/CR/LF in attributes -> space)
  * symbol sets           code/src/commons/vasim_helper.cpp:40-480
  * CC marking / split    code/src/commons/NFA.cpp:188-227, nfa_utils.cpp:54-91
  * out-degree limiting   code/src/commons/nfa_utils.cpp:507-680
  * grouping / merging    code/src/commons/nfa_utils.cpp:382-424, 466-486
  * group graph read-out  code/src/commons/graph.cu:169-206, graph.h:184-219
Its output is checked id-for-id against dumps of the reference's own
front-end (oracle/_ref/ref_frontend, fixtures in tests/golden/).
"""
import xml.etree.ElementTree as ET

import numpy as np

START_NONE, START_OF_DATA, START_ALL_INPUT = 0, 1, 2


class ParseError(ValueError):
    pass


def _strtoul16(h):
    """C strtoul(h, NULL, 16) as an unsigned 64-bit value."""
    i = 0
    while i < len(h) and h[i] in " \t\n\v\f\r":
        i += 1
    neg = False
    if i < len(h) and h[i] in "+-":
        neg = h[i] == "-"
        i += 1
    if h[i:i + 2].lower() == "0x" and i + 2 < len(h) and h[i + 2] in "0123456789abcdefABCDEF":
        i += 2
    v = 0
    while i < len(h) and h[i] in "0123456789abcdefABCDEF":
        v = v * 16 + int(h[i], 16)
        i += 1
    return (-v) & 0xFFFFFFFFFFFFFFFF if neg else v


def symbol_set(text):
    """VASim parseSymbolSet over the UTF-8 bytes of `text`; returns a bool[256]."""
    col = np.zeros(256, dtype=bool)
    if text == "*":
        col[:] = True
        return col
    if text == ".":
        col[:] = True
        col[ord("\n")] = False
        return col
    if len(text) > 0 and text[0] == "{" and text[-1] == "}":
        raise ParseError("curly braces not implemented: " + text)
    s = text.encode("utf-8")
    OPEN = 256
    st = {"escaped": False, "inverting": False, "range_set": False, "brackets": 0,
          "last": 0, "rstart": 0}

    def setc(ch):
        col[ch] = True
        if st["range_set"]:
            a, b = st["rstart"], ch
            if a <= b:
                col[a:b + 1] = True
            st["range_set"] = False
        st["last"] = ch

    escapes = {ord("n"): 10, ord("r"): 13, ord("t"): 9, ord("a"): 7, ord("b"): 8, ord("f"): 12,
               ord("v"): 11, ord("'"): ord("'"), ord('"'): ord('"')}
    i = 0
    while i < len(s):
        c = s[i]
        esc = st["escaped"]
        if c in (ord("["), ord("]")):
            if esc:
                setc(c)
                st["escaped"] = False
            elif c == ord("["):
                st["last"] = OPEN
                st["brackets"] += 1
            else:
                st["brackets"] -= 1
        elif c in (ord("{"), ord("}")):
            setc(c)  # the pending escape, if any, is kept
        elif c == ord("\\"):
            if esc:
                setc(c)
                st["escaped"] = False
            else:
                st["escaped"] = True
        elif c in escapes:
            if esc:
                setc(escapes[c])
                st["escaped"] = False
            else:
                setc(c)
        elif c == ord("-"):
            if esc or st["last"] == OPEN:
                setc(ord("-"))
                st["escaped"] = False
            else:
                st["range_set"] = True
                st["rstart"] = st["last"]
        elif c == ord("s") and esc:
            for x in (10, 9, 13, 11, 12, 32):
                col[x] = True
            st["escaped"] = False
        elif c == ord("d") and esc:
            col[48:58] = True
            st["escaped"] = False
        elif c == ord("w") and esc:
            col[ord("_")] = True
            col[48:58] = True
            col[65:91] = True
            col[97:123] = True
            st["escaped"] = False
        elif c == ord("^"):
            if esc:
                setc(c)
                st["escaped"] = False
            else:
                st["inverting"] = True
        elif c == ord("x") and esc:
            i += 2
            setc(_strtoul16(bytes(s[i - 1:i + 1]).decode("latin-1")) & 0xFF)
            st["escaped"] = False
        else:
            st["escaped"] = False
            setc(c)
        i += 1
    if st["inverting"]:
        col = ~col
    if st["brackets"] != 0:
        raise ParseError("malformed brackets: " + text)
    return col


def load_anml(xml_text):
    """Returns (nodes, adj): nodes = list of dicts in file order, adj = ordered
    deduplicated target lists by node index."""
    root = ET.fromstring(xml_text)
    net = None
    if root.tag == "anml":
        net = root.find("automata-network")
    elif root.tag == "automata-network":
        net = root
    if net is None:
        raise ParseError("no automata-network")
    nodes, targets, ids = [], [], {}
    for el in net:
        if el.tag == "state-transition-element":
            sid = el.get("id", "")
            if sid in ids:
                raise ParseError("duplicate id " + sid)
            start = {"start-of-data": START_OF_DATA, "all-input": START_ALL_INPUT}.get(
                el.get("start", ""), START_NONE)
            nd = {"id": sid, "bits": symbol_set(el.get("symbol-set", "")), "start": start,
                  "report": False}
            tg = []
            for ch in el:
                if ch.tag == "activate-on-match":
                    tg.append(ch.get("element", ""))
                elif ch.tag == "report-on-match":
                    nd["report"] = True
            ids[sid] = len(nodes)
            nodes.append(nd)
            targets.append(tg)
        elif el.tag == "description":
            continue
        else:
            raise ParseError("unsupported element " + el.tag)
    adj = []
    for tg in targets:
        lst = []
        for t in tg:
            if t not in ids:
                raise ParseError("unknown target " + t)
            if ids[t] not in lst:
                lst.append(ids[t])
        adj.append(lst)
    return nodes, adj


class _Cc:
    def __init__(self):
        self.attr, self.adj, self.frm, self.by_int = [], [], [], []

    def handle(self, a):
        self.attr.append(a)
        self.adj.append([])
        self.frm.append([])
        return len(self.attr) - 1

    def add_node(self, a):
        h = self.handle(a)
        self.by_int.append(h)
        return h

    def add_edge(self, f, t):
        if t not in self.adj[f]:
            self.adj[f].append(t)
        if f not in self.frm[t]:
            self.frm[t].append(f)


def _limit(cc, limit=4):
    orig = len(cc.by_int)
    it = 0
    while True:
        it += 1
        pick, pick_i, best = None, None, None
        for i in range(len(cc.by_int) - 1, -1, -1):
            h = cc.by_int[i]
            d = len(cc.adj[h])
            if d > limit and (best is None or d < best):
                best, pick, pick_i = d, h, i
        if pick is None:
            return True
        from_nodes, to_nodes = list(cc.frm[pick]), list(cc.adj[pick])
        for fn in list(cc.frm[pick]):
            cc.adj[fn].remove(pick)
        for t in list(cc.adj[pick]):
            cc.frm[t].remove(pick)
        cc.adj[pick], cc.frm[pick] = [], []
        self_loop = pick in to_nodes
        if self_loop:
            to_nodes.remove(pick)
            from_nodes.remove(pick)
        p, t = 0, 0
        while t < len(to_nodes):
            if p == 0:
                h = cc.handle(cc.attr[pick])
                cc.by_int[pick_i] = h
            else:
                h = cc.add_node(cc.attr[pick])
            L = limit
            if self_loop:
                L = limit - 1
                cc.add_edge(h, h)
            for kk in range(L):
                if t + kk < len(to_nodes):
                    cc.add_edge(h, to_nodes[t + kk])
            for f in from_nodes:
                cc.add_edge(f, h)
            p += 1
            t += L
        if it >= orig * 2:
            return False


def build_groups(nodes, adj, group_num=10, max_nfa_size=-1):
    """Returns a list of group dicts (row_offsets, col_indices, symbol_sets,
    node_attrs, always_active, start_states, cc_begin, orig_node)."""
    V = len(nodes)
    und = [[] for _ in range(V)]
    for i in range(V):
        for t in adj[i]:
            und[i].append(t)
            und[t].append(i)
    cc_of = [-1] * V
    ncc = 0
    for i in range(V):
        if cc_of[i] >= 0:
            continue
        cc_of[i] = ncc
        stack = [i]
        while stack:
            x = stack.pop()
            for y in und[x]:
                if cc_of[y] < 0:
                    cc_of[y] = ncc
                    stack.append(y)
        ncc += 1
    ccs = [_Cc() for _ in range(ncc)]
    local = [ccs[cc_of[i]].add_node(i) for i in range(V)]
    for i in range(V):
        for t in adj[i]:
            ccs[cc_of[i]].add_edge(local[i], local[t])
    kept = [c for c in range(ncc) if _limit(ccs[c])]
    if max_nfa_size != -1:
        kept = [c for c in kept if len(ccs[c].by_int) <= max_nfa_size]
    n = len(kept)
    gnum = min(group_num, n)
    per = np.float32(n) / np.float32(gnum)
    bound = per
    members, cur = [], []
    for i in range(n):
        if cur and np.float32(i + 1) > bound and len(members) + 1 < gnum:
            bound = np.float32(bound + per)
            members.append(cur)
            cur = []
        cur.append(kept[i])
    if cur:
        members.append(cur)
    groups = []
    for mem in members:
        bits, attrs, aas, starts, cc_begin, orig, edges = [], [], [], [], [], [], []
        base = 0
        for c in mem:
            cc = ccs[c]
            cc_begin.append(base)
            gid = {h: base + i for i, h in enumerate(cc.by_int)}
            for i, h in enumerate(cc.by_int):
                s = base + i
                nd = nodes[cc.attr[h]]
                orig.append(cc.attr[h])
                words = np.packbits(nd["bits"].reshape(8, 32)[:, ::-1], axis=1).view(">u4")
                bits.append(words.reshape(8).astype(np.uint32))
                a = 0
                if nd["start"] == START_ALL_INPUT:
                    a |= 1
                    aas.append(s)
                if nd["start"] == START_OF_DATA:
                    starts.append(s)
                if nd["report"]:
                    a |= 2
                attrs.append(a)
                for t in cc.adj[h]:
                    edges.append((s, gid[t]))
            base += len(cc.by_int)
        cc_begin.append(base)
        edges.sort()
        row = np.zeros(base + 1, dtype=np.int32)
        for s, _ in edges:
            row[s + 1] += 1
        groups.append({
            "row_offsets": np.cumsum(row).astype(np.int32),
            "col_indices": np.array([t for _, t in edges], dtype=np.int32),
            "symbol_sets": np.array(bits, dtype=np.uint32).reshape(base, 8),
            "node_attrs": np.array(attrs, dtype=np.uint8),
            "always_active": np.array(aas, dtype=np.int32),
            "start_states": np.array(starts, dtype=np.int32),
            "cc_begin": np.array(cc_begin, dtype=np.int32),
            "orig_node": np.array(orig, dtype=np.int32),
        })
    return groups


def parse_ref_dump(text):
    """Reads the text dump written by oracle/_ref/ref_frontend."""
    lines = text.splitlines()
    assert lines[0].startswith("NGAPREF")
    groups, g = [], None
    for ln in lines[1:]:
        f = ln.split()
        if not f:
            continue
        if f[0] == "groups":
            continue
        if f[0] == "group":
            g = {"V": int(f[3]), "bits": [], "attrs": [], "names": [], "edges": []}
            groups.append(g)
        elif f[0] == "n":
            g["bits"].append([int(x, 16) for x in f[2:10]])
            g["attrs"].append(int(f[10]))
            g["names"].append(f[11] if len(f) > 11 else "")
        elif f[0] == "e":
            g["edges"].append((int(f[1]), int(f[2])))
        elif f[0] == "aas":
            g["aas"] = [int(x) for x in f[1:]]
        elif f[0] == "start":
            g["start"] = [int(x) for x in f[1:]]
    out = []
    for g in groups:
        V = g["V"]
        row = np.zeros(V + 1, dtype=np.int32)
        for s, _ in g["edges"]:
            row[s + 1] += 1
        out.append({
            "row_offsets": np.cumsum(row).astype(np.int32),
            "col_indices": np.array([t for _, t in g["edges"]], dtype=np.int32),
            "symbol_sets": np.array(g["bits"], dtype=np.uint32).reshape(V, 8),
            "node_attrs": np.array(g["attrs"], dtype=np.uint8),
            "always_active": np.array(g.get("aas", []), dtype=np.int32),
            "start_states": np.array(g.get("start", []), dtype=np.int32),
            "names": g["names"],
        })
    return out
