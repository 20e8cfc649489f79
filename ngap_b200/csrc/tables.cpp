// Tiles, byte classes, shared-memory images and prefix-memoization tables.
//
// A tile is a set of whole CCs: of one group for shared-memory tiles, of any
// groups for global tiles. CCs never share states or edges, so the way CCs
// are packed into tiles changes no report: every state keeps its report id
// (group-local sid | group << 22, TileHost::sid). Two facts about the graph
// are used:
//   * an edge into an always-active state is redundant, because the reference
//     puts every always-active state in every frontier (code/src/ngap/ngap.cu:
//     2252-2256); such edges are dropped here;
//   * after that, a CC without cycles has a longest path of L states, so a
//     report at position p depends only on input[p-L+1 .. p]. Tiles made of
//     such CCs can be matched in independent chunks with L-1 positions of
//     warm-up, reports in the warm-up being left to the previous chunk.
//
// Byte classes: two bytes are equivalent for a tile when every state of the
// tile accepts both or neither. With at most 32 (64) classes a state's symbol
// class shrinks from 256 bits to one (two) words and the input is translated
// to class ids once per window.
//
// Prefix tables follow ngap::getPrecomputeResultsForKGroupsInCsr and
// recursivePrecomputeForK (code/src/ngap/ngap.cu:2358-2513): table 1 maps a
// symbol to the always-active states accepting it; table d maps d symbols to
// the successors of table d-1's states accepting the last symbol; each table
// also lists the report states among its states. Here the symbols are byte
// classes (the reference keys by bytes; the lists are the same for every byte
// of a class), and lists are deduplicated (the reference keeps duplicates; the
// set of activations is the same).
#include "tables.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cstring>
#include <map>
#include <numeric>
#include <thread>

namespace ngap {

namespace {

struct CcInfo {
  int32_t group;        // group index (report ids carry it in bits 22 and up)
  int32_t begin, end;   // group-local state range
  bool bounded;         // acyclic once edges into always-active states are dropped
  bool layered;         // cyclic only through sticky self-loops (see layer_flags)
  int32_t max_path;
};

// Sticky states of a CC: not always-active, a self-loop, every byte accepted.
// Such a state, once matched, matches at every later position of the segment.
void sticky_flags(const GroupGraph& g, int32_t b, int32_t e, std::vector<char>& sticky) {
  sticky.assign(e - b, 0);
  for (int32_t v = b; v < e; v++) {
    if (g.attrs[v] & 1) continue;
    bool all = true;
    for (int w = 0; w < 8; w++) all = all && g.bits[(size_t)v * 8 + w] == 0xffffffffu;
    if (!all) continue;
    for (int32_t k = g.row_offsets[v]; k < g.row_offsets[v + 1]; k++)
      if (g.cols[k] == v) sticky[v - b] = 1;
  }
}

// A CC is layered when it has sticky states, the graph without edges into
// always-active states and without sticky self-loops is acyclic, and no sticky
// state is reachable from another one. Then the first match of each sticky
// state depends only on an acyclic part (its "pre" states: those with a path
// to a sticky state through non-sticky states), and once the first matches
// are known the rest is acyclic with the sticky states as sources. Returns
// false otherwise; on success pre[] marks the pre states (stickies included),
// and lp1 / lp2 are the longest paths (in states) of the activation part and
// of the part with the sticky states as sources.
bool layer_flags(const GroupGraph& g, int32_t b, int32_t e, std::vector<char>& sticky,
                 std::vector<char>& pre, int32_t& lp1, int32_t& lp2) {
  const int32_t n = e - b;
  sticky_flags(g, b, e, sticky);
  bool any = false;
  for (char x : sticky) any = any || x;
  if (!any) return false;
  auto edge_ok = [&](int32_t v, int32_t u) {  // kept edge v -> u (group ids)
    return !(g.attrs[u] & 1) && !(u == v && sticky[v - b]);
  };
  std::vector<int32_t> indeg(n, 0), order;
  order.reserve(n);
  for (int32_t v = b; v < e; v++)
    for (int32_t k = g.row_offsets[v]; k < g.row_offsets[v + 1]; k++)
      if (edge_ok(v, g.cols[k])) indeg[g.cols[k] - b]++;
  for (int32_t i = 0; i < n; i++)
    if (indeg[i] == 0) order.push_back(i);
  for (size_t h = 0; h < order.size(); h++) {
    const int32_t v = order[h] + b;
    for (int32_t k = g.row_offsets[v]; k < g.row_offsets[v + 1]; k++) {
      const int32_t u = g.cols[k];
      if (edge_ok(v, u) && --indeg[u - b] == 0) order.push_back(u - b);
    }
  }
  if ((int32_t)order.size() != n) return false;
  // no sticky state reachable from a sticky state
  std::vector<char> from(n, 0);
  for (int32_t i : order) {
    const int32_t v = i + b;
    for (int32_t k = g.row_offsets[v]; k < g.row_offsets[v + 1]; k++) {
      const int32_t u = g.cols[k];
      if (edge_ok(v, u) && (sticky[i] || from[i])) from[u - b] = 1;
    }
  }
  for (int32_t i = 0; i < n; i++)
    if (sticky[i] && from[i]) return false;
  // pre states, in reverse topological order
  pre.assign(n, 0);
  for (int32_t h = n - 1; h >= 0; h--) {
    const int32_t i = order[h], v = i + b;
    if (sticky[i]) {
      pre[i] = 1;
      continue;
    }
    for (int32_t k = g.row_offsets[v]; k < g.row_offsets[v + 1]; k++) {
      const int32_t u = g.cols[k];
      if (edge_ok(v, u) && pre[u - b]) pre[i] = 1;
    }
  }
  // longest paths: lp1 over pre states (edges out of stickies dropped), lp2
  // over all states with edges into stickies dropped
  std::vector<int32_t> d1(n, 1), d2(n, 1);
  lp1 = lp2 = 0;
  for (int32_t i : order) {
    const int32_t v = i + b;
    lp2 = std::max(lp2, d2[i]);
    if (pre[i]) lp1 = std::max(lp1, d1[i]);
    for (int32_t k = g.row_offsets[v]; k < g.row_offsets[v + 1]; k++) {
      const int32_t u = g.cols[k];
      if (!edge_ok(v, u)) continue;
      if (!sticky[u - b]) d2[u - b] = std::max(d2[u - b], d2[i] + 1);
      if (pre[i] && pre[u - b] && !sticky[i]) d1[u - b] = std::max(d1[u - b], d1[i] + 1);
    }
  }
  return true;
}

// Shortcuts through the sticky states of a layered CC, for its layered tile.
// For a sticky state s that is not a start-of-data state, let P be the
// states with an edge into s (other than its self-loop) and D the successors
// u of s (not s, not always-active, not sticky) that every state of P also
// leads to. When v in P matches at q, s matches at q + 1 (it accepts every
// byte), so s's first match f is at most q + 1: v's edge enables u at q + 1,
// which s enables as well when q + 1 > f; and at q + 1 = f, s was enabled by
// some state of P (s is no start state), whose edge enables u at f. So the
// edges P -> D can go if s enables D from its first match on (inclusive)
// instead of after it. States that then reach no report state through the
// remaining edges (edges into always-active or sticky states do not count)
// are left out of the layered tile; sticky states stay (activation slots).
// drop[k - row_offsets[b]] marks dropped edges, dset[s - b] lists D of s,
// keep[v - b] the states of the layered tile.
void layered_shortcuts(const GroupGraph& g, int32_t b, int32_t e, const std::vector<char>& sticky,
                       std::vector<char>& drop, std::vector<std::vector<int32_t>>& dset,
                       std::vector<char>& keep) {
  const int32_t n = e - b, e0 = g.row_offsets[b];
  drop.assign(g.row_offsets[e] - e0, 0);
  dset.assign(n, {});
  std::vector<std::vector<int32_t>> pred(n);
  for (int32_t v = b; v < e; v++)
    for (int32_t k = g.row_offsets[v]; k < g.row_offsets[v + 1]; k++) {
      const int32_t u = g.cols[k];
      if (u != v && sticky[u - b]) pred[u - b].push_back(v);
    }
  auto has_edge = [&](int32_t v, int32_t u) {
    return std::binary_search(g.cols.begin() + g.row_offsets[v],
                              g.cols.begin() + g.row_offsets[v + 1], u);  // rows are sorted
  };
  for (int32_t s = b; s < e; s++) {
    if (!sticky[s - b] || pred[s - b].empty() ||
        std::binary_search(g.starts.begin(), g.starts.end(), s))
      continue;
    std::vector<int32_t>& d = dset[s - b];
    for (int32_t k = g.row_offsets[s]; k < g.row_offsets[s + 1]; k++) {
      const int32_t u = g.cols[k];
      if (u == s || (g.attrs[u] & 1) || sticky[u - b]) continue;
      bool all = true;
      for (int32_t v : pred[s - b]) all = all && has_edge(v, u);
      if (all) d.push_back(u);
    }
    for (int32_t v : pred[s - b])
      for (int32_t k = g.row_offsets[v]; k < g.row_offsets[v + 1]; k++)
        if (std::binary_search(d.begin(), d.end(), g.cols[k])) drop[k - e0] = 1;
  }
  // states that reach a report state through the kept edges (reverse search)
  std::vector<std::vector<int32_t>> rev(n);
  for (int32_t v = b; v < e; v++)
    for (int32_t k = g.row_offsets[v]; k < g.row_offsets[v + 1]; k++) {
      const int32_t u = g.cols[k];
      if ((g.attrs[u] & 1) || sticky[u - b] || drop[k - e0]) continue;
      rev[u - b].push_back(v);
    }
  keep.assign(n, 0);
  std::vector<int32_t> todo;
  for (int32_t v = b; v < e; v++)
    if (g.attrs[v] & 2) {
      keep[v - b] = 1;
      todo.push_back(v);
    }
  while (!todo.empty()) {
    const int32_t u = todo.back();
    todo.pop_back();
    for (int32_t v : rev[u - b])
      if (!keep[v - b]) {
        keep[v - b] = 1;
        todo.push_back(v);
      }
  }
  for (int32_t i = 0; i < n; i++)
    if (sticky[i]) keep[i] = 1;
}

// Longest path (in states) of a CC whose edges into always-active states are
// removed; -1 if a cycle remains.
int32_t cc_longest_path(const GroupGraph& g, int32_t b, int32_t e) {
  int32_t n = e - b;
  std::vector<int32_t> indeg(n, 0), lp(n, 1), order;
  order.reserve(n);
  for (int32_t v = b; v < e; v++)
    for (int32_t k = g.row_offsets[v]; k < g.row_offsets[v + 1]; k++) {
      int32_t u = g.cols[k];
      if (g.attrs[u] & 1) continue;
      indeg[u - b]++;
    }
  for (int32_t i = 0; i < n; i++)
    if (indeg[i] == 0) order.push_back(i);
  for (size_t h = 0; h < order.size(); h++) {
    int32_t v = order[h] + b;
    for (int32_t k = g.row_offsets[v]; k < g.row_offsets[v + 1]; k++) {
      int32_t u = g.cols[k];
      if (g.attrs[u] & 1) continue;
      lp[u - b] = std::max(lp[u - b], lp[v - b] + 1);
      if (--indeg[u - b] == 0) order.push_back(u - b);
    }
  }
  if ((int32_t)order.size() != n) return -1;
  int32_t m = 0;
  for (int32_t x : lp) m = std::max(m, x);
  return m;
}

// Partition of the 256 bytes into classes, refined state by state; class ids
// are numbered in order of their smallest byte.
struct Partition {
  uint16_t id[256];
  int n = 1;
  Partition() { memset(id, 0, sizeof(id)); }
  void refine(const uint32_t* bits) {
    int16_t map[512];
    memset(map, -1, sizeof(map));
    uint16_t nid[256];
    int n2 = 0;
    for (int b = 0; b < 256; b++) {
      int k = id[b] * 2 + (int)((bits[b >> 5] >> (b & 31)) & 1u);
      if (map[k] < 0) map[k] = (int16_t)n2++;
      nid[b] = (uint16_t)map[k];
    }
    memcpy(id, nid, sizeof(id));
    n = n2;
  }
};

int class_words(int ncls) { return (ncls + 31) / 32; }  // mask words per state: 1..8

inline bool accepts_cls(const TileHost& t, uint32_t v, int c) {
  return (t.cmask[(size_t)v * t.cw + (c >> 5)] >> (c & 31)) & 1u;
}

inline bool is_report(const TileHost& t, uint32_t v) { return (t.rep[v >> 5] >> (v & 31)) & 1u; }

// One level of prefix lists: the non-empty keys in ascending order with their
// state lists (sorted, deduplicated), flat.
struct Level {
  std::vector<uint32_t> keys;
  std::vector<uint32_t> off{0};  // keys.size() + 1
  std::vector<uint32_t> list;
};

// Lays out one table, dense (offsets indexed by key) or hashed, whichever
// takes fewer bytes; false when a list is too long for the hashed slot format.
bool finish_table(PrefixTableHost& pt, uint64_t space, const Level& lv, const TileHost& t,
                  int cutoff_opt) {
  pt = PrefixTableHost();
  const size_t nz = lv.keys.size();
  bool any_rep = false;
  for (uint32_t v : lv.list) any_rep = any_rep || is_report(t, v);
  uint64_t cap = 16;
  while (cap < 2 * (uint64_t)nz) cap <<= 1;
  const uint64_t dense_bytes = (space + 1) * 4 * (any_rep ? 2 : 1);
  pt.dense = space <= kDenseKeys || (space <= kMaxDenseKeys && dense_bytes <= cap * 16);
  pt.entries = (int64_t)lv.list.size();
  for (size_t i = 0; i < nz; i++)
    pt.max_len = std::max<int32_t>(pt.max_len, (int32_t)(lv.off[i + 1] - lv.off[i]));
  if (pt.dense && !any_rep && pt.max_len < 64 && lv.list.size() < (1u << 25)) {
    // one word per key: the lone state itself, or where a longer list starts
    pt.inline1 = true;
    pt.voff.assign(space, kHashEmpty);
    for (size_t i = 0; i < nz; i++) {
      const uint32_t len = lv.off[i + 1] - lv.off[i];
      if (len == 1) {
        pt.voff[lv.keys[i]] = lv.list[lv.off[i]];
      } else {
        pt.voff[lv.keys[i]] = 0x80000000u | ((uint32_t)pt.vlist.size() << 6) | len;
        pt.vlist.insert(pt.vlist.end(), lv.list.begin() + lv.off[i], lv.list.begin() + lv.off[i + 1]);
      }
    }
    pt.cutoff = nz > 0 ? (int32_t)(lv.list.size() / nz) : 0;
    if (cutoff_opt >= 0) pt.cutoff = cutoff_opt;
    return true;
  }
  pt.vlist = lv.list;
  if (pt.dense) {
    pt.voff.assign(space + 1, 0);
    if (any_rep) pt.roff.assign(space + 1, 0);
    for (size_t i = 0; i < nz; i++) {
      pt.voff[lv.keys[i] + 1] = lv.off[i + 1] - lv.off[i];
      if (any_rep) {
        uint32_t r = 0;
        for (uint32_t j = lv.off[i]; j < lv.off[i + 1]; j++) r += is_report(t, lv.list[j]) ? 1u : 0u;
        pt.roff[lv.keys[i] + 1] = r;
      }
    }
    for (uint64_t k = 0; k < space; k++) {
      pt.voff[k + 1] += pt.voff[k];
      if (any_rep) pt.roff[k + 1] += pt.roff[k];
    }
    for (uint32_t v : lv.list)
      if (is_report(t, v)) pt.rlist.push_back(v);
  } else {
    pt.hmask = (uint32_t)(cap - 1);
    pt.slots.assign(cap * 4, 0);
    for (uint64_t sl = 0; sl < cap; sl++) pt.slots[sl * 4] = kHashEmpty;
    for (size_t i = 0; i < nz; i++) {
      const uint32_t vb = lv.off[i], rb = (uint32_t)pt.rlist.size();
      for (uint32_t j = lv.off[i]; j < lv.off[i + 1]; j++)
        if (is_report(t, lv.list[j])) pt.rlist.push_back(lv.list[j]);
      const uint32_t vl = lv.off[i + 1] - vb, rl = (uint32_t)pt.rlist.size() - rb;
      if (vl >= 65536 || rl >= 65536) return false;
      uint32_t h = prefix_hash(lv.keys[i]) & pt.hmask;
      while (pt.slots[(size_t)h * 4] != kHashEmpty) h = (h + 1) & pt.hmask;
      uint32_t* e = &pt.slots[(size_t)h * 4];
      e[0] = lv.keys[i];
      e[1] = vb;
      e[2] = rb;
      e[3] = (vl << 16) | rl;
    }
  }
  // PrecTable::calcCutoff (precompute_table.cu:171-186): mean non-empty list length.
  pt.cutoff = nz > 0 ? (int32_t)(lv.list.size() / nz) : 0;
  if (cutoff_opt >= 0) pt.cutoff = cutoff_opt;
  return true;
}

// Level d from level d - 1: key * L + c -> successors of key's states that
// accept class c. Keys stay ascending because each slice of `prev` is expanded
// in order. Work is split over threads by slices of prev's keys; false when
// more than `cap` entries would be produced.
bool next_level(const Level& prev, const TileHost& t, uint32_t L, int64_t cap, Level& cur) {
  const size_t nk = prev.keys.size();
  int nth = (int)std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), 32);
  nth = (int)std::min<size_t>(nth, nk / 256 + 1);
  std::vector<Level> part(nth);
  std::atomic<int64_t> total{0};
  auto work = [&](int id) {
    const size_t lo = nk * id / nth, hi = nk * (id + 1) / nth;
    Level& out = part[id];
    std::vector<uint32_t> mark(t.nstates, 0), l;
    uint32_t stamp = 0;
    int64_t reported = 0;
    for (size_t i = lo; i < hi; i++) {
      for (uint32_t c = 0; c < L; c++) {
        l.clear();
        stamp++;
        for (uint32_t j = prev.off[i]; j < prev.off[i + 1]; j++) {
          const uint32_t* sc = &t.succ[(size_t)prev.list[j] * 4];
          for (int k = 0; k < 4; k++) {
            uint32_t u = sc[k];
            if (u == kNoSucc) continue;
            u &= 0x7fffffffu;
            if (mark[u] == stamp || !accepts_cls(t, u, (int)c)) continue;
            mark[u] = stamp;
            l.push_back(u);
          }
        }
        if (l.empty()) continue;
        std::sort(l.begin(), l.end());
        out.keys.push_back(prev.keys[i] * L + c);
        out.list.insert(out.list.end(), l.begin(), l.end());
        out.off.push_back((uint32_t)out.list.size());
      }
      if ((i & 255) == 255) {  // publish progress; stop once all threads together pass cap
        const int64_t now = (int64_t)out.list.size();
        if (total.fetch_add(now - reported) + (now - reported) > cap) return;
        reported = now;
      }
    }
  };
  std::vector<std::thread> th;
  for (int i = 1; i < nth; i++) th.emplace_back(work, i);
  work(0);
  for (auto& x : th) x.join();
  int64_t sum = 0;
  for (auto& pp : part) sum += (int64_t)pp.list.size();
  if (sum > cap || sum >= (int64_t)UINT32_MAX) return false;
  cur = Level();
  cur.keys.reserve(std::accumulate(part.begin(), part.end(), (size_t)0,
                                   [](size_t a, const Level& x) { return a + x.keys.size(); }));
  cur.list.reserve((size_t)sum);
  for (auto& pp : part) {
    const uint32_t base = (uint32_t)cur.list.size();
    cur.keys.insert(cur.keys.end(), pp.keys.begin(), pp.keys.end());
    for (size_t i = 1; i < pp.off.size(); i++) cur.off.push_back(base + pp.off[i]);
    cur.list.insert(cur.list.end(), pp.list.begin(), pp.list.end());
  }
  return true;
}

int64_t table_bytes(const PrefixTableHost& pk) {
  return 4 * (int64_t)(pk.voff.size() + pk.roff.size() + pk.slots.size() + pk.vlist.size() +
                       pk.rlist.size());
}

void build_prefix_tables(TileHost& t, const TableOpts& opts, bool global) {
  // depth < 0: as deep as the size caps allow
  const int want = opts.precompute_depth < 0 ? kMaxDepth
                                             : std::max(1, std::min(opts.precompute_depth, kMaxDepth));
  const int64_t cap = opts.max_table_entries > 0
                          ? opts.max_table_entries
                          : (global ? opts.global_table_entries : (int64_t)2 << 20);
  const int64_t budget = global ? opts.auto_global_table_bytes : opts.auto_table_bytes;
  // keys are base-L numbers over the L live classes (the dead class ends paths)
  const uint32_t L = (uint32_t)t.nlive;
  Level prev;
  for (uint32_t c = 0; c < L; c++) {
    const size_t before = prev.list.size();
    for (uint32_t a : t.aas)
      if (accepts_cls(t, a, (int)c)) prev.list.push_back(a);
    if (prev.list.size() == before) continue;
    prev.keys.push_back(c);
    prev.off.push_back((uint32_t)prev.list.size());
  }
  finish_table(t.pt[0], (uint64_t)L, prev, t, opts.precompute_cutoff);
  uint64_t space = (uint64_t)L;
  int64_t bytes = table_bytes(t.pt[0]);
  t.depth = 1;
  for (int d = 2; d <= want; d++) {
    if (space * (uint64_t)L >= (1ull << 32)) break;  // keys are 32-bit
    space *= (uint64_t)L;
    Level cur;
    if (!next_level(prev, t, L, cap, cur)) break;
    if (!finish_table(t.pt[d - 1], space, cur, t, opts.precompute_cutoff)) {
      t.pt[d - 1] = PrefixTableHost();
      break;
    }
    bytes += table_bytes(t.pt[d - 1]);
    if (opts.precompute_depth < 0 && bytes > budget) {  // automatic depth: bounded device bytes
      t.pt[d - 1] = PrefixTableHost();
      break;
    }
    t.depth = d;
    prev.keys.swap(cur.keys);
    prev.off.swap(cur.off);
    prev.list.swap(cur.list);
  }
  // positions injected per refill: keep one refill's lists within about half
  // of a warp's shared worklist
  const PrefixTableHost& deep = t.pt[t.depth - 1];
  const int mean = std::max(1, deep.cutoff);
  t.inj_batch = std::max(1, std::min(32, 512 / (mean + 1)));
  // scanning the always-active list: table 1's mean is the states matched per position
  t.inj_batch0 = std::max(1, std::min(32, 2048 / (std::max(1, t.pt[0].cutoff) + 1)));
}

void build_image(TileHost& t) {
  auto r16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
  const size_t n = (size_t)t.nstates;
  t.narrow = t.nstates <= kNarrowMaxStates;
  // wide tiles are read through L2: with one class word, a state's record also
  // carries its successors' class masks, so that an expansion is one round trip
  t.fused = !t.narrow && t.cw == 1;
  t.off_cmask = (int32_t)r16(n * (t.narrow ? 8 : (t.fused ? 32 : 16)));
  t.off_rep = t.off_cmask + (int32_t)r16(n * t.cw * 4);
  t.off_sticky = t.off_rep + (int32_t)r16(((n + 31) / 32) * 4);
  t.off_cls = t.off_sticky + (int32_t)r16(((n + 31) / 32) * 4);
  t.image.assign((size_t)t.off_cls + 256, 0);
  if (t.narrow) {  // 4 x u16 per state: 15-bit id, bit 15 = report, 0xffff = none
    uint16_t* s16 = reinterpret_cast<uint16_t*>(t.image.data());
    for (size_t i = 0; i < n * 4; i++) {
      const uint32_t u = t.succ[i];
      s16[i] = u == kNoSucc ? (uint16_t)0xffff
                            : (uint16_t)((u & 0x7fffu) | ((u >> 31) ? 0x8000u : 0u));
    }
  } else if (t.fused) {  // [4 x u32 successor][4 x u32 its class mask, 0 = none] per state
    uint32_t* rec = reinterpret_cast<uint32_t*>(t.image.data());
    for (size_t i = 0; i < n; i++)
      for (int j = 0; j < 4; j++) {
        const uint32_t u = t.succ[i * 4 + j];
        rec[i * 8 + j] = u;
        rec[i * 8 + 4 + j] = u == kNoSucc ? 0u : t.cmask[(size_t)(u & 0x7fffffffu)];
      }
  } else {
    memcpy(t.image.data(), t.succ.data(), n * 16);
  }
  memcpy(t.image.data() + t.off_cmask, t.cmask.data(), n * t.cw * 4);
  memcpy(t.image.data() + t.off_rep, t.rep.data(), t.rep.size() * 4);
  memcpy(t.image.data() + t.off_sticky, t.sticky.data(), t.sticky.size() * 4);
  memcpy(t.image.data() + t.off_cls, t.cls.data(), 256);
  const int pcw = plan_class_words(t.ncls);
  t.plan_bytes = (int64_t)r16(n * (t.narrow ? 8 : (pcw == 1 ? 32 : 16))) + (int64_t)r16(n * pcw * 4) +
                 2 * (int64_t)r16(((n + 31) / 32) * 4) + 256;
}

int degree_error() {
  set_error("internal error: a state has more than 4 successors after degree limiting");
  return NGAP_E_INVALID;
}

// Tile variants: kPlain (the CCs as they are), kActivation (layered CCs: their
// pre states, sticky states terminal and reported as activations into slots
// 0..nact-1), kLayered (layered CCs without edges into sticky states, the
// sticky states pre-registered from the activation pass).
enum { kPlain = 0, kActivation = 1, kLayered = 2 };

bool emit_tile(const GroupSet& gs, const std::vector<CcInfo>& ccs, bool global, int variant,
               int pair, const TableOpts& opts, std::vector<TileHost>& tiles) {
  if (ccs.empty()) return true;
  TileHost t;
  t.group = ccs[0].group;
  t.phase = variant;
  t.pair = variant == kPlain ? -1 : pair;
  // per CC: local ids of its states in the tile (-1: not in the tile) and sticky flags
  std::vector<std::vector<int32_t>> loc(ccs.size());
  std::vector<std::vector<char>> stk(ccs.size());
  // layered tiles: dropped edges, shortcut successors of each sticky state, kept states
  std::vector<std::vector<char>> drop(ccs.size()), keep(ccs.size());
  std::vector<std::vector<std::vector<int32_t>>> dset(ccs.size());
  int32_t n = 0;
  bool bounded = true;
  int32_t mp = 0;
  Partition part;
  for (size_t ci = 0; ci < ccs.size(); ci++) {
    const CcInfo& c = ccs[ci];
    const GroupGraph& g = gs.groups[c.group];
    std::vector<char> pre;
    int32_t lp1 = 0, lp2 = 0;
    if (variant != kPlain) {
      if (!layer_flags(g, c.begin, c.end, stk[ci], pre, lp1, lp2)) return false;
      mp = std::max(mp, variant == kActivation ? lp1 : lp2);
      if (variant == kLayered) layered_shortcuts(g, c.begin, c.end, stk[ci], drop[ci], dset[ci], keep[ci]);
    } else {
      bounded = bounded && c.bounded;
      mp = std::max(mp, c.max_path);
    }
    loc[ci].assign(c.end - c.begin, -1);
    for (int32_t v = c.begin; v < c.end; v++) {
      if (variant == kActivation && !pre[v - c.begin]) continue;
      if (variant == kLayered && !keep[ci][v - c.begin]) continue;
      loc[ci][v - c.begin] = n++;
      part.refine(&g.bits[(size_t)v * 8]);
    }
  }
  t.nstates = n;
  t.num_ccs = (int32_t)ccs.size();
  t.max_path = bounded ? mp : -1;
  t.global = global;
  if (n == 0) return true;
  t.cw = class_words(part.n);
  t.cls.resize(256);
  {
    // bytes no state accepts share one (dead) class; number it last. The
    // keys count only the live classes, so prefix tables reach one more
    // level within 32-bit keys than keys over raw bytes (95 printable
    // classes: depth 4 instead of 3)
    uint32_t any[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (size_t ci = 0; ci < ccs.size(); ci++) {
      const CcInfo& c = ccs[ci];
      const GroupGraph& g = gs.groups[c.group];
      for (int32_t v = c.begin; v < c.end; v++)
        if (loc[ci][v - c.begin] >= 0)
          for (int w = 0; w < 8; w++) any[w] |= g.bits[(size_t)v * 8 + w];
    }
    int dead = -1;
    for (int b = 0; b < 256 && dead < 0; b++)
      if (!((any[b >> 5] >> (b & 31)) & 1u)) dead = part.id[b];
    t.ncls = part.n;
    t.nlive = dead < 0 ? part.n : part.n - 1;
    for (int b = 0; b < 256; b++) {
      int id = part.id[b];
      if (dead >= 0) id = id == dead ? part.n - 1 : (id > dead ? id - 1 : id);
      t.cls[b] = (uint8_t)id;
    }
  }
  t.succ.assign((size_t)n * 4, kNoSucc);
  t.bits.resize((size_t)n * 8);
  t.cmask.assign((size_t)n * t.cw, 0);
  t.rep.assign((n + 31) / 32, 0);
  t.sid.resize(n);
  std::vector<uint32_t> aas_bit((n + 31) / 32, 0);
  t.sticky.assign((n + 31) / 32, 0);
  std::vector<int32_t> act_cc;  // layered tiles: CC of each activation slot
  for (size_t ci = 0; ci < ccs.size(); ci++) {
    const CcInfo& c = ccs[ci];
    const GroupGraph& g = gs.groups[c.group];
    const std::vector<int32_t>& lc = loc[ci];
    for (int32_t v = c.begin; v < c.end; v++) {
      const int32_t local = lc[v - c.begin];
      if (local < 0) continue;
      const bool sv = variant != kPlain && stk[ci][v - c.begin];
      t.sid[local] = (uint32_t)v | ((uint32_t)c.group << 22);
      const uint32_t* bv = &g.bits[(size_t)v * 8];
      for (int w = 0; w < 8; w++) t.bits[(size_t)local * 8 + w] = bv[w];
      for (int b = 0; b < 256; b++)
        if ((bv[b >> 5] >> (b & 31)) & 1u) {
          int cl = t.cls[b];
          t.cmask[(size_t)local * t.cw + (cl >> 5)] |= 1u << (cl & 31);
        }
      if (variant == kActivation) {
        // sticky states are the only reports; their id is the activation slot
        if (sv) {
          t.rep[local >> 5] |= 1u << (local & 31);
          t.sid[local] = (uint32_t)t.nact++;
        }
      } else if (g.attrs[v] & 2) {
        t.rep[local >> 5] |= 1u << (local & 31);
      }
      if (variant == kLayered && sv) {
        t.sticky[local >> 5] |= 1u << (local & 31);
        t.act_local.push_back((uint32_t)local);
        act_cc.push_back((int32_t)ci);
        t.nact++;
      }
      if (g.attrs[v] & 1) {
        t.aas.push_back((uint32_t)local);
        aas_bit[local >> 5] |= 1u << (local & 31);
      }
      int j = 0;
      for (int32_t k = g.row_offsets[v]; k < g.row_offsets[v + 1]; k++) {
        int32_t u = g.cols[k];
        if (g.attrs[u] & 1) continue;  // redundant: u is active at every position
        if (variant == kActivation && sv) continue;  // sticky states end the activation part
        if (variant != kPlain && stk[ci][u - c.begin]) {
          // into a sticky state: kept only by the activation part (not its self-loop)
          if (variant == kLayered || u == v) continue;
        }
        if (variant == kLayered && drop[ci][k - g.row_offsets[c.begin]]) continue;  // a shortcut
        const int32_t ul = lc[u - c.begin];
        if (ul < 0) continue;          // not a pre state: no path to a sticky state
        if (j >= 4) return false;      // the degree limiter guarantees at most 4
        const bool urep = variant == kActivation ? (bool)stk[ci][u - c.begin]
                                                 : (g.attrs[u] & 2) != 0;
        t.succ[(size_t)local * 4 + j++] = (uint32_t)ul | (urep ? 0x80000000u : 0u);
      }
    }
    // start-of-data states of the CC, ascending (the group's list is ascending)
    auto lo = std::lower_bound(g.starts.begin(), g.starts.end(), c.begin);
    for (auto it = lo; it != g.starts.end() && *it < c.end; ++it)
      if (lc[*it - c.begin] >= 0) t.start.push_back((uint32_t)lc[*it - c.begin]);
  }
  // layered tiles: bits 28..31 of a slot's act_local mark its successors
  // (record order) that the sticky state enables from its first match on
  // (shortcuts, layered_shortcuts); the others it enables after it
  if (variant == kLayered) {
    if (n > (int32_t)kActIdMask) return false;
    for (int32_t i = 0; i < t.nact; i++) {
      const CcInfo& c = ccs[act_cc[i]];
      const uint32_t s = t.act_local[i];
      const std::vector<int32_t>& d = dset[act_cc[i]][(t.sid[s] & 0x3fffffu) - c.begin];
      uint32_t incl = 0;
      for (int j = 0; j < 4; j++) {
        const uint32_t u = t.succ[(size_t)s * 4 + j];
        if (u != kNoSucc &&
            std::binary_search(d.begin(), d.end(), (int32_t)(t.sid[u & 0x7fffffffu] & 0x3fffffu)))
          incl |= 1u << j;
      }
      t.act_local[i] = s | incl << 28;
    }
  }
  // sticky states of plain tiles: not always-active, a self-loop and every
  // byte accepted; once such a state matches it matches at every later
  // position of the segment (layered tiles marked theirs above; activation
  // tiles have none: their sticky states are terminal)
  if (variant == kPlain) {
    for (int32_t v = 0; v < n; v++) {
      bool all = true;
      for (int w = 0; w < 8; w++) all = all && t.bits[(size_t)v * 8 + w] == 0xffffffffu;
      bool self = false;
      for (int j = 0; j < 4; j++)
        self = self || (t.succ[(size_t)v * 4 + j] & 0x7fffffffu) == (uint32_t)v;
      const bool aas = (aas_bit[v >> 5] >> (v & 31)) & 1u;
      if (all && self && !aas) t.sticky[v >> 5] |= 1u << (v & 31);
    }
  }
  for (uint32_t w : t.sticky) t.nsticky += __builtin_popcount(w);
  if (variant == kLayered) {  // union of the successors' class masks of every slot
    t.stk_union.assign((size_t)t.nact * t.cw, 0);
    for (int32_t i = 0; i < t.nact; i++) {
      const uint32_t s = t.act_local[i] & kActIdMask;
      for (int j = 0; j < 4; j++) {
        const uint32_t u = t.succ[(size_t)s * 4 + j];
        if (u == kNoSucc) continue;
        for (int k = 0; k < t.cw; k++)
          t.stk_union[(size_t)i * t.cw + k] |= t.cmask[(size_t)(u & 0x7fffffffu) * t.cw + k];
      }
    }
  }
  build_prefix_tables(t, opts, global);
  build_image(t);
  tiles.push_back(std::move(t));
  return true;
}

// Packs CCs into tiles in order: a tile is closed when the next CC would pass
// `max_states` or, for shared-memory tiles, the image budget. Layered CCs are
// packed into pairs of tiles (activation, layered) over the same CCs.
class TilePacker {
 public:
  TilePacker(const GroupSet& gs, const TableOpts& opts, bool global, bool layered,
             int64_t max_states, int* pairs, std::vector<TileHost>& tiles)
      : gs_(gs), opts_(opts), global_(global), layered_(layered), max_states_(max_states),
        pairs_(pairs), tiles_(tiles) {}

  bool add(const CcInfo& ci) {
    const GroupGraph& g = gs_.groups[ci.group];
    const int32_t sz = ci.end - ci.begin;
    Partition trial = part_;
    if (!global_)
      for (int32_t v = ci.begin; v < ci.end; v++) trial.refine(&g.bits[(size_t)v * 8]);
    const bool fits = n_ + sz <= max_states_ &&
                      (global_ || image_bytes(n_ + sz, plan_class_words(trial.n)) <= opts_.image_budget);
    if (!open_.empty() && !fits) {
      if (!flush()) return false;
      if (!global_)
        for (int32_t v = ci.begin; v < ci.end; v++) part_.refine(&g.bits[(size_t)v * 8]);
    } else {
      part_ = trial;
    }
    open_.push_back(ci);
    n_ += sz;
    return true;
  }

  bool flush() {
    bool ok = true;
    if (!open_.empty()) {
      if (layered_) {
        const int pair = (*pairs_)++;
        ok = emit_tile(gs_, open_, global_, kActivation, pair, opts_, tiles_) &&
             emit_tile(gs_, open_, global_, kLayered, pair, opts_, tiles_);
      } else {
        ok = emit_tile(gs_, open_, global_, kPlain, -1, opts_, tiles_);
      }
    }
    open_.clear();
    n_ = 0;
    part_ = Partition();
    return ok;
  }

 private:
  const GroupSet& gs_;
  const TableOpts& opts_;
  bool global_, layered_;
  int64_t max_states_;
  int* pairs_;
  std::vector<TileHost>& tiles_;
  std::vector<CcInfo> open_;
  int64_t n_ = 0;
  Partition part_;
};

// CC indices of one kind -> the sets that become global tiles. Clusters by
// alphabet (the bytes any state of the CC accepts) with at most 32 byte
// classes become global when they would need more than two shared-memory
// tiles; the remaining CCs of the kind form one more global set when they too
// would need more than two.
std::vector<std::vector<int>> global_sets_of(const GroupSet& gs, const std::vector<CcInfo>& ccs,
                                             const std::vector<int>& kind, const TableOpts& opts) {
  std::map<std::array<uint32_t, 8>, std::vector<int>> clusters;
  for (int i : kind) {
    const GroupGraph& g = gs.groups[ccs[i].group];
    std::array<uint32_t, 8> alpha{};
    for (int32_t v = ccs[i].begin; v < ccs[i].end; v++)
      for (int w = 0; w < 8; w++) alpha[w] |= g.bits[(size_t)v * 8 + w];
    clusters[alpha].push_back(i);
  }
  const int64_t two_tiles = 2 * (int64_t)opts.image_budget;
  std::vector<std::vector<int>> sets;
  std::vector<int> rest;
  Partition rest_part;
  int64_t rest_n = 0;
  for (auto& kv : clusters) {
    Partition part;
    int64_t n = 0;
    for (int i : kv.second) {
      const GroupGraph& g = gs.groups[ccs[i].group];
      n += ccs[i].end - ccs[i].begin;
      for (int32_t v = ccs[i].begin; v < ccs[i].end; v++) part.refine(&g.bits[(size_t)v * 8]);
    }
    if (plan_class_words(part.n) == 1 && image_bytes(n, 1) > two_tiles) {
      sets.push_back(kv.second);
    } else {
      for (int i : kv.second) {
        const GroupGraph& g = gs.groups[ccs[i].group];
        for (int32_t v = ccs[i].begin; v < ccs[i].end; v++) rest_part.refine(&g.bits[(size_t)v * 8]);
      }
      rest.insert(rest.end(), kv.second.begin(), kv.second.end());
      rest_n += n;
    }
  }
  if (!rest.empty() && image_bytes(rest_n, plan_class_words(rest_part.n)) > two_tiles)
    sets.push_back(rest);
  return sets;
}

}  // namespace

int build_tiles(const GroupSet& gs, const TableOpts& opts, std::vector<TileHost>& tiles) {
  tiles.clear();
  std::vector<CcInfo> ccs;
  std::vector<int> bounded, layered;
  std::vector<char> sticky, pre;
  for (int gi = 0; gi < (int)gs.groups.size(); gi++) {
    const GroupGraph& g = gs.groups[gi];
    const int nccs = (int)g.cc_begin.size() - 1;
    for (int c = 0; c < nccs; c++) {
      CcInfo ci;
      ci.group = gi;
      ci.begin = g.cc_begin[c];
      ci.end = g.cc_begin[c + 1];
      int32_t lp = cc_longest_path(g, ci.begin, ci.end);
      ci.bounded = lp >= 0 && lp <= opts.max_warmup;
      ci.max_path = ci.bounded ? lp : -1;
      ci.layered = false;
      if (!ci.bounded && lp < 0 && opts.layered) {
        int32_t lp1 = 0, lp2 = 0;
        ci.layered = layer_flags(g, ci.begin, ci.end, sticky, pre, lp1, lp2) &&
                     lp1 <= opts.max_warmup && lp2 <= opts.max_warmup;
      }
      if (ci.bounded) bounded.push_back((int)ccs.size());
      if (ci.layered) layered.push_back((int)ccs.size());
      ccs.push_back(ci);
    }
  }
  // Global tiles (tile_mode 2: every acyclic or layered CC; 0: the sets
  // global_sets_of picks); everything else, other cyclic CCs included, uses
  // shared-memory tiles of one group.
  std::vector<char> in_global(ccs.size(), 0);
  std::vector<std::vector<int>> gsets[2];
  if (opts.tile_mode == 2) {
    if (!bounded.empty()) gsets[0].push_back(bounded);
    if (!layered.empty()) gsets[1].push_back(layered);
  } else if (opts.tile_mode == 0) {
    gsets[0] = global_sets_of(gs, ccs, bounded, opts);
    gsets[1] = global_sets_of(gs, ccs, layered, opts);
  }
  // Acyclic and layered tiles get parallelism from chunks, so they fill the
  // budget. A cyclic tile is one sequential unit per segment, so those stay
  // small to give the GPU enough independent units.
  const int64_t cap_chunked = opts.tile_states > 0 ? opts.tile_states : (int64_t)kMaxTileStates - 2;
  const int64_t cap_cyclic = opts.tile_states > 0 ? opts.tile_states : (int64_t)opts.unbounded_tile_states;
  int pairs = 0;
  for (int k = 0; k < 2; k++)
    for (auto& set : gsets[k]) {
      std::sort(set.begin(), set.end());  // (group, CC) order
      TilePacker pk(gs, opts, true, k == 1, cap_chunked, &pairs, tiles);
      for (int i : set) {
        in_global[i] = 1;
        if (!pk.add(ccs[i])) return degree_error();
      }
      if (!pk.flush()) return degree_error();
    }
  for (int gi = 0; gi < (int)gs.groups.size(); gi++) {
    TilePacker b(gs, opts, false, false, cap_chunked, &pairs, tiles);
    TilePacker l(gs, opts, false, true, cap_chunked, &pairs, tiles);
    TilePacker u(gs, opts, false, false, cap_cyclic, &pairs, tiles);
    for (size_t i = 0; i < ccs.size(); i++) {
      const CcInfo& ci = ccs[i];
      if (ci.group != gi || in_global[i]) continue;
      TilePacker& pk = ci.bounded ? b : (ci.layered ? l : u);
      if (!pk.add(ci)) return degree_error();
    }
    if (!b.flush() || !l.flush() || !u.flush()) return degree_error();
  }
  return NGAP_OK;
}

int table_opts_from(const ngap_table_opts* opts, const char* fn, TableOpts& out, int* device) {
  ngap_table_opts o{};
  o.precompute_cutoff = -1;
  if (opts) o = *opts;
  if (o.precompute_depth < -1 || o.precompute_depth > kMaxDepth) {
    set_error("%s: precompute_depth must be in -1..%d (got %d)", fn, kMaxDepth, o.precompute_depth);
    return NGAP_E_INVALID;
  }
  if (o.tile_mode < NGAP_TILES_AUTO || o.tile_mode > NGAP_TILES_GLOBAL) {
    set_error("%s: tile_mode must be NGAP_TILES_AUTO, _SHARED or _GLOBAL (got %d)", fn, o.tile_mode);
    return NGAP_E_INVALID;
  }
  out = TableOpts();
  out.precompute_depth = o.precompute_depth;
  out.precompute_cutoff = o.precompute_cutoff;
  out.tile_states = o.tile_states;
  out.max_table_entries = o.max_table_entries;
  out.tile_mode = o.tile_mode;
  if (device) *device = o.device;
  return NGAP_OK;
}

}  // namespace ngap
