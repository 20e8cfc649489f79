// Tiles, byte classes, shared-memory images and prefix-memoization tables.
//
// A tile is a set of whole CCs of one group. CCs never share states or edges,
// so splitting a group into tiles changes no report: a report keeps its
// group-local sid (TileHost::sid) and its group index. Two facts about the
// graph are used:
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
#include <cstring>
#include <map>

namespace ngap {

namespace {

struct CcInfo {
  int32_t begin, end;
  bool bounded;
  int32_t max_path;
};

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

int class_words(int ncls) { return ncls <= 32 ? 1 : (ncls <= 64 ? 2 : 8); }

inline bool accepts_cls(const TileHost& t, uint32_t v, int c) {
  return (t.cmask[(size_t)v * t.cw + (c >> 5)] >> (c & 31)) & 1u;
}

inline bool is_report(const TileHost& t, uint32_t v) { return (t.rep[v >> 5] >> (v & 31)) & 1u; }

// Lays out one table; false when a list is too long for the hashed slot format.
bool finish_table(PrefixTableHost& pt, uint64_t space,
                  const std::map<uint32_t, std::vector<uint32_t>>& lists, const TileHost& t,
                  int cutoff_opt) {
  pt = PrefixTableHost();
  pt.dense = space <= kDenseKeys;
  int64_t total = 0, nonzero = 0;
  if (pt.dense) {
    pt.voff.assign(space + 1, 0);
    pt.roff.assign(space + 1, 0);
    std::vector<uint32_t> vcount(space, 0), rcount(space, 0);
    for (auto& kv : lists) {
      vcount[kv.first] = (uint32_t)kv.second.size();
      for (uint32_t v : kv.second)
        if (is_report(t, v)) rcount[kv.first]++;
    }
    for (uint64_t k = 0; k < space; k++) {
      pt.voff[k + 1] = pt.voff[k] + vcount[k];
      pt.roff[k + 1] = pt.roff[k] + rcount[k];
    }
    pt.vlist.resize(pt.voff[space]);
    pt.rlist.resize(pt.roff[space]);
    for (auto& kv : lists) {
      uint32_t vo = pt.voff[kv.first], ro = pt.roff[kv.first];
      for (uint32_t v : kv.second) {
        pt.vlist[vo++] = v;
        if (is_report(t, v)) pt.rlist[ro++] = v;
      }
    }
  } else {
    uint64_t cap = 16;
    while (cap < 2 * lists.size()) cap <<= 1;
    pt.hmask = (uint32_t)(cap - 1);
    pt.slots.assign(cap * 4, 0);
    for (uint64_t s = 0; s < cap; s++) pt.slots[s * 4] = kHashEmpty;
    for (auto& kv : lists) {
      const uint32_t vb = (uint32_t)pt.vlist.size(), rb = (uint32_t)pt.rlist.size();
      for (uint32_t v : kv.second) {
        pt.vlist.push_back(v);
        if (is_report(t, v)) pt.rlist.push_back(v);
      }
      const uint32_t vl = (uint32_t)pt.vlist.size() - vb, rl = (uint32_t)pt.rlist.size() - rb;
      if (vl >= 65536 || rl >= 65536) return false;
      uint32_t h = prefix_hash(kv.first) & pt.hmask;
      while (pt.slots[(size_t)h * 4] != kHashEmpty) h = (h + 1) & pt.hmask;
      uint32_t* sl = &pt.slots[(size_t)h * 4];
      sl[0] = kv.first;
      sl[1] = vb;
      sl[2] = rb;
      sl[3] = (vl << 16) | rl;
    }
  }
  if (pt.rlist.empty()) pt.roff.clear();  // no reports: the offsets are never read
  for (auto& kv : lists) {
    total += (int64_t)kv.second.size();
    nonzero++;
  }
  // PrecTable::calcCutoff (precompute_table.cu:171-186): mean non-empty list length.
  pt.cutoff = nonzero > 0 ? (int32_t)(total / nonzero) : 0;
  if (cutoff_opt >= 0) pt.cutoff = cutoff_opt;
  return true;
}

void build_prefix_tables(TileHost& t, const TableOpts& opts) {
  // depth < 0: as deep as the size caps allow
  const int want = opts.precompute_depth < 0 ? kMaxDepth
                                             : std::max(1, std::min(opts.precompute_depth, kMaxDepth));
  const int64_t cap = opts.max_table_entries > 0 ? opts.max_table_entries : (int64_t)2 << 20;
  // keys are base-L numbers over the L live classes (the dead class ends paths)
  const uint32_t L = (uint32_t)t.nlive;
  std::map<uint32_t, std::vector<uint32_t>> prev, cur;
  for (uint32_t c = 0; c < L; c++) {
    std::vector<uint32_t> l;
    for (uint32_t a : t.aas)
      if (accepts_cls(t, a, (int)c)) l.push_back(a);
    if (!l.empty()) prev[c] = std::move(l);
  }
  finish_table(t.pt[0], (uint64_t)L, prev, t, opts.precompute_cutoff);
  uint64_t space = (uint64_t)L;
  t.depth = 1;
  std::vector<uint32_t> mark(t.nstates, 0);
  uint32_t stamp = 0;
  for (int d = 2; d <= want; d++) {
    if (space * (uint64_t)L >= (1ull << 32)) break;  // keys are 32-bit
    space *= (uint64_t)L;
    cur.clear();
    int64_t total = 0;
    bool too_big = false;
    for (auto& kv : prev) {
      for (int c = 0; c < (int)L && !too_big; c++) {
        std::vector<uint32_t> l;
        stamp++;
        for (uint32_t v : kv.second) {
          const uint32_t* sc = &t.succ[(size_t)v * 4];
          for (int j = 0; j < 4; j++) {
            uint32_t u = sc[j];
            if (u == kNoSucc) continue;
            u &= 0x7fffffffu;
            if (!accepts_cls(t, u, c) || mark[u] == stamp) continue;
            mark[u] = stamp;
            l.push_back(u);
          }
        }
        if (!l.empty()) {
          std::sort(l.begin(), l.end());
          total += (int64_t)l.size();
          cur[kv.first * L + (uint32_t)c] = std::move(l);
          if (total > cap) too_big = true;
        }
      }
      if (too_big) break;
    }
    if (too_big) break;
    if (!finish_table(t.pt[d - 1], space, cur, t, opts.precompute_cutoff)) {
      t.pt[d - 1] = PrefixTableHost();
      break;
    }
    if (opts.precompute_depth < 0) {  // automatic depth: bounded device bytes per tile
      int64_t bytes = 0;
      for (int k = 0; k < d; k++) {
        const PrefixTableHost& pk = t.pt[k];
        bytes += 4 * (int64_t)(pk.voff.size() + pk.roff.size() + pk.slots.size() +
                               pk.vlist.size() + pk.rlist.size());
      }
      if (bytes > opts.auto_table_bytes) {
        t.pt[d - 1] = PrefixTableHost();
        break;
      }
    }
    t.depth = d;
    prev.swap(cur);
  }
  // positions injected per refill: keep one refill's lists within about half
  // of a warp's shared worklist
  const PrefixTableHost& deep = t.pt[t.depth - 1];
  const int mean = std::max(1, deep.cutoff);
  t.inj_batch = std::max(1, std::min(32, 512 / (mean + 1)));
}

void build_image(TileHost& t) {
  auto r16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
  const size_t n = (size_t)t.nstates;
  t.narrow = t.nstates <= kNarrowMaxStates;
  t.off_cmask = (int32_t)r16(n * (t.narrow ? 8 : 16));
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
  } else {
    memcpy(t.image.data(), t.succ.data(), n * 16);
  }
  memcpy(t.image.data() + t.off_cmask, t.cmask.data(), n * t.cw * 4);
  memcpy(t.image.data() + t.off_rep, t.rep.data(), t.rep.size() * 4);
  memcpy(t.image.data() + t.off_sticky, t.sticky.data(), t.sticky.size() * 4);
  memcpy(t.image.data() + t.off_cls, t.cls.data(), 256);
}

int degree_error() {
  set_error("internal error: a state has more than 4 successors after degree limiting");
  return NGAP_E_INVALID;
}

bool emit_tile(const GroupGraph& g, int gi, const std::vector<CcInfo>& ccs, const TableOpts& opts,
               std::vector<TileHost>& tiles) {
  if (ccs.empty()) return true;
  TileHost t;
  t.group = gi;
  int32_t n = 0;
  bool bounded = true;
  int32_t mp = 0;
  Partition part;
  for (auto& c : ccs) {
    n += c.end - c.begin;
    bounded = bounded && c.bounded;
    mp = std::max(mp, c.max_path);
    for (int32_t v = c.begin; v < c.end; v++) part.refine(&g.bits[(size_t)v * 8]);
  }
  t.nstates = n;
  t.num_ccs = (int32_t)ccs.size();
  t.max_path = bounded ? mp : -1;
  t.cw = class_words(part.n);
  t.cls.resize(256);
  if (t.cw == 8) {  // more than 64 classes: classes are the bytes themselves
    t.ncls = 256;
    t.nlive = 256;
    for (int b = 0; b < 256; b++) t.cls[b] = (uint8_t)b;
  } else {
    // bytes no state accepts share one (dead) class; number it last
    uint32_t any[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (auto& c : ccs)
      for (int32_t v = c.begin; v < c.end; v++)
        for (int w = 0; w < 8; w++) any[w] |= g.bits[(size_t)v * 8 + w];
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
  int32_t local = 0;
  for (auto& c : ccs) {
    for (int32_t v = c.begin; v < c.end; v++, local++) {
      t.sid[local] = (uint32_t)v;
      const uint32_t* bv = &g.bits[(size_t)v * 8];
      for (int w = 0; w < 8; w++) t.bits[(size_t)local * 8 + w] = bv[w];
      for (int b = 0; b < 256; b++)
        if ((bv[b >> 5] >> (b & 31)) & 1u) {
          int cl = t.cls[b];
          t.cmask[(size_t)local * t.cw + (cl >> 5)] |= 1u << (cl & 31);
        }
      if (g.attrs[v] & 2) t.rep[local >> 5] |= 1u << (local & 31);
      if (g.attrs[v] & 1) t.aas.push_back((uint32_t)local);
      int j = 0;
      for (int32_t k = g.row_offsets[v]; k < g.row_offsets[v + 1]; k++) {
        int32_t u = g.cols[k];
        if (g.attrs[u] & 1) continue;  // redundant: u is active at every position
        if (j >= 4) return false;      // the degree limiter guarantees at most 4
        uint32_t ul = (uint32_t)(u - c.begin + (local - (v - c.begin)));
        t.succ[(size_t)local * 4 + j++] = ul | ((g.attrs[u] & 2) ? 0x80000000u : 0u);
      }
    }
  }
  // start-of-data states in ascending sid order
  for (int32_t s : g.starts) {
    int32_t base = 0;
    for (auto& c : ccs) {
      if (s >= c.begin && s < c.end) {
        t.start.push_back((uint32_t)(base + s - c.begin));
        break;
      }
      base += c.end - c.begin;
    }
  }
  // sticky states: not always-active, a self-loop and every byte accepted; once
  // such a state matches it matches at every later position of the segment
  t.sticky.assign((n + 31) / 32, 0);
  for (int32_t v = 0; v < n; v++) {
    bool all = true;
    for (int w = 0; w < 8; w++) all = all && t.bits[(size_t)v * 8 + w] == 0xffffffffu;
    bool self = false;
    for (int j = 0; j < 4; j++) self = self || (t.succ[(size_t)v * 4 + j] & 0x7fffffffu) == (uint32_t)v;
    bool aas = std::find(t.aas.begin(), t.aas.end(), (uint32_t)v) != t.aas.end();
    if (all && self && !aas) {
      t.sticky[v >> 5] |= 1u << (v & 31);
      t.nsticky++;
    }
  }
  build_prefix_tables(t, opts);
  build_image(t);
  tiles.push_back(std::move(t));
  return true;
}

}  // namespace

int build_tiles(const GroupSet& gs, const TableOpts& opts, std::vector<TileHost>& tiles) {
  tiles.clear();
  // Acyclic tiles get parallelism from chunks, so they fill the image budget.
  // A cyclic tile is one sequential unit per segment, so those stay small to
  // give the GPU enough independent units.
  const int64_t max_states[2] = {
      opts.tile_states > 0 ? opts.tile_states : (int64_t)kMaxTileStates - 2,
      opts.tile_states > 0 ? opts.tile_states : (int64_t)opts.unbounded_tile_states};
  for (int gi = 0; gi < (int)gs.groups.size(); gi++) {
    const GroupGraph& g = gs.groups[gi];
    std::vector<CcInfo> open[2];  // [0] bounded, [1] unbounded
    int32_t open_n[2] = {0, 0};
    Partition open_part[2];
    const int nccs = (int)g.cc_begin.size() - 1;
    for (int c = 0; c < nccs; c++) {
      CcInfo ci;
      ci.begin = g.cc_begin[c];
      ci.end = g.cc_begin[c + 1];
      int32_t lp = cc_longest_path(g, ci.begin, ci.end);
      ci.bounded = lp >= 0 && lp <= opts.max_warmup;
      ci.max_path = ci.bounded ? lp : -1;
      const int k = ci.bounded ? 0 : 1;
      const int32_t sz = ci.end - ci.begin;
      Partition trial = open_part[k];
      for (int32_t v = ci.begin; v < ci.end; v++) trial.refine(&g.bits[(size_t)v * 8]);
      const bool fits = open_n[k] + sz <= max_states[k] &&
                        image_bytes(open_n[k] + sz, class_words(trial.n)) <= opts.image_budget;
      if (!open[k].empty() && !fits) {
        if (!emit_tile(g, gi, open[k], opts, tiles)) return degree_error();
        open[k].clear();
        open_n[k] = 0;
        open_part[k] = Partition();
        for (int32_t v = ci.begin; v < ci.end; v++) open_part[k].refine(&g.bits[(size_t)v * 8]);
      } else {
        open_part[k] = trial;
      }
      open[k].push_back(ci);
      open_n[k] += sz;
    }
    for (int k = 0; k < 2; k++)
      if (!emit_tile(g, gi, open[k], opts, tiles)) return degree_error();
  }
  return NGAP_OK;
}

}  // namespace ngap
