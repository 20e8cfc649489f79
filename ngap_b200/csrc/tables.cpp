// Tiles and prefix-memoization tables.
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
// Prefix tables follow ngap::getPrecomputeResultsForKGroupsInCsr and
// recursivePrecomputeForK (code/src/ngap/ngap.cu:2358-2513): table 1 maps a
// byte to the always-active states accepting it; table d maps a d-byte key to
// the successors of table d-1's states accepting the last byte; each table also
// lists the report states among its states. Lists are deduplicated (the
// reference keeps duplicates; the set of activations is the same).
#include "tables.h"

#include <algorithm>
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

inline bool accepts(const TileHost& t, uint32_t v, int s) {
  return (t.bits[(size_t)v * 8 + (s >> 5)] >> (s & 31)) & 1u;
}

inline bool is_report(const TileHost& t, uint32_t v) { return (t.rep[v >> 5] >> (v & 31)) & 1u; }

void finish_table(PrefixTableHost& pt, int depth, const std::map<uint32_t, std::vector<uint32_t>>& lists,
                  const TileHost& t, int cutoff_opt) {
  pt.dense = depth <= 2;
  uint64_t space = 1ull << (8 * depth);
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
    pt.voff.push_back(0);
    pt.roff.push_back(0);
    for (auto& kv : lists) {
      pt.keys.push_back(kv.first);
      for (uint32_t v : kv.second) pt.vlist.push_back(v);
      pt.voff.push_back((uint32_t)pt.vlist.size());
      bool any = false;
      for (uint32_t v : kv.second)
        if (is_report(t, v)) {
          pt.rlist.push_back(v);
          any = true;
        }
      if (any) {
        pt.rkeys.push_back(kv.first);
        pt.roff.push_back((uint32_t)pt.rlist.size());
      }
    }
  }
  for (auto& kv : lists) {
    total += (int64_t)kv.second.size();
    nonzero++;
  }
  // PrecTable::calcCutoff (precompute_table.cu:171-186): mean non-empty list length.
  pt.cutoff = nonzero > 0 ? (int32_t)(total / nonzero) : 0;
  if (cutoff_opt >= 0) pt.cutoff = cutoff_opt;
}

void build_prefix_tables(TileHost& t, const TableOpts& opts) {
  int want = std::max(1, std::min(opts.precompute_depth, kMaxDepth));
  int64_t cap = opts.max_table_entries > 0 ? opts.max_table_entries : (int64_t)8 << 20;
  std::map<uint32_t, std::vector<uint32_t>> prev, cur;
  for (int s = 0; s < 256; s++) {
    std::vector<uint32_t> l;
    for (uint32_t a : t.aas)
      if (accepts(t, a, s)) l.push_back(a);
    if (!l.empty()) prev[(uint32_t)s] = std::move(l);
  }
  finish_table(t.pt[0], 1, prev, t, opts.precompute_cutoff);
  t.depth = 1;
  std::vector<uint32_t> mark(t.nstates, 0);
  uint32_t stamp = 0;
  for (int d = 2; d <= want; d++) {
    cur.clear();
    int64_t total = 0;
    bool too_big = false;
    for (auto& kv : prev) {
      for (int s = 0; s < 256 && !too_big; s++) {
        std::vector<uint32_t> l;
        stamp++;
        for (uint32_t v : kv.second) {
          const uint32_t* sc = &t.succ[(size_t)v * 4];
          for (int j = 0; j < 4; j++) {
            uint32_t u = sc[j];
            if (u == kNoSucc) continue;
            u &= 0x7fffffffu;
            if (!accepts(t, u, s) || mark[u] == stamp) continue;
            mark[u] = stamp;
            l.push_back(u);
          }
        }
        if (!l.empty()) {
          std::sort(l.begin(), l.end());
          total += (int64_t)l.size();
          cur[(kv.first << 8) | (uint32_t)s] = std::move(l);
          if (total > cap) too_big = true;
        }
      }
      if (too_big) break;
    }
    if (too_big) break;
    finish_table(t.pt[d - 1], d, cur, t, opts.precompute_cutoff);
    t.depth = d;
    prev.swap(cur);
  }
}

bool emit_tile(const GroupGraph& g, int gi, const std::vector<CcInfo>& ccs, const TableOpts& opts,
               std::vector<TileHost>& tiles) {
  if (ccs.empty()) return true;
  TileHost t;
  t.group = gi;
  int32_t n = 0;
  bool bounded = true;
  int32_t mp = 0;
  for (auto& c : ccs) {
    n += c.end - c.begin;
    bounded = bounded && c.bounded;
    mp = std::max(mp, c.max_path);
  }
  t.nstates = n;
  t.num_ccs = (int32_t)ccs.size();
  t.max_path = bounded ? mp : -1;
  t.succ.assign((size_t)n * 4, kNoSucc);
  t.bits.resize((size_t)n * 8);
  t.rep.assign((n + 31) / 32, 0);
  t.sid.resize(n);
  int32_t local = 0;
  for (auto& c : ccs) {
    for (int32_t v = c.begin; v < c.end; v++, local++) {
      t.sid[local] = (uint32_t)v;
      for (int w = 0; w < 8; w++) t.bits[(size_t)local * 8 + w] = g.bits[(size_t)v * 8 + w];
      if (g.attrs[v] & 2) t.rep[local >> 5] |= 1u << (local & 31);
      if (g.attrs[v] & 1) t.aas.push_back((uint32_t)local);
      int j = 0;
      for (int32_t k = g.row_offsets[v]; k < g.row_offsets[v + 1]; k++) {
        int32_t u = g.cols[k];
        if (g.attrs[u] & 1) continue;  // redundant: u is active at every position
        if (j >= 4) return false;  // the degree limiter guarantees at most 4
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
  build_prefix_tables(t, opts);
  tiles.push_back(std::move(t));
  return true;
}

int degree_error() {
  set_error("internal error: a state has more than 4 successors after degree limiting");
  return NGAP_E_INVALID;
}

}  // namespace

int build_tiles(const GroupSet& gs, const TableOpts& opts, std::vector<TileHost>& tiles) {
  tiles.clear();
  const int32_t tile_states = opts.tile_states > 0 ? opts.tile_states : 2048;
  for (int gi = 0; gi < (int)gs.groups.size(); gi++) {
    const GroupGraph& g = gs.groups[gi];
    std::vector<CcInfo> open[2];  // [0] bounded, [1] unbounded
    int32_t open_n[2] = {0, 0};
    const int nccs = (int)g.cc_begin.size() - 1;
    for (int c = 0; c < nccs; c++) {
      CcInfo ci;
      ci.begin = g.cc_begin[c];
      ci.end = g.cc_begin[c + 1];
      int32_t lp = cc_longest_path(g, ci.begin, ci.end);
      ci.bounded = lp >= 0 && lp <= opts.max_warmup;
      ci.max_path = ci.bounded ? lp : -1;
      int k = ci.bounded ? 0 : 1;
      int32_t sz = ci.end - ci.begin;
      if (!open[k].empty() && open_n[k] + sz > tile_states) {
        if (!emit_tile(g, gi, open[k], opts, tiles)) return degree_error();
        open[k].clear();
        open_n[k] = 0;
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
