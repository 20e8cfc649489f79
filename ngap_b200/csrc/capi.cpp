// Host-side C ABI: errors, ANML front-end, grouping, group views and the
// CPU checker behind the CLI's --validation flag.
#include <algorithm>
#include <cmath>
#include <atomic>
#include <chrono>
#include <cstdarg>
#include <cstring>
#include <memory>
#include <thread>

#include "common.h"
#include "handles.h"
#include "tables.h"

namespace ngap {

namespace {
thread_local std::string g_err;
}

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
}

const std::string& last_error() { return g_err; }

}  // namespace ngap

using namespace ngap;

extern "C" {

int ngap_last_error(char* buf, size_t n) {
  const std::string& e = last_error();
  if (buf && n > 0) {
    size_t k = std::min(n - 1, e.size());
    memcpy(buf, e.data(), k);
    buf[k] = '\0';
  }
  return (int)e.size();
}

const char* ngap_version(void) { return "ngap_b200 0.1.0 (sm_100a)"; }

int ngap_nfa_load_anml(const char* path, ngap_nfa** out) {
  if (!path || !out) {
    set_error("ngap_nfa_load_anml: null argument");
    return NGAP_E_INVALID;
  }
  *out = nullptr;
  std::unique_ptr<ngap_nfa> h(new ngap_nfa());
  int rc = load_anml_file(path, h->nfa);
  if (rc != NGAP_OK) return rc;
  *out = h.release();
  return NGAP_OK;
}

int ngap_nfa_parse_anml(const char* xml, size_t len, ngap_nfa** out) {
  if (!xml || !out) {
    set_error("ngap_nfa_parse_anml: null argument");
    return NGAP_E_INVALID;
  }
  *out = nullptr;
  std::unique_ptr<ngap_nfa> h(new ngap_nfa());
  int rc = parse_anml(xml, len, h->nfa);
  if (rc != NGAP_OK) return rc;
  *out = h.release();
  return NGAP_OK;
}

void ngap_nfa_destroy(ngap_nfa* nfa) { delete nfa; }

int64_t ngap_nfa_num_states(const ngap_nfa* nfa) { return nfa ? (int64_t)nfa->nfa.nodes.size() : -1; }

int64_t ngap_nfa_num_edges(const ngap_nfa* nfa) { return nfa ? nfa->nfa.num_edges() : -1; }

int ngap_groups_build(const ngap_nfa* nfa, const ngap_group_opts* opts, ngap_groups** out) {
  if (!nfa || !out) {
    set_error("ngap_groups_build: null argument");
    return NGAP_E_INVALID;
  }
  *out = nullptr;
  GroupOpts o;
  if (opts) {
    o.group_num = opts->group_num;
    o.max_nfa_size = opts->max_nfa_size;
    o.quit_degree = opts->quit_degree != 0;
    o.remove_degree = opts->remove_degree != 0;
  }
  std::unique_ptr<ngap_groups> h(new ngap_groups());
  int rc = build_groups(nfa->nfa, o, h->gs);
  if (rc != NGAP_OK) return rc;
  *out = h.release();
  return NGAP_OK;
}

int ngap_groups_count(const ngap_groups* g) { return g ? (int)g->gs.groups.size() : -1; }

int ngap_groups_cc_stats(const ngap_groups* g, int64_t* total, int64_t* failed, int64_t* too_big) {
  if (!g) return NGAP_E_INVALID;
  if (total) *total = g->gs.num_ccs_total;
  if (failed) *failed = g->gs.num_ccs_failed;
  if (too_big) *too_big = g->gs.num_ccs_too_big;
  return NGAP_OK;
}

int ngap_group_view_get(const ngap_groups* g, int group, ngap_group_view* out) {
  if (!g || !out || group < 0 || group >= (int)g->gs.groups.size()) {
    set_error("ngap_group_view_get: bad argument");
    return NGAP_E_INVALID;
  }
  const GroupGraph& gg = g->gs.groups[group];
  out->num_states = gg.V;
  out->num_edges = gg.E;
  out->num_aas = (int32_t)gg.aas.size();
  out->num_start = (int32_t)gg.starts.size();
  out->num_ccs = (int32_t)gg.cc_begin.size() - 1;
  out->row_offsets = gg.row_offsets.data();
  out->col_indices = gg.cols.data();
  out->symbol_sets = gg.bits.data();
  out->node_attrs = gg.attrs.data();
  out->always_active = gg.aas.data();
  out->start_states = gg.starts.data();
  out->cc_begin = gg.cc_begin.data();
  out->orig_node = gg.orig_node.data();
  return NGAP_OK;
}

void ngap_groups_destroy(ngap_groups* g) { delete g; }

namespace {

// The tiles ngap_tables_build would make, planned on the host.
int plan_tiles(const char* fn, const ngap_groups* g, const ngap_table_opts* opts,
               std::vector<TileHost>& tiles) {
  TableOpts to;
  const int rc = table_opts_from(opts, fn, to, nullptr);
  if (rc != NGAP_OK) return rc;
  return build_tiles(g->gs, to, tiles);
}

// [vb, ve) and [rb, re) of `key` in a prefix table, laid out as the matching
// kernel reads it (dense offsets by key, or linear-probing hash slots
// {key, list begin, report-list begin, list length << 16 | report length}).
// As the kernel's pt_find; `one` receives the lone state of an inline1 key
// (kNoSucc otherwise), whose list [vb, ve) is then empty.
void table_find(const PrefixTableHost& t, uint32_t key, uint32_t& vb, uint32_t& ve, uint32_t& rb,
                uint32_t& re, uint32_t& one) {
  vb = ve = rb = re = 0;
  one = kNoSucc;
  if (t.inline1) {
    const uint32_t x = t.voff[key];
    if (x == kHashEmpty) return;
    if (x >> 31) {
      vb = (x >> 6) & 0x1ffffffu;
      ve = vb + (x & 63u);
    } else {
      one = x;
    }
    return;
  }
  if (t.dense) {
    vb = t.voff[key];
    ve = t.voff[key + 1];
    if (!t.roff.empty()) {
      rb = t.roff[key];
      re = t.roff[key + 1];
    }
    return;
  }
  uint32_t h = prefix_hash(key) & t.hmask;
  for (uint32_t probe = 0; probe <= t.hmask; probe++) {
    const uint32_t* s = &t.slots[(size_t)h * 4];
    if (s[0] == key) {
      vb = s[1];
      ve = s[1] + (s[3] >> 16);
      rb = s[2];
      re = s[2] + (s[3] & 0xffffu);
      return;
    }
    if (s[0] == kHashEmpty) return;
    h = (h + 1) & t.hmask;
  }
}

}  // namespace

int ngap_features_host(const uint8_t* data, uint64_t bytes, const uint64_t* offsets,
                       const uint64_t* lengths, int n, int window, float* out) {
  if (n < 0 || (n > 0 && (!data || !offsets || !lengths || !out)) || window < 1) {
    set_error("ngap_features_host: bad argument");
    return NGAP_E_INVALID;
  }
  for (int i = 0; i < n; i++)
    if (offsets[i] > bytes || lengths[i] > bytes - offsets[i]) {  // no wrap-around
      set_error("ngap_features_host: region %d is out of range", i);
      return NGAP_E_INVALID;
    }
  for (int r = 0; r < n; r++) {
    const uint8_t* p = data + offsets[r];
    const uint64_t L = lengths[r];
    float* o = out + (size_t)r * NGAP_FEAT_BYTES;
    uint32_t hist[256] = {0};
    const uint64_t W = (uint64_t)window;
    const uint64_t nwin = L == 0 ? 0 : (L < W ? 1 : L / W);
    const uint64_t wl = L < W ? L : W;
    // H = log2(wl) - sum_b c_b log2(c_b) / wl, with c log2 c tabulated per window length
    thread_local std::vector<double> clogc;
    if (clogc.size() != wl + 1) {
      clogc.assign(wl + 1, 0.0);
      for (uint64_t c = 2; c <= wl; c++) clogc[c] = (double)c * std::log2((double)c);
    }
    const double lw = wl ? std::log2((double)wl) : 0.0;
    double sum = 0.0, mx = 0.0;
    for (uint64_t k = 0; k < nwin; k++) {
      // four interleaved counters per byte value: a run of equal bytes does
      // not chain every increment on the previous one
      uint32_t c4[4][256];
      std::memset(c4, 0, sizeof(c4));
      const uint8_t* q = p + k * W;
      uint64_t i = 0;
      for (; i + 4 <= wl; i += 4) {
        c4[0][q[i]]++;
        c4[1][q[i + 1]]++;
        c4[2][q[i + 2]]++;
        c4[3][q[i + 3]]++;
      }
      for (; i < wl; i++) c4[0][q[i]]++;
      double s = 0.0;
      for (int b = 0; b < 256; b++) {
        const uint32_t cb = c4[0][b] + c4[1][b] + c4[2][b] + c4[3][b];
        s += clogc[cb];
        hist[b] += cb;
      }
      const double h = std::max(0.0, lw - s / (double)wl);
      sum += h;
      mx = std::max(mx, h);
    }
    for (uint64_t i = nwin * wl; i < L; i++) hist[p[i]]++;  // bytes past the last window
    const double invL = L ? 1.0 / (double)L : 0.0;
    for (int b = 0; b < 256; b++) o[b] = (float)(hist[b] * invL);
    o[256] = nwin ? (float)(sum / (double)nwin / 8.0) : 0.f;
    o[257] = (float)(mx / 8.0);
  }
  return NGAP_OK;
}

int ngap_tiles_describe(const ngap_groups* g, const ngap_table_opts* opts, ngap_tile_desc* out,
                        int cap, int* n) {
  if (!g || !n || (cap > 0 && !out)) {
    set_error("ngap_tiles_describe: null argument");
    return NGAP_E_INVALID;
  }
  *n = 0;
  std::vector<TileHost> tiles;
  const int rc = plan_tiles("ngap_tiles_describe", g, opts, tiles);
  if (rc != NGAP_OK) return rc;
  *n = (int)tiles.size();
  for (int i = 0; i < std::min(cap, (int)tiles.size()); i++) {
    const TileHost& t = tiles[i];
    ngap_tile_desc d{};
    d.phase = t.phase;
    d.pair = t.pair;
    d.group = t.group;
    d.num_states = t.nstates;
    d.num_ccs = t.num_ccs;
    d.nact = t.nact;
    d.nsticky = t.nsticky;
    d.global = t.global ? 1 : 0;
    d.depth = t.depth;
    d.max_path = t.max_path;
    d.nlive = t.nlive;
    d.naas = (int32_t)t.aas.size();
    for (uint32_t a : t.act_local) d.shortcuts += __builtin_popcount(a >> 28);
    int64_t b = (int64_t)t.image.size();
    for (int k = 0; k < t.depth; k++) {
      const PrefixTableHost& p = t.pt[k];
      b += 4 * (int64_t)(p.voff.size() + p.roff.size() + p.slots.size() + p.vlist.size() +
                         p.rlist.size());
      if (p.dense) d.dense_levels |= 1 << k;
    }
    d.table_bytes = b;
    out[i] = d;
  }
  return NGAP_OK;
}

int ngap_tiles_lookup(const ngap_groups* g, const ngap_table_opts* opts, int tile,
                      const uint8_t* keys, int nkeys, int len, uint32_t* ids, int64_t* off,
                      uint32_t* reports, int64_t* roff, int64_t cap) {
  if (!g || nkeys < 0 || !off || !roff || (nkeys > 0 && !keys) || (cap > 0 && (!ids || !reports))) {
    set_error("ngap_tiles_lookup: null argument");
    return NGAP_E_INVALID;
  }
  std::vector<TileHost> tiles;
  const int rc = plan_tiles("ngap_tiles_lookup", g, opts, tiles);
  if (rc != NGAP_OK) return rc;
  if (tile < 0 || tile >= (int)tiles.size()) {
    set_error("ngap_tiles_lookup: tile %d of %d", tile, (int)tiles.size());
    return NGAP_E_INVALID;
  }
  const TileHost& t = tiles[tile];
  if (len < 1 || len > t.depth) {
    set_error("ngap_tiles_lookup: len must be in 1..%d (the tile's depth)", t.depth);
    return NGAP_E_INVALID;
  }
  const PrefixTableHost& pt = t.pt[len - 1];
  const uint32_t L = (uint32_t)t.nlive;
  int64_t nv = 0, nr = 0;
  off[0] = roff[0] = 0;
  for (int k = 0; k < nkeys; k++) {
    uint32_t key = 0, vb = 0, ve = 0, rb = 0, re = 0;
    bool dead = false;
    for (int i = 0; i < len; i++) {
      const uint32_t c = t.cls[keys[(size_t)k * len + i]];
      dead = dead || c >= L;  // a dead byte ends every path: no lookup
      key = key * L + c;
    }
    uint32_t one = kNoSucc;
    if (!dead) table_find(pt, key, vb, ve, rb, re, one);
    if (one != kNoSucc) {
      if (nv < cap) ids[nv] = t.sid[one];
      nv++;
    }
    for (uint32_t j = vb; j < ve; j++, nv++)
      if (nv < cap) ids[nv] = t.sid[pt.vlist[j]];
    for (uint32_t j = rb; j < re; j++, nr++)
      if (nr < cap) reports[nr] = t.sid[pt.rlist[j]];
    off[k + 1] = nv;
    roff[k + 1] = nr;
  }
  if (nv > cap || nr > cap) {
    set_error("ngap_tiles_lookup: %lld states and %lld reports, room for %lld", (long long)nv,
              (long long)nr, (long long)cap);
    return NGAP_E_INVALID;
  }
  return NGAP_OK;
}

// The reference validates with a CPU frontier simulation (ngap.cu:2171-2268)
// and a sort/unique comparison (ngap.cu:2270-2344). This checker does the same
// with a deduplicated frontier; it is used by the CLI's --validation only.
int64_t ngap_cpu_validate_reference(const ngap_groups* g, const uint8_t* input, int64_t num_seg,
                                    int64_t seg_len, int is_dup, uint64_t* out, int64_t cap,
                                    double* elapsed_ms) {
  if (!g || (!input && num_seg * seg_len > 0)) return -1;
  auto t0 = std::chrono::high_resolution_clock::now();
  const int ngroups = (int)g->gs.groups.size();
  const int64_t units = (int64_t)ngroups * num_seg;
  std::vector<std::vector<uint64_t>> per(units);
  unsigned nth = std::max(1u, std::thread::hardware_concurrency());
  std::vector<std::thread> pool;
  std::atomic<int64_t> next(0);
  auto worker = [&]() {
    std::vector<int32_t> cur, nxt;
    std::vector<uint8_t> mark;
    while (true) {
      int64_t u = next.fetch_add(1);
      if (u >= units) break;
      const int gi = (int)(u / num_seg);
      const int64_t seg = u % num_seg;
      const GroupGraph& gg = g->gs.groups[gi];
      mark.assign(gg.V, 0);
      cur.clear();
      if (seg == 0 || is_dup) cur.insert(cur.end(), gg.starts.begin(), gg.starts.end());
      cur.insert(cur.end(), gg.aas.begin(), gg.aas.end());
      std::sort(cur.begin(), cur.end());
      cur.erase(std::unique(cur.begin(), cur.end()), cur.end());
      const int64_t lo = seg * seg_len, hi = lo + seg_len;
      std::vector<uint64_t>& rep = per[u];
      for (int64_t it = lo; it < hi && !cur.empty(); it++) {
        const uint8_t s = input[it];
        nxt.clear();
        for (int32_t v : cur) {
          if (!((gg.bits[(size_t)v * 8 + (s >> 5)] >> (s & 31)) & 1u)) continue;
          if (gg.attrs[v] & 2) rep.push_back(((uint64_t)it << 32) | ((uint32_t)v | ((uint32_t)gi << 22)));
          for (int32_t e = gg.row_offsets[v]; e < gg.row_offsets[v + 1]; e++) {
            int32_t x = gg.cols[e];
            if (!mark[x]) {
              mark[x] = 1;
              nxt.push_back(x);
            }
          }
        }
        for (int32_t a : gg.aas)
          if (!mark[a]) {
            mark[a] = 1;
            nxt.push_back(a);
          }
        for (int32_t x : nxt) mark[x] = 0;
        cur.swap(nxt);
      }
    }
  };
  for (unsigned i = 0; i < nth; i++) pool.emplace_back(worker);
  for (auto& th : pool) th.join();
  std::vector<uint64_t> all;
  for (auto& v : per) all.insert(all.end(), v.begin(), v.end());
  std::sort(all.begin(), all.end());
  all.erase(std::unique(all.begin(), all.end()), all.end());
  auto t1 = std::chrono::high_resolution_clock::now();
  if (elapsed_ms) *elapsed_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  if ((int64_t)all.size() > cap) return -1;
  for (size_t i = 0; i < all.size(); i++) out[i] = (all[i] << 32) | (all[i] >> 32);
  return (int64_t)all.size();
}

}  // extern "C"
