// Non-blocking worklist matching kernel for sm_100a.
//
// Semantics (the same set of reports as the reference CPU matcher,
// code/src/ngap/ngap.cu:2171-2268, and as advanceAndFilterNonBlockingAllGroups,
// code/src/ngap/kernel_ngap_OA.cu:7-374): a worklist entry (v, q) means "state
// v matched input[q]". Expanding it tests each successor u against
// input[q + 1]; a match reports (sid(u) | group << 22, q + 1) when u is a
// report state and creates entry (u, q + 1). Always-active states enter at
// every position, either by scanning the always-active list (depth 0,
// kernel_ngap_OA.cu:227-241) or through the prefix tables: the table of depth
// k maps input[q .. q+k) to the states reached at q + k - 1 and, per depth, to
// the reports at q .. q+k-1 (ngap.cu:2358-2513, kernel_ngap_OA.cu:242-311).
//
// B200 organisation (not the reference's): one warp per unit (a tile of CCs
// over a range of positions), many warps per SM, no block-wide barrier in the
// hot loop. Per warp, in shared memory: a LIFO worklist of packed entries
// (state << 13 | offset in the window) pushed with ballot/popc aggregation and
// spilling to a per-warp global overflow stack; a double-buffered input window
// filled by cp.async.bulk (TMA 1-D copy, completion on an mbarrier, bounded
// wait); a report buffer flushed with one global atomic per flush. Entries that
// fall on the first position of the next window are carried over with exact
// deduplication through a per-warp bitmap.
#pragma once

#include <cstdint>

#include "device_types.h"

namespace ngap {

constexpr int kWarpsPerCta = 8;
constexpr int kCtaThreads = kWarpsPerCta * 32;
constexpr int kStackCap = 1024;   // entries per warp in shared memory
constexpr int kReportBuf = 64;    // reports per warp buffered in shared memory
constexpr int kInjectLow = 256;   // inject new positions while the stack holds fewer entries
constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kNoEntry = 0xffffffffu;  // never a valid entry: offsets stay < 8191

// Error flags written by the kernel (bit set => condition happened).
constexpr int kErrQueue = 1;      // overflow stack full: results incomplete
constexpr int kErrResults = 2;    // more reports than capacity
constexpr int kErrTimeout = 4;    // an mbarrier wait gave up
constexpr int kErrCarry = 8;      // carry buffer full

struct MatchParams {
  const TileDev* tiles;
  const UnitDev* units;
  int32_t nunits;
  const uint8_t* input;     // 16-byte aligned, readable up to round_up(len, 16)
  int32_t window;           // W <= kMaxWindow
  int32_t depth;            // 0: scan the AAS list; >= 1: tables up to min(depth, tile.depth)
  int32_t active_threshold; // privatize when more lanes than this expand
  int32_t unique;
  int32_t report_off;
  unsigned long long* rep_count;
  uint64_t* reports;        // key = offset << 32 | id
  uint64_t rep_cap;
  int* err;
  unsigned int* unit_counter;
  uint32_t* carry;          // [slots][carry_cap]
  uint32_t* marks;          // [slots][mark_words]
  uint32_t* ovf;            // [slots][ovf_cap]
  int32_t carry_cap, mark_words, ovf_cap;
  unsigned long long* work; // [0] entries expanded, [1] entries injected
};

__host__ __device__ inline int window_buf_bytes(int W) { return ((W + 48) + 15) & ~15; }

__host__ __device__ inline int warp_smem_bytes(int W) {
  return kStackCap * 4 + 2 * window_buf_bytes(W) + kReportBuf * 8 + 3 * 32 * 4 + 16;
}

struct WarpSmem {
  uint32_t* stack;           // kStackCap
  uint8_t* in[2];            // window buffers
  unsigned long long* rbuf;  // kReportBuf
  uint32_t* inj;             // 3 x 32 words of injection scratch
  uint64_t* bar;             // 2 mbarriers
};

// Per-warp state kept in registers (uniform across the warp).
struct WarpRun {
  int top;     // stack size
  int ovf_n;   // overflow stack size
  int ncarry;  // carry entries for the next window
  int nrep;    // buffered reports
  uint32_t* ovf;
  uint32_t* carry;
  uint32_t* marks;
};

// Everything a warp needs about its current unit and window.
struct UnitCtx {
  const TileDev* t;
  const uint8_t* in;  // window bytes: in[0] = input[wb]
  int64_t wb, hi, emit_lo;
  int wlen;
  uint32_t gbits;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// 1-D bulk copy global -> shared (no multicast), completion counted on the
// mbarrier. Source, destination and size are multiples of 16 bytes.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Bounded wait for the mbarrier phase with the given parity; false = gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (int it = 0; it < (1 << 24); it++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ bool accepts(const uint32_t* __restrict__ bits, uint32_t v, uint32_t s) {
  return (__ldg(bits + (size_t)v * 8 + (s >> 5)) >> (s & 31)) & 1u;
}

__device__ __forceinline__ bool is_report(const uint32_t* __restrict__ rep, uint32_t v) {
  return (__ldg(rep + (v >> 5)) >> (v & 31)) & 1u;
}

__device__ __forceinline__ unsigned lanemask_lt(int lane) { return (1u << lane) - 1u; }

__device__ __forceinline__ void flush_reports(const MatchParams& p, WarpSmem& ws, WarpRun& w, int lane) {
  if (w.nrep == 0) return;
  unsigned long long base = 0;
  if (lane == 0) base = atomicAdd(p.rep_count, (unsigned long long)w.nrep);
  base = __shfl_sync(kFull, base, 0);
  if (!p.report_off) {
    for (int i = lane; i < w.nrep; i += 32) {
      unsigned long long idx = base + (unsigned long long)i;
      if (idx < p.rep_cap) p.reports[idx] = ws.rbuf[i];
    }
    if (lane == 0 && base + (unsigned long long)w.nrep > p.rep_cap) atomicOr(p.err, kErrResults);
  }
  w.nrep = 0;
  __syncwarp();
}

// Warp-aggregated report emission: lanes with pred append (offset, id).
__device__ __forceinline__ void emit_report(const MatchParams& p, WarpSmem& ws, WarpRun& w, int lane,
                                            bool pred, uint32_t id, uint32_t off) {
  unsigned m = __ballot_sync(kFull, pred);
  if (m == 0) return;
  int cnt = __popc(m);
  if (w.nrep + cnt > kReportBuf) flush_reports(p, ws, w, lane);
  if (pred) ws.rbuf[w.nrep + __popc(m & lanemask_lt(lane))] = ((unsigned long long)off << 32) | id;
  w.nrep += cnt;
  __syncwarp();
}

// Stores entry e at stack index i, spilling past kStackCap to the overflow stack.
__device__ __forceinline__ void store_entry(const MatchParams& p, WarpSmem& ws, WarpRun& w, int i,
                                            uint32_t e) {
  if (i < kStackCap) {
    ws.stack[i] = e;
  } else {
    int j = w.ovf_n + (i - kStackCap);
    if (j < p.ovf_cap) w.ovf[j] = e;
    else atomicOr(p.err, kErrQueue);
  }
}

__device__ __forceinline__ void grow_stack(const MatchParams& p, WarpRun& w, int cnt) {
  int nt = w.top + cnt;
  if (nt > kStackCap) {
    w.ovf_n = min(w.ovf_n + (nt - kStackCap), p.ovf_cap);
    nt = kStackCap;
  }
  w.top = nt;
}

// Warp-aggregated push of one entry per predicated lane.
__device__ __forceinline__ void push_entry(const MatchParams& p, WarpSmem& ws, WarpRun& w, int lane,
                                           bool pred, uint32_t e) {
  unsigned m = __ballot_sync(kFull, pred);
  if (m == 0) return;
  if (pred) store_entry(p, ws, w, w.top + __popc(m & lanemask_lt(lane)), e);
  grow_stack(p, w, __popc(m));
  __syncwarp();
}

// Records a state matched at the next window's first position, once.
__device__ __forceinline__ void carry_state(const MatchParams& p, WarpRun& w, int lane, bool pred,
                                            uint32_t u) {
  bool fresh = false;
  if (pred) {
    uint32_t bit = 1u << (u & 31);
    fresh = !(atomicOr(w.marks + (u >> 5), bit) & bit);
  }
  unsigned m = __ballot_sync(kFull, fresh);
  if (m == 0) return;
  if (fresh) {
    int i = w.ncarry + __popc(m & lanemask_lt(lane));
    if (i < p.carry_cap) w.carry[i] = u;
    else atomicOr(p.err, kErrCarry);
  }
  w.ncarry = min(w.ncarry + __popc(m), p.carry_cap);
  __syncwarp();
}

// Looks up key in a prefix table; returns [b, e) of its state (or report) list.
__device__ __forceinline__ void pt_lookup(const PrefixTableDev& t, uint32_t key, bool reports,
                                          uint32_t& b, uint32_t& e) {
  const uint32_t* off = reports ? t.roff : t.voff;
  if (t.dense) {
    b = __ldg(off + key);
    e = __ldg(off + key + 1);
    return;
  }
  const uint32_t* keys = reports ? t.rkeys : t.keys;
  int lo = 0, hi = (reports ? t.nrkeys : t.nkeys) - 1;
  b = e = 0;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    uint32_t k = __ldg(keys + mid);
    if (k == key) {
      b = __ldg(off + mid);
      e = __ldg(off + mid + 1);
      return;
    }
    if (k < key) lo = mid + 1;
    else hi = mid - 1;
  }
}

// Handles a state u (bit 31 = report flag) that matched at window offset r,
// 1 <= r <= wlen: report it, then push it (r < wlen), carry it (r == wlen), or
// with privatization expand it in registers. Warp-collective: every lane
// calls it with the same LEVEL and privatize.
template <int LEVEL>
__device__ __forceinline__ void handle_match(const MatchParams& p, WarpSmem& ws, WarpRun& w,
                                             const UnitCtx& c, int lane, bool pred, uint32_t u,
                                             int r, bool privatize) {
  const int64_t q = c.wb + r;
  const bool rep = pred && (u >> 31) && q >= c.emit_lo;
  u &= 0x7fffffffu;
  emit_report(p, ws, w, lane, rep, rep ? (__ldg(c.t->sid + u) | c.gbits) : 0u, (uint32_t)q);
  const bool has_next = pred && q + 1 < c.hi;
  if (LEVEL > 0 && privatize) {
    const bool inner = has_next && r < c.wlen;
    carry_state(p, w, lane, has_next && !inner, u);
    uint4 sc = make_uint4(kNoSucc, kNoSucc, kNoSucc, kNoSucc);
    uint32_t s = 0;
    if (inner) {
      sc = __ldg(c.t->succ + u);
      s = c.in[r + 1];
    }
    const uint32_t cs[4] = {sc.x, sc.y, sc.z, sc.w};
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const bool ok = inner && cs[j] != kNoSucc && accepts(c.t->bits, cs[j] & 0x7fffffffu, s);
      handle_match<(LEVEL > 0 ? LEVEL - 1 : 0)>(p, ws, w, c, lane, ok, cs[j], r + 1, privatize);
    }
    return;
  }
  carry_state(p, w, lane, has_next && r == c.wlen, u);
  push_entry(p, ws, w, lane, has_next && r < c.wlen, (u << kEntryPosBits) | (uint32_t)r);
}

// Always-active states for window offsets [r0, r0 + 32) (one per lane).
__device__ __forceinline__ void inject(const MatchParams& p, WarpSmem& ws, WarpRun& w,
                                       const UnitCtx& c, int lane, int r0, int depth,
                                       unsigned long long& n_injected) {
  const TileDev& t = *c.t;
  const int r = r0 + lane;
  const bool valid = r < c.wlen;
  const int64_t q = c.wb + r;
  if (depth == 0) {  // scan the always-active list
    const uint32_t s = valid ? c.in[r] : 0u;
    for (int i = 0; i < t.naas; i++) {
      const uint32_t a = __ldg(t.aas + i);
      const bool ok = valid && accepts(t.bits, a, s);
      const bool rep = ok && is_report(t.rep, a) && q >= c.emit_lo;
      emit_report(p, ws, w, lane, rep, rep ? (__ldg(t.sid + a) | c.gbits) : 0u, (uint32_t)q);
      push_entry(p, ws, w, lane, ok && q + 1 < c.hi, (a << kEntryPosBits) | (uint32_t)r);
      n_injected += ok;
    }
    return;
  }
  // table depth clamped at the window end: states land at q + k - 1 < window end
  const int k = valid ? min(depth, c.wlen - r) : 0;
  uint32_t key = 0, vb = 0, ve = 0;
  for (int d = 0; d < depth; d++) {
    const bool act = d < k;
    if (act) key = (key << 8) | c.in[r + d];
    uint32_t rb = 0, re = 0;
    if (act) pt_lookup(t.pt[d], key, true, rb, re);
    const int len = (int)(re - rb);
    const int mx = __reduce_max_sync(kFull, len);
    for (int i = 0; i < mx; i++) {
      const bool ok = i < len && q + d >= c.emit_lo;
      const uint32_t v = ok ? __ldg(t.pt[d].rlist + rb + i) : 0u;
      emit_report(p, ws, w, lane, ok, ok ? (__ldg(t.sid + v) | c.gbits) : 0u, (uint32_t)(q + d));
    }
    if (act && d == k - 1) pt_lookup(t.pt[d], key, false, vb, ve);
  }
  // entries at the unit's last position have nothing to expand
  const uint32_t len = (k > 0 && q + k < c.hi) ? (ve - vb) : 0u;
  n_injected += len;
  uint32_t incl = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  if (total == 0) return;
  ws.inj[lane] = incl;
  ws.inj[32 + lane] = vb;
  ws.inj[64 + lane] = (uint32_t)(k > 0 ? k : 1);
  __syncwarp();
  // cooperative copy of all lanes' lists onto the stack
  for (uint32_t idx = lane; idx < total; idx += 32) {
    int l0 = 0, l1 = 31;
    while (l0 < l1) {  // first lane whose inclusive prefix exceeds idx
      const int m = (l0 + l1) >> 1;
      if (ws.inj[m] > idx) l1 = m;
      else l0 = m + 1;
    }
    const uint32_t before = l0 > 0 ? ws.inj[l0 - 1] : 0u;
    const int kk = (int)ws.inj[64 + l0];
    const uint32_t v = __ldg(t.pt[kk - 1].vlist + ws.inj[32 + l0] + (idx - before));
    store_entry(p, ws, w, w.top + (int)idx, (v << kEntryPosBits) | (uint32_t)(r0 + l0 + kk - 1));
  }
  grow_stack(p, w, (int)total);
  __syncwarp();
}

template <int PRIV>
__global__ void __launch_bounds__(kCtaThreads) match_kernel(MatchParams p) {
  extern __shared__ __align__(128) uint8_t smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int W = p.window;
  uint8_t* base = smem_raw + (size_t)warp * warp_smem_bytes(W);
  WarpSmem ws;
  ws.stack = reinterpret_cast<uint32_t*>(base);
  ws.in[0] = base + kStackCap * 4;
  ws.in[1] = ws.in[0] + window_buf_bytes(W);
  ws.rbuf = reinterpret_cast<unsigned long long*>(ws.in[1] + window_buf_bytes(W));
  ws.inj = reinterpret_cast<uint32_t*>(ws.rbuf + kReportBuf);
  ws.bar = reinterpret_cast<uint64_t*>(ws.inj + 3 * 32);
  const int slot = blockIdx.x * kWarpsPerCta + warp;
  WarpRun w;
  w.top = w.ovf_n = w.ncarry = w.nrep = 0;
  w.ovf = p.ovf + (size_t)slot * p.ovf_cap;
  w.carry = p.carry + (size_t)slot * p.carry_cap;
  w.marks = p.marks + (size_t)slot * p.mark_words;
  if (lane == 0) {
    mbar_init(&ws.bar[0], 1);
    mbar_init(&ws.bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  uint32_t phase[2] = {0u, 0u};
  bool pending[2] = {false, false};
  bool dead = false;
  unsigned long long n_expanded = 0, n_injected = 0;

  auto issue = [&](int buf, int64_t wb, int64_t hi) {
    const int64_t we = min(wb + (int64_t)W, hi);
    const int64_t end = min(we + 1, hi);  // window bytes plus one look-ahead byte
    const int64_t a0 = wb & ~(int64_t)15;
    const uint32_t bytes = (uint32_t)(((end - a0) + 15) & ~(int64_t)15);
    if (lane == 0) {
      mbar_expect_tx(&ws.bar[buf], bytes);
      bulk_g2s(ws.in[buf], p.input + a0, bytes, &ws.bar[buf]);
    }
    pending[buf] = true;
  };

  while (!dead) {
    unsigned uid = 0;
    if (lane == 0) uid = atomicAdd(p.unit_counter, 1u);
    uid = __shfl_sync(kFull, uid, 0);
    if (uid >= (unsigned)p.nunits) break;
    const UnitDev un = p.units[uid];
    UnitCtx c;
    c.t = &p.tiles[un.tile];
    c.hi = un.hi;
    c.emit_lo = un.emit_lo;
    c.gbits = (uint32_t)c.t->group << 22;
    const int depth = p.depth == 0 ? 0 : min(p.depth, c.t->depth);
    int cur = 0;
    issue(0, un.lo, c.hi);
    for (int64_t wb = un.lo; wb < c.hi; wb += W) {
      const int64_t we = min(wb + (int64_t)W, c.hi);
      c.wb = wb;
      c.wlen = (int)(we - wb);
      if (!mbar_wait(&ws.bar[cur], phase[cur])) {
        if (lane == 0) atomicOr(p.err, kErrTimeout);
        dead = true;
        break;
      }
      phase[cur] ^= 1u;
      pending[cur] = false;
      if (we < c.hi) issue(cur ^ 1, we, c.hi);
      c.in = ws.in[cur] + (wb & 15);
      __syncwarp();
      // carried states: matched at wb
      w.top = 0;
      if (w.ncarry > 0) {
        for (int i = lane; i < w.ncarry; i += 32) {
          const uint32_t u = w.carry[i];
          w.marks[u >> 5] = 0u;
          store_entry(p, ws, w, i, u << kEntryPosBits);
        }
        const int n = w.ncarry;
        w.ncarry = 0;
        grow_stack(p, w, n);
        __syncwarp();
      }
      // start-of-data states at the unit's first position (ngap_buffer.cu:613-631)
      if (wb == un.lo && (un.flags & 1u)) {
        const uint32_t s0 = c.in[0];
        for (int i0 = 0; i0 < c.t->nstart; i0 += 32) {
          const int i = i0 + lane;
          const uint32_t v = i < c.t->nstart ? __ldg(c.t->start + i) : 0u;
          const bool ok = i < c.t->nstart && accepts(c.t->bits, v, s0);
          const bool rep = ok && is_report(c.t->rep, v) && un.lo >= c.emit_lo;
          emit_report(p, ws, w, lane, rep, rep ? (__ldg(c.t->sid + v) | c.gbits) : 0u,
                      (uint32_t)un.lo);
          push_entry(p, ws, w, lane, ok && un.lo + 1 < c.hi, v << kEntryPosBits);
        }
      }
      int cursor = 0;  // next window offset to inject
      while (true) {
        if (w.top < kInjectLow && cursor < c.wlen) {
          inject(p, ws, w, c, lane, cursor, depth, n_injected);
          cursor += 32;
          continue;
        }
        if (w.top == 0) {
          if (w.ovf_n > 0) {  // refill from the overflow stack
            const int m = min(w.ovf_n, kStackCap);
            for (int i = lane; i < m; i += 32) ws.stack[i] = w.ovf[w.ovf_n - m + i];
            w.ovf_n -= m;
            w.top = m;
            __syncwarp();
            continue;
          }
          if (cursor < c.wlen) continue;
          break;
        }
        // expand up to 32 entries from the top of the stack
        const int n = min(w.top, 32);
        const bool has = lane < n;
        uint32_t e = has ? ws.stack[w.top - 1 - lane] : kNoEntry;
        w.top -= n;
        __syncwarp();
        if (p.unique) {  // identical entries in one step are expanded once (--unique)
          const unsigned peers = __match_any_sync(kFull, e);
          if ((__ffs(peers) - 1) != lane) e = kNoEntry;
        }
        const uint32_t v = e >> kEntryPosBits;
        const int r = (int)(e & ((1u << kEntryPosBits) - 1));
        const bool go = e != kNoEntry && c.wb + r + 1 < c.hi;
        uint4 sc = make_uint4(kNoSucc, kNoSucc, kNoSucc, kNoSucc);
        uint32_t s = 0;
        if (go) {
          sc = __ldg(c.t->succ + v);
          s = c.in[r + 1];
        }
        n_expanded += go;
        const bool privatize = PRIV > 0 && __popc(__ballot_sync(kFull, go)) > p.active_threshold;
        const uint32_t cs[4] = {sc.x, sc.y, sc.z, sc.w};
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const bool ok = go && cs[j] != kNoSucc && accepts(c.t->bits, cs[j] & 0x7fffffffu, s);
          handle_match<PRIV>(p, ws, w, c, lane, ok, cs[j], r + 1, privatize);
        }
      }
      cur ^= 1;
    }
    if (dead) {
      for (int i = lane; i < w.ncarry; i += 32) w.marks[w.carry[i] >> 5] = 0u;
      w.ncarry = w.top = w.ovf_n = 0;
      // wait (bounded) for any copy still in flight before leaving
      for (int b = 0; b < 2; b++)
        if (pending[b]) {
          mbar_wait(&ws.bar[b], phase[b]);
          pending[b] = false;
        }
      __syncwarp();
    }
  }
  flush_reports(p, ws, w, lane);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    n_expanded += __shfl_xor_sync(kFull, n_expanded, o);
    n_injected += __shfl_xor_sync(kFull, n_injected, o);
  }
  if (lane == 0) {
    atomicAdd(&p.work[0], n_expanded);
    atomicAdd(&p.work[1], n_injected);
  }
}

}  // namespace ngap
