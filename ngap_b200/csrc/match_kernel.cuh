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
// k maps the next k input symbols to the states reached at q + k - 1 and, per
// depth, to the reports at q .. q+k-1 (ngap.cu:2358-2513,
// kernel_ngap_OA.cu:242-311).
//
// B200 organisation (not the reference's):
//  * a CTA takes a task (a tile and a range of its units) and stages the
//    tile's table image (successors, byte-class masks, report bits, byte ->
//    class map) into shared memory once; its warps (kWarpsPerCta) then take units of that
//    task, one warp per unit, with no block-wide barrier in the hot loop;
//  * per warp, in shared memory: a LIFO worklist of packed entries
//    (state << 13 | offset in the window); one expansion step pops up to 32
//    entries, evaluates all their successors, and pushes the survivors with a
//    single bit-sliced ballot prefix sum; entries past the shared capacity
//    spill to a per-warp global overflow stack;
//  * input windows are fetched by cp.async.bulk (1-D TMA, completion on an
//    mbarrier, bounded wait), double-buffered, and translated to class ids in
//    place;
//  * reports go through a per-warp shared buffer flushed with one global atomic;
//    states that land on the next window's first position are carried over
//    with exact deduplication through a per-warp bitmap.
#pragma once

#include <cstdint>

#include "device_types.h"

namespace ngap {

constexpr int kWarpsPerCta = 20;
constexpr int kCtaThreads = kWarpsPerCta * 32;
constexpr int kStackCap = 512;    // entries per warp in shared memory
constexpr int kReportBuf = 64;    // reports per warp buffered in shared memory
constexpr int kInjectLow = 256;   // inject new positions while the stack holds fewer entries
constexpr int kStickyCap = 64;    // sticky states tracked per warp (more fall back to entries)
constexpr int kPendCap = 16;      // sticky states met while copying one injection batch
constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kNoEntry = 0xffffffffu;  // never a valid entry: offsets stay < 8191
constexpr uint32_t kIdMask = 0x7fffffffu;

// Error flags written by the kernel (bit set => condition happened).
constexpr int kErrQueue = 1;      // overflow stack full: results incomplete
constexpr int kErrResults = 2;    // more reports than capacity
constexpr int kErrTimeout = 4;    // an mbarrier wait gave up
constexpr int kErrCarry = 8;      // carry buffer full

struct MatchParams {
  const TileDev* tiles;
  const UnitDev* units;
  const TaskDev* tasks;
  int32_t ntasks;
  int32_t image_region;     // shared-memory bytes reserved for a tile image
  const uint8_t* input;     // 16-byte aligned, readable up to round_up(len, 16)
  int32_t window;           // W <= kMaxWindow
  int32_t depth;            // 0: scan the AAS list; >= 1: tables up to min(depth, tile.depth)
  int32_t active_threshold; // privatize when more lanes than this expand
  int32_t unique;
  int32_t report_off;
  int32_t off_shift;        // bit position of the offset in report keys (32 when not batched)
  unsigned long long* rep_count;
  uint64_t* reports;        // key = offset << 32 | id
  uint64_t rep_cap;
  int* err;
  unsigned int* task_counter;
  uint32_t* carry;          // [slots][carry_cap]
  uint32_t* marks;          // [slots][mark_words]
  uint32_t* ovf;            // [slots][ovf_cap]
  int32_t carry_cap, mark_words, ovf_cap;
  unsigned long long* work; // [0] entries expanded, [1] entries injected
  uint32_t* act;            // activation slots (first match of sticky states, offset in the
                            // segment; 0xffffffff = none)
  const uint32_t* act_list; // per row (segment of a pair): the slots that have a first match,
  const uint32_t* act_cnt;  // at the row's offset, and their count
  uint32_t* stk_g;          // [slots][2][stk_g_cap]: sticky lists of layered units beyond
  int32_t stk_g_cap;        // kStickyCap
  unsigned long long* unit_work;  // [units]: entries expanded + injected per unit (tracing), or null
  unsigned long long* unit_cycles;  // [units]: SM clock cycles per unit (tracing), or null
  int32_t free_begin;       // units [free_begin, free_begin + nfree) are taken warp by warp
  int32_t nfree;
  int32_t free_tile;        // the one tile of all free units (descriptors staged per CTA), or -1
  unsigned int* free_cursor;  // next free unit (zeroed before the launch)
  int32_t wait_rounds;      // try_wait rounds before an mbarrier wait gives up
  int32_t skip_copy_unit;   // test hook: this unit's first window copy is not issued (-1: none),
                            // so its wait runs out and the launch reports kErrTimeout
};

constexpr int32_t kWaitRounds = 1 << 24;  // default bound of an mbarrier wait

constexpr uint32_t kNoAct = 0xffffffffu;

// A window buffer: up to kMaxDepth - 1 look-behind bytes, 15 bytes of
// alignment, W window bytes and one look-ahead byte.
__host__ __device__ inline int window_buf_bytes(int W) { return ((W + 48) + 15) & ~15; }
static_assert(kMaxDepth - 1 + 15 + 1 + 15 <= 48, "window buffer slack");

__host__ __device__ inline int warp_smem_bytes(int W) {
  return kStackCap * 4 + 2 * window_buf_bytes(W) + kReportBuf * 8 + 3 * 32 * 4 + 16 +
         kStickyCap * 8 + kPendCap * 8 + 16;
}

__host__ __device__ inline int cta_smem_bytes(int W, int image_region) {
  return image_region + kWarpsPerCta * warp_smem_bytes(W);
}

struct WarpSmem {
  uint32_t* stack;           // kStackCap
  uint8_t* in[2];            // window buffers
  unsigned long long* rbuf;  // kReportBuf
  uint32_t* inj;             // 3 x 32 words of injection scratch
  uint64_t* bar;             // 2 mbarriers
  uint32_t* stk_s;           // kStickyCap sticky states active in the unit
  uint32_t* stk_q;           //   and the position of their first match (low 32 bits)
  uint32_t* pend_s;          // kPendCap sticky states met while copying a batch
  uint32_t* pend_q;
  uint32_t* pend_n;          // count (one word)
};

// Per-warp state kept in registers (uniform across the warp).
struct WarpRun {
  int top;     // stack size
  int ovf_n;   // overflow stack size
  int ncarry;  // carry entries for the next window
  int nrep;    // buffered reports
  int nstk;    // sticky states active in the unit
  uint32_t base;                // current unit's stream start (low 32 bits of positions)
  unsigned long long key_hi;    // current unit's stream index in the report key
  uint32_t* ovf;
  uint32_t* carry;
  uint32_t* marks;
  uint32_t* act;   // activation units: the segment's slots (reports become atomicMin)
  int stk_cap;     // capacity of the sticky list (ws.stk_s / stk_q)
  bool stk_rep;    // layered units: some registered sticky state is a report state
};

// The tile a warp works on: hot tables in shared memory (or global memory
// when the image does not fit) and the cold ones in global memory.
struct TileView {
  const uint4* succ;    // wide tiles
  const uint32_t* cmask;
  const uint32_t* rep;
  const uint32_t* sticky;  // sticky-state bitmap, nullptr when the tile has none
  const uint8_t* cls;
  const TileDev* t;
  const PrefixTableDev* pt;  // the tile's prefix tables (shared-memory copy)
  int cw;
  int narrow;
  int fused;       // records of 2 x uint4: successors, then their class masks
  uint32_t nlive;  // live classes: base of the prefix-table keys
  uint32_t rep_levels;  // bit d: the depth-(d+1) table has report lists
};

// Successors of v in the 32-bit convention (bit 31 = report, kNoSucc = none).
__device__ __forceinline__ uint4 load_succ(const TileView& tv, uint32_t v) {
  if (!tv.narrow) return tv.succ[(size_t)v << tv.fused];
  const uint2 x = reinterpret_cast<const uint2*>(tv.succ)[v];  // narrow tiles: 4 x u16
  auto wide = [](uint32_t h) {
    return h == 0xffffu ? kNoSucc : ((h & 0x7fffu) | ((h & 0x8000u) << 16));
  };
  return make_uint4(wide(x.x & 0xffffu), wide(x.x >> 16), wide(x.y & 0xffffu), wide(x.y >> 16));
}

// Fused tiles: the class masks of v's four successors (0 where none), the
// second half of v's 32-byte record.
__device__ __forceinline__ uint4 load_smask(const TileView& tv, uint32_t v) {
  return tv.succ[((size_t)v << 1) + 1];
}

// Successor j of a state accepts class c: from the record's masks (fused
// tiles) or from the successor's own class mask.
__device__ __forceinline__ bool succ_accepts(const TileView& tv, uint32_t u, uint32_t m, uint32_t c);

// Everything about the current unit and window.
struct UnitCtx {
  const uint8_t* in;  // window symbols (class ids): in[0] = symbol at wb; in[-1 .. -(kMaxDepth-1)]
                      // hold the look-behind bytes when the window is not the unit's first
  int64_t wb, hi, emit_lo;
  int wlen;
  int iend;           // always-active injection covers window offsets below iend
  int lim;            // hi - wb, capped: a window offset r has a next symbol when r + 1 < lim
  int elo;            // emit_lo - wb, clamped: reports at window offsets >= elo are kept
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

// Bounded wait for the mbarrier phase with the given parity: at most `rounds`
// try_wait rounds; false = gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int32_t rounds) {
  for (int32_t it = 0; it < rounds; it++) {
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

__device__ __forceinline__ bool accepts(const TileView& tv, uint32_t v, uint32_t c) {
  return (tv.cmask[(size_t)v * tv.cw + (c >> 5)] >> (c & 31)) & 1u;
}

__device__ __forceinline__ bool succ_accepts(const TileView& tv, uint32_t u, uint32_t m, uint32_t c) {
  if (tv.fused) return (m >> c) & 1u;  // m = 0 when there is no successor
  return u != kNoSucc && accepts(tv, u & kIdMask, c);
}

__device__ __forceinline__ bool is_report(const TileView& tv, uint32_t v) {
  return (tv.rep[v >> 5] >> (v & 31)) & 1u;
}

__device__ __forceinline__ unsigned lanemask_lt(int lane) { return (1u << lane) - 1u; }

// Exclusive prefix sum over the warp of counts < 2^B, one ballot per bit.
template <int B>
__device__ __forceinline__ int warp_excl(int cnt, int lane, int& total) {
  int ex = 0;
  total = 0;
#pragma unroll
  for (int b = 0; b < B; b++) {
    const unsigned m = __ballot_sync(kFull, (cnt >> b) & 1);
    ex += __popc(m & lanemask_lt(lane)) << b;
    total += __popc(m) << b;
  }
  return ex;
}

__device__ __forceinline__ void flush_reports(const MatchParams& p, WarpSmem& ws, WarpRun& w, int lane) {
  if (w.nrep == 0) return;
  unsigned long long base = 0;
  if (lane == 0) base = atomicAdd(p.rep_count, (unsigned long long)w.nrep);
  base = __shfl_sync(kFull, base, 0);
  if (!p.report_off) {
    for (int i = lane; i < w.nrep; i += 32) {
      const unsigned long long idx = base + (unsigned long long)i;
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
  if (w.act) {  // activation pass: id is the sticky state's slot
    if (pred) atomicMin(w.act + id, off - w.base);
    return;
  }
  const unsigned m = __ballot_sync(kFull, pred);
  if (m == 0) return;
  const int cnt = __popc(m);
  if (w.nrep + cnt > kReportBuf) flush_reports(p, ws, w, lane);
  if (pred)
    ws.rbuf[w.nrep + __popc(m & lanemask_lt(lane))] =
        w.key_hi | ((unsigned long long)(off - w.base) << p.off_shift) | id;
  w.nrep += cnt;
  __syncwarp();
}

// Stores entry e at stack index i, spilling past kStackCap to the overflow stack.
__device__ __forceinline__ void store_entry(const MatchParams& p, WarpSmem& ws, WarpRun& w, int i,
                                            uint32_t e) {
  if (i < kStackCap) {
    ws.stack[i] = e;
  } else {
    const int j = w.ovf_n + (i - kStackCap);
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
  const unsigned m = __ballot_sync(kFull, pred);
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
    const uint32_t bit = 1u << (u & 31);
    fresh = !(atomicOr(w.marks + (u >> 5), bit) & bit);
  }
  const unsigned m = __ballot_sync(kFull, fresh);
  if (m == 0) return;
  if (fresh) {
    const int i = w.ncarry + __popc(m & lanemask_lt(lane));
    if (i < p.carry_cap) w.carry[i] = u;
    else atomicOr(p.err, kErrCarry);
  }
  w.ncarry = min(w.ncarry + __popc(m), p.carry_cap);
  __syncwarp();
}

// Looks up key in a prefix table: [vb, ve) of its state list when want_v and
// [rb, re) of its report list when want_r; empty ranges when absent. A
// single-word (inline1) table gives a list of one in `one` (kNoEntry when the
// list is empty or longer; [vb, ve) is then empty or the longer list).
__device__ __forceinline__ void pt_find(const PrefixTableDev& t, uint32_t key, bool want_v,
                                        bool want_r, uint32_t& vb, uint32_t& ve, uint32_t& rb,
                                        uint32_t& re, uint32_t& one) {
  vb = ve = rb = re = 0;
  one = kNoEntry;
  if (!want_v && !want_r) return;
  if (t.inline1) {  // no report lists in these tables
    if (want_v) {
      const uint32_t x = __ldg(t.voff + key);
      if (x != kHashEmpty) {
        if (x >> 31) {
          vb = (x >> 6) & 0x1ffffffu;
          ve = vb + (x & 63u);
        } else {
          one = x;
        }
      }
    }
    return;
  }
  if (t.dense) {
    if (want_v) {
      vb = __ldg(t.voff + key);
      ve = __ldg(t.voff + key + 1);
    }
    if (want_r) {
      rb = __ldg(t.roff + key);
      re = __ldg(t.roff + key + 1);
    }
    return;
  }
  uint32_t h = prefix_hash(key) & t.hmask;
  for (uint32_t probe = 0; probe <= t.hmask; probe++) {  // at least half the slots are empty
    const uint4 s = __ldg(t.slots + h);
    if (s.x == key) {
      vb = s.y;
      ve = s.y + (s.w >> 16);
      rb = s.z;
      re = s.z + (s.w & 0xffffu);
      return;
    }
    if (s.x == kHashEmpty) return;
    h = (h + 1) & t.hmask;
  }
}

// Reports (slow path, taken only when some lane has one) for up to 4 matched
// states u[j] (bit 31 = report flag) at stream position q.
__device__ __forceinline__ void report4(const MatchParams& p, WarpSmem& ws, WarpRun& w,
                                        const TileView& tv, int lane, const bool ok[4],
                                        const uint32_t u[4], int64_t q, bool in_range) {
  bool any = false;
#pragma unroll
  for (int j = 0; j < 4; j++) any |= ok[j] && (u[j] >> 31);
  if (!__any_sync(kFull, any && in_range)) return;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const bool rep = in_range && ok[j] && (u[j] >> 31);
    emit_report(p, ws, w, lane, rep, rep ? (__ldg(tv.t->sid + (u[j] & kIdMask))) : 0u,
                (uint32_t)q);
  }
}

// ---- sticky states ----------------------------------------------------------
// A sticky state (not always-active, a self-loop, every byte accepted) that
// matches at position q matches again at every later position of the segment,
// so from q on it acts like an always-active state. Instead of a chain of
// worklist entries advancing one position per step, a warp keeps the unit's
// active sticky states in a small shared list with their first match; the
// injection of each position adds their work, and a state registered late
// catches up the positions already injected.

__device__ __forceinline__ bool is_sticky(const TileView& tv, uint32_t v) {
  return (tv.sticky[v >> 5] >> (v & 31)) & 1u;
}

// Work of active sticky state s at stream position t (act: s matched at t - 1):
// its own report at t, and its other successors tested against the symbol at
// t. Warp-collective.
__device__ __forceinline__ void sticky_at(const MatchParams& p, WarpSmem& ws, WarpRun& w,
                                          const TileView& tv, const UnitCtx& c, int lane,
                                          uint32_t s, const uint32_t us[4], bool srep, bool act,
                                          int64_t t) {
  const int r = (int)(t - c.wb);
  const uint32_t sym = act ? c.in[r] : 0u;
  const bool rs = act && srep && t >= c.emit_lo;
  emit_report(p, ws, w, lane, rs, rs ? __ldg(tv.t->sid + s) : 0u, (uint32_t)t);
  bool ok[4];
#pragma unroll
  for (int j = 0; j < 4; j++)
    ok[j] = act && us[j] != kNoSucc && (us[j] & kIdMask) != s && accepts(tv, us[j] & kIdMask, sym);
  report4(p, ws, w, tv, lane, ok, us, t, t >= c.emit_lo);
  const bool need = act && t + 1 < c.hi;
#pragma unroll
  for (int j = 0; j < 4; j++)
    push_entry(p, ws, w, lane, need && ok[j], ((us[j] & kIdMask) << kEntryPosBits) | (uint32_t)r);
}

// Sticky state s's work over positions [t0, t1), lanes over positions.
__device__ __forceinline__ void sticky_span(const MatchParams& p, WarpSmem& ws, WarpRun& w,
                                         const TileView& tv, const UnitCtx& c, int lane, uint32_t s,
                                         int64_t t0, int64_t t1) {
  const uint4 sc = load_succ(tv, s);
  const uint32_t us[4] = {sc.x, sc.y, sc.z, sc.w};
  const bool srep = is_report(tv, s);
  for (int64_t tb = t0; tb < t1; tb += 32) {
    const int64_t t = tb + lane;
    sticky_at(p, ws, w, tv, c, lane, s, us, srep, t < t1, t);
  }
}

// Warp-uniform: sticky state s matched at q. Positions below inj_end have been
// injected already and are caught up here; later ones are handled by
// injection. Returns false when the list is full (the caller keeps an entry).
__device__ __forceinline__ bool register_sticky(const MatchParams& p, WarpSmem& ws, WarpRun& w,
                                             const TileView& tv, const UnitCtx& c, int lane,
                                             uint32_t s, int64_t q, int64_t inj_end) {
  int found = -1;
  for (int i0 = 0; i0 < w.nstk && found < 0; i0 += 32) {
    const int i = i0 + lane;
    const unsigned m = __ballot_sync(kFull, i < w.nstk && ws.stk_s[i] == s);
    if (m) found = i0 + __ffs(m) - 1;
  }
  int64_t t1;
  if (found >= 0) {
    const int64_t old = (int64_t)ws.stk_q[found];
    if (q >= old) return true;  // already active from an earlier position
    t1 = min(old + 1, inj_end);
    __syncwarp();
    if (lane == 0) ws.stk_q[found] = (uint32_t)q;
  } else {
    if (w.nstk >= w.stk_cap) return false;
    if (lane == 0) {
      ws.stk_s[w.nstk] = s;
      ws.stk_q[w.nstk] = (uint32_t)q;
    }
    w.nstk++;
    t1 = inj_end;
  }
  __syncwarp();
  t1 = min(t1, c.hi);
  if (q + 1 < t1) sticky_span(p, ws, w, tv, c, lane, s, q + 1, t1);
  return true;
}

// Registers the sticky states of all predicated lanes; true on lanes whose
// state was registered (those need no worklist entry).
__device__ __forceinline__ bool register_each(const MatchParams& p, WarpSmem& ws, WarpRun& w,
                                              const TileView& tv, const UnitCtx& c, int lane,
                                              bool pred, uint32_t s, int64_t q, int64_t inj_end) {
  unsigned m = __ballot_sync(kFull, pred);
  bool mine = false;
  while (m) {
    const int src = __ffs(m) - 1;
    m &= m - 1;
    const uint32_t ss = __shfl_sync(kFull, s, src);
    const long long qq = __shfl_sync(kFull, (long long)q, src);
    const bool ok = register_sticky(p, ws, w, tv, c, lane, ss, (int64_t)qq, inj_end);
    if (lane == src) mine = ok;
  }
  return mine;
}

// Always-active states for window offsets [r0, r0 + batch) (one per lane).
__device__ __forceinline__ void inject_aas(const MatchParams& p, WarpSmem& ws, WarpRun& w,
                                           const TileView& tv, const UnitCtx& c, int lane, int r0,
                                           int batch, int depth, unsigned long long& n_injected) {
  const TileDev& t = *tv.t;
  const int r = r0 + lane;
  const bool valid = lane < batch && r < c.iend;
  const int64_t q = c.wb + r;
  if (depth == 0) {  // scan the always-active list
    const uint32_t s = valid ? c.in[r] : 0u;
    for (int i = 0; i < t.naas; i++) {
      const uint32_t a = __ldg(t.aas + i);
      const bool ok = valid && accepts(tv, a, s);
      const bool rep = ok && is_report(tv, a) && q >= c.emit_lo;
      emit_report(p, ws, w, lane, rep, rep ? (__ldg(t.sid + a)) : 0u, (uint32_t)q);
      push_entry(p, ws, w, lane, ok && q + 1 < c.hi, (a << kEntryPosBits) | (uint32_t)r);
      n_injected += ok;
    }
    return;
  }
  // table depth clamped at the window end: states land at q + k - 1 < window end;
  // a dead-class symbol at offset d ends every path, so only reports of the
  // first d symbols remain and no state needs expanding
  const int kmax = valid ? min(depth, c.wlen - r) : 0;
  int k = kmax;
  uint32_t key = 0;  // live classes of the next k symbols, base nlive
  for (int d = 0; d < depth; d++) {
    if (d < k) {
      const uint32_t sym = c.in[r + d];
      if (sym >= tv.nlive) k = d;
      else key = key * tv.nlive + sym;
    }
  }
  const bool keep_states = k == kmax;
  uint32_t vb = 0, ve = 0, one = kNoEntry;
  if (keep_states && k > 0) {  // one lookup: the deepest table the lane can use
    uint32_t rb, re;
    pt_find(tv.pt[k - 1], key, true, false, vb, ve, rb, re, one);
  }
  if (tv.rep_levels) {  // reports of the first k symbols, level by level
    uint32_t kk = 0;
    for (int d = 0; d < depth; d++) {
      const bool act = d < k;
      if (act) kk = kk * tv.nlive + c.in[r + d];
      if (!((tv.rep_levels >> d) & 1u)) continue;
      const PrefixTableDev& pt = tv.pt[d];
      uint32_t b0, e0, rb, re, o1;
      pt_find(pt, kk, false, act, b0, e0, rb, re, o1);
      const int len = (int)(re - rb);
      const int mx = __reduce_max_sync(kFull, len);
      for (int i = 0; i < mx; i++) {
        const bool ok = i < len && q + d >= c.emit_lo;
        const uint32_t v = ok ? __ldg(pt.rlist + rb + i) : 0u;
        emit_report(p, ws, w, lane, ok, ok ? (__ldg(t.sid + v)) : 0u, (uint32_t)(q + d));
      }
    }
  }
  // entries at the unit's last position have nothing to expand
  const uint32_t len =
      (keep_states && k > 0 && q + k < c.hi) ? (ve - vb) + (one != kNoEntry ? 1u : 0u) : 0u;
  n_injected += len;
  uint32_t incl = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  if (total == 0) return;
  if (__reduce_max_sync(kFull, len) <= 4u) {
    // short lists (the usual case with deep tables): every lane copies its own
    const int kk = k > 0 ? k : 1;
    const uint32_t off = (uint32_t)(r + kk - 1);
    const uint32_t* vl = tv.pt[kk - 1].vlist;
    for (uint32_t j = 0; j < len; j++) {
      const uint32_t v = one != kNoEntry ? one : __ldg(vl + vb + j);
      uint32_t e = (v << kEntryPosBits) | off;
      if (tv.sticky && is_sticky(tv, v)) {  // registered after the copy instead
        const uint32_t slot = atomicAdd(ws.pend_n, 1u);
        if (slot < (uint32_t)kPendCap) {
          ws.pend_s[slot] = v;
          ws.pend_q[slot] = (uint32_t)(c.wb + off);
          e = kNoEntry;
        }
      }
      store_entry(p, ws, w, w.top + (int)(incl - len + j), e);
    }
    grow_stack(p, w, (int)total);
    __syncwarp();
    return;
  }
  ws.inj[lane] = incl;
  ws.inj[32 + lane] = one != kNoEntry ? one : vb;  // a lone state itself, or where the list starts
  ws.inj[64 + lane] = (uint32_t)(k > 0 ? k : 1) | (one != kNoEntry ? 0x100u : 0u);
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
    const uint32_t kraw = ws.inj[64 + l0];
    const int kk = (int)(kraw & 0xffu);
    const uint32_t v = (kraw & 0x100u) ? ws.inj[32 + l0]
                                       : __ldg(tv.pt[kk - 1].vlist + ws.inj[32 + l0] + (idx - before));
    const uint32_t off = (uint32_t)(r0 + l0 + kk - 1);
    uint32_t e = (v << kEntryPosBits) | off;
    if (tv.sticky && is_sticky(tv, v)) {  // registered after the copy instead
      const uint32_t slot = atomicAdd(ws.pend_n, 1u);
      if (slot < (uint32_t)kPendCap) {
        ws.pend_s[slot] = v;
        ws.pend_q[slot] = (uint32_t)(c.wb + off);
        e = kNoEntry;
      }
    }
    store_entry(p, ws, w, w.top + (int)idx, e);
  }
  grow_stack(p, w, (int)total);
  __syncwarp();
}

__device__ __forceinline__ void sticky_positions(const MatchParams& p, WarpSmem& ws, WarpRun& w,
                                                 const TileView& tv, const UnitCtx& c, int lane,
                                                 int r0, int batch);

// Table words of the next injection batch, read ahead (see inject_aas2):
// kf[h] = k | use << 8 | word << 9 for the lane's position h (use: the whole
// key is live and the list is wanted; word: x[h] holds its inline1 word).
struct InjAhead {
  int r0 = -1 << 30;  // window offset of the batch they belong to; invalid otherwise
  uint32_t x[2];
  uint32_t kf[2];
};

// The lane's position h of the batch at r0: k (live classes of the next
// symbols, a dead class or the window end stop it), whether the whole key is
// live (use), and the key.
__device__ __forceinline__ void inject_key(const TileView& tv, const UnitCtx& c, int lane, int r0,
                                           int batch, int depth, int h, int& k, bool& use,
                                           uint32_t& key) {
  const int r = r0 + 32 * h + lane;
  const bool valid = 32 * h + lane < batch && r < c.iend;
  const int kmax = valid ? min(depth, c.wlen - r) : 0;
  k = kmax;
  key = 0u;
  for (int d = 0; d < depth; d++) {
    if (d < k) {
      const uint32_t sym = c.in[r + d];
      if (sym >= tv.nlive) k = d;
      else key = key * tv.nlive + sym;
    }
  }
  use = k == kmax && k > 0;
}

// Always-active states through the prefix tables for window offsets
// [r0, r0 + batch), batch <= 64, two positions per lane (r0 + lane and
// r0 + 32 + lane), for tiles without sticky states: both table lookups of a
// lane are issued before either list is read, so a warp has two lookups in
// flight per lane. Same entries and reports as inject_aas over the two halves.
// AHEAD (the lean PRIV 0 instances): after this batch's lookups, the lane's inline
// table words of the next batch are read too, and the next call uses them.
template <bool AHEAD>
__device__ __forceinline__ void inject_aas2(const MatchParams& p, WarpSmem& ws, WarpRun& w,
                                            const TileView& tv, const UnitCtx& c, int lane, int r0,
                                            int batch, int depth, unsigned long long& n_injected,
                                            InjAhead& ahead) {
  const TileDev& t = *tv.t;
  int k[2], r[2];
  bool use[2];
  uint32_t vb[2], ve[2], one[2];
  const bool read_ahead = AHEAD && ahead.r0 == r0;  // read during the last batch's expansions
#pragma unroll
  for (int h = 0; h < 2; h++) {
    r[h] = r0 + 32 * h + lane;
    vb[h] = ve[h] = 0u;
    one[h] = kNoEntry;
    uint32_t key = 0u;
    bool word = false;
    if (read_ahead) {
      k[h] = (int)(ahead.kf[h] & 0xffu);
      use[h] = (ahead.kf[h] >> 8) & 1u;
      word = (ahead.kf[h] >> 9) & 1u;
    }
    if (!read_ahead || (use[h] && !word)) inject_key(tv, c, lane, r0, batch, depth, h, k[h], use[h], key);
    if (!use[h]) continue;
    if (word) {  // decode the inline1 word read ahead
      const uint32_t x = ahead.x[h];
      if (x != kHashEmpty) {
        if (x >> 31) {
          vb[h] = (x >> 6) & 0x1ffffffu;
          ve[h] = vb[h] + (x & 63u);
        } else {
          one[h] = x;
        }
      }
    } else {
      uint32_t rb, re;
      pt_find(tv.pt[k[h] - 1], key, true, false, vb[h], ve[h], rb, re, one[h]);
    }
  }
  // read the next batch's table words now: their DRAM round trip overlaps
  // this batch's list copies and the expansions that follow
  ahead.r0 = -1 << 30;
  const int r1 = r0 + batch;
  // (only for inline tables, where the word read ahead is the whole lookup;
  // for the others it would cost a second key computation and no load)
  if (AHEAD && r1 < c.iend && tv.pt[depth - 1].inline1) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      int kn;
      bool un;
      uint32_t key;
      inject_key(tv, c, lane, r1, batch, depth, h, kn, un, key);
      bool word = false;
      if (un) {
        const PrefixTableDev& pt = tv.pt[kn - 1];
        if (pt.inline1) {
          ahead.x[h] = __ldg(pt.voff + key);
          word = true;
        }
      }
      ahead.kf[h] = (uint32_t)kn | (un ? 0x100u : 0u) | (word ? 0x200u : 0u);
    }
    ahead.r0 = r1;
  }
  if (tv.rep_levels) {  // reports of the first k symbols, level by level
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int64_t q = c.wb + r[h];
      uint32_t kk = 0;
      for (int d = 0; d < depth; d++) {
        const bool act = d < k[h];
        if (act) kk = kk * tv.nlive + c.in[r[h] + d];
        if (!((tv.rep_levels >> d) & 1u)) continue;
        const PrefixTableDev& pt = tv.pt[d];
        uint32_t b0, e0, rb, re, o1;
        pt_find(pt, kk, false, act, b0, e0, rb, re, o1);
        const int len = (int)(re - rb);
        const int mx = __reduce_max_sync(kFull, len);
        for (int i = 0; i < mx; i++) {
          const bool ok = i < len && q + d >= c.emit_lo;
          const uint32_t v = ok ? __ldg(pt.rlist + rb + i) : 0u;
          emit_report(p, ws, w, lane, ok, ok ? (__ldg(t.sid + v)) : 0u, (uint32_t)(q + d));
        }
      }
    }
  }
  // entries at the unit's last position have nothing to expand
  uint32_t len[2];
#pragma unroll
  for (int h = 0; h < 2; h++) {
    len[h] = (use[h] && r[h] + k[h] < c.lim)
                 ? (ve[h] - vb[h]) + (one[h] != kNoEntry ? 1u : 0u)
                 : 0u;
    n_injected += len[h];
  }
  const uint32_t mine = len[0] + len[1];
  uint32_t incl = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  if (total == 0) return;
  if (__reduce_max_sync(kFull, max(len[0], len[1])) <= 4u) {
    // short lists: every lane copies its own two
    uint32_t pos = incl - mine;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const uint32_t off = (uint32_t)(r[h] + k[h] - 1);
      const uint32_t* vl = tv.pt[(k[h] > 0 ? k[h] : 1) - 1].vlist;
      for (uint32_t j = 0; j < len[h]; j++)
        store_entry(p, ws, w, w.top + (int)(pos + j),
                    ((one[h] != kNoEntry ? one[h] : __ldg(vl + vb[h] + j)) << kEntryPosBits) | off);
      pos += len[h];
    }
    grow_stack(p, w, (int)total);
    __syncwarp();
    return;
  }
  // long lists: the two halves one after the other, each copied cooperatively
  int base = w.top;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    uint32_t hi = len[h];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, hi, o);
      if (lane >= o) hi += y;
    }
    const uint32_t ht = __shfl_sync(kFull, hi, 31);
    ws.inj[lane] = hi;
    ws.inj[32 + lane] = one[h] != kNoEntry ? one[h] : vb[h];
    ws.inj[64 + lane] = (uint32_t)(k[h] > 0 ? k[h] : 1) | (one[h] != kNoEntry ? 0x100u : 0u);
    __syncwarp();
    for (uint32_t idx = lane; idx < ht; idx += 32) {
      int l0 = 0, l1 = 31;
      while (l0 < l1) {  // first lane whose inclusive prefix exceeds idx
        const int m = (l0 + l1) >> 1;
        if (ws.inj[m] > idx) l1 = m;
        else l0 = m + 1;
      }
      const uint32_t before = l0 > 0 ? ws.inj[l0 - 1] : 0u;
      const uint32_t kraw = ws.inj[64 + l0];
      const int kk = (int)(kraw & 0xffu);
      const uint32_t v = (kraw & 0x100u)
                             ? ws.inj[32 + l0]
                             : __ldg(tv.pt[kk - 1].vlist + ws.inj[32 + l0] + (idx - before));
      const uint32_t off = (uint32_t)(r0 + 32 * h + l0 + kk - 1);
      store_entry(p, ws, w, base + (int)idx, (v << kEntryPosBits) | off);
    }
    base += (int)ht;
    __syncwarp();
  }
  grow_stack(p, w, (int)total);
  __syncwarp();
}

// Injection of a batch of positions: always-active states, then the sticky
// states met while copying, then the work of every active sticky state at
// these positions. Layered tiles (phase 2) do their sticky work separately.
__device__ __forceinline__ void inject(const MatchParams& p, WarpSmem& ws, WarpRun& w,
                                       const TileView& tv, const UnitCtx& c, int lane, int r0,
                                       int batch, int depth, unsigned long long& n_injected) {
  inject_aas(p, ws, w, tv, c, lane, r0, batch, depth, n_injected);
  if (!tv.sticky || tv.t->phase == 2) return;
  __syncwarp();
  const int np = min((int)*ws.pend_n, kPendCap);
  for (int i = 0; i < np; i++) {
    const uint32_t s = ws.pend_s[i];
    const int64_t qq = (int64_t)ws.pend_q[i];
    const bool ok = register_sticky(p, ws, w, tv, c, lane, s, qq, c.wb + r0);
    push_entry(p, ws, w, lane, !ok && lane == 0 && qq + 1 < c.hi,
               (s << kEntryPosBits) | (uint32_t)(qq - c.wb));
  }
  __syncwarp();
  if (lane == 0) *ws.pend_n = 0u;
  __syncwarp();
  sticky_positions(p, ws, w, tv, c, lane, r0, batch);
}

// Work of every active sticky state at window offsets [r0, r0 + batch)
// (lanes over positions): count the successors that match, one prefix sum,
// write; reports (rare) through the warp-collective path.
__device__ __forceinline__ void sticky_positions(const MatchParams& p, WarpSmem& ws, WarpRun& w,
                                                 const TileView& tv, const UnitCtx& c, int lane,
                                                 int r0, int batch) {
  if (w.nstk == 0) return;
  const int r = r0 + lane;
  const bool valid = lane < batch && r < c.wlen;
  const int64_t t = c.wb + r;
  const uint32_t sym = valid ? c.in[r] : 0u;
  const bool need = valid && t + 1 < c.hi;
  int cnt = 0;
  bool any_rep = false;
  for (int i = 0; i < w.nstk; i++) {
    const uint32_t s = ws.stk_s[i];
    if (!(valid && t > (int64_t)ws.stk_q[i])) continue;
    any_rep |= is_report(tv, s) && t >= c.emit_lo;
    const uint4 sc = load_succ(tv, s);
    const uint32_t us[4] = {sc.x, sc.y, sc.z, sc.w};
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const uint32_t u = us[j] & kIdMask;
      if (us[j] != kNoSucc && u != s && accepts(tv, u, sym)) {
        cnt++;
        any_rep |= (us[j] >> 31) && t >= c.emit_lo;
      }
    }
  }
  if (__any_sync(kFull, any_rep)) {
    for (int i = 0; i < w.nstk; i++) {
      const uint32_t s = ws.stk_s[i];
      const bool act = valid && t > (int64_t)ws.stk_q[i];
      const bool rs = act && is_report(tv, s) && t >= c.emit_lo;
      emit_report(p, ws, w, lane, rs, rs ? __ldg(tv.t->sid + s) : 0u, (uint32_t)t);
      const uint4 sc = load_succ(tv, s);
      const uint32_t us[4] = {sc.x, sc.y, sc.z, sc.w};
      bool ok[4];
#pragma unroll
      for (int j = 0; j < 4; j++)
        ok[j] = act && us[j] != kNoSucc && (us[j] & kIdMask) != s &&
                accepts(tv, us[j] & kIdMask, sym);
      report4(p, ws, w, tv, lane, ok, us, t, t >= c.emit_lo);
    }
  }
  const int pc = need ? cnt : 0;
  int incl = pc;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  const int total = __shfl_sync(kFull, incl, 31);
  if (total == 0) return;
  if (pc) {
    int pos = w.top + incl - pc;
    for (int i = 0; i < w.nstk; i++) {
      const uint32_t s = ws.stk_s[i];
      if (t <= (int64_t)ws.stk_q[i]) continue;
      const uint4 sc = load_succ(tv, s);
      const uint32_t us[4] = {sc.x, sc.y, sc.z, sc.w};
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const uint32_t u = us[j] & kIdMask;
        if (us[j] != kNoSucc && u != s && accepts(tv, u, sym))
          store_entry(p, ws, w, pos++, (u << kEntryPosBits) | (uint32_t)r);
      }
    }
  }
  grow_stack(p, w, total);
  __syncwarp();
}

// Layered tiles: the work of the unit's sticky states at window offsets
// [r0, r0 + 32) (lanes over positions). The list holds activation slots
// (stk_s) and first matches (stk_q). Per group of 32 sticky states: lane k
// reads state k's slot and first match (its act_local word and first match
// go to the injection scratch); one loop tests every state's union mask
// (the classes any successor accepts) at every lane's class, with loads that
// do not depend on each other; then each lane visits only the states that
// passed at its position (about two), reads their successor records and
// pushes the matches through a shared-memory counter. A state enables its
// successors after its first match, its shortcut successors (act_local bits
// 28..31) at it too. Reports of successors (rare) take a warp-collective
// pass afterwards.
__device__ __forceinline__ void layered_sticky_positions(const MatchParams& p, WarpSmem& ws,
                                                         WarpRun& w, const TileView& tv,
                                                         const UnitCtx& c, int lane, int r0) {
  const TileDev& t = *tv.t;
  const int r = r0 + lane;
  const bool valid = r < c.wlen;
  const int64_t tp = c.wb + r;
  const uint32_t sym = valid ? c.in[r] : 0u;
  const bool need = valid && tp + 1 < c.hi;
  const bool emit = valid && tp >= c.emit_lo;
  if (w.stk_rep) {  // a reporting sticky state reports at every position after its first match
    for (int i = 0; i < w.nstk; i++) {
      const uint32_t s = __ldg(t.act_local + ws.stk_s[i]) & kActIdMask;
      const bool rs = emit && tp > (int64_t)ws.stk_q[i] && is_report(tv, s);
      emit_report(p, ws, w, lane, rs, rs ? __ldg(t.sid + s) : 0u, (uint32_t)tp);
    }
  }
  const uint32_t word = sym >> 5, bit = 1u << (sym & 31);
  for (int i0 = 0; i0 < w.nstk; i0 += 32) {
    const int n = min(32, w.nstk - i0);
    uint32_t kslot = 0u, kq = 0u;
    if (lane < n) {
      kslot = ws.stk_s[i0 + lane];
      kq = ws.stk_q[i0 + lane];
      ws.inj[lane] = __ldg(t.act_local + kslot);
      ws.inj[32 + lane] = kq;
    }
    if (lane == 0) ws.inj[64] = 0u;  // entries pushed by the group
    // bit k: state i0 + k has matched by this lane's position and some
    // successor of it accepts the lane's class
    uint32_t hit = 0u;
#pragma unroll 4
    for (int k = 0; k < n; k++) {
      const uint32_t sl = __shfl_sync(kFull, kslot, k);
      const uint32_t qk = __shfl_sync(kFull, kq, k);
      const bool h = valid && tp >= (int64_t)qk &&
                     (__ldg(t.stk_union + (size_t)sl * tv.cw + word) & bit);
      hit |= h ? 1u << k : 0u;
    }
    __syncwarp();
    bool rep = false;
    for (uint32_t todo = hit; todo; todo &= todo - 1u) {
      const int k = __ffs(todo) - 1;
      const uint32_t al = ws.inj[k];
      const uint32_t on = tp > (int64_t)ws.inj[32 + k] ? 0xfu : al >> 28;
      const uint4 su = load_succ(tv, al & kActIdMask);
      const uint32_t us[4] = {su.x, su.y, su.z, su.w};
      bool ok[4];
      int cnt = 0;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        ok[j] = ((on >> j) & 1u) && us[j] != kNoSucc && accepts(tv, us[j] & kIdMask, sym);
        cnt += ok[j];
        rep |= ok[j] && (us[j] >> 31) && emit;
      }
      if (need && cnt) {
        int pos = w.top + (int)atomicAdd(&ws.inj[64], (uint32_t)cnt);
#pragma unroll
        for (int j = 0; j < 4; j++)
          if (ok[j]) store_entry(p, ws, w, pos++, ((us[j] & kIdMask) << kEntryPosBits) | (uint32_t)r);
      }
    }
    __syncwarp();
    const int total = (int)ws.inj[64];
    if (__any_sync(kFull, rep)) {  // reports of successors: warp-collective, state by state
      for (uint32_t any = __reduce_or_sync(kFull, hit); any; any &= any - 1u) {
        const int k = __ffs(any) - 1;
        const uint32_t al = ws.inj[k];
        const uint32_t on = !((hit >> k) & 1u) ? 0u
                            : (tp > (int64_t)ws.inj[32 + k] ? 0xfu : al >> 28);
        const uint4 su = load_succ(tv, al & kActIdMask);
        const uint32_t us[4] = {su.x, su.y, su.z, su.w};
        bool ok[4];
#pragma unroll
        for (int j = 0; j < 4; j++)
          ok[j] = ((on >> j) & 1u) && us[j] != kNoSucc && accepts(tv, us[j] & kIdMask, sym);
        report4(p, ws, w, tv, lane, ok, us, tp, emit);
      }
    }
    grow_stack(p, w, total);
    __syncwarp();
  }
}

// Expands the up-to-32 entries on top of the stack: one step of the worklist.
template <int PRIV>
__device__ __forceinline__ void expand_step(const MatchParams& p, WarpSmem& ws, WarpRun& w,
                                            const TileView& tv, const UnitCtx& c, int lane,
                                            int cursor, unsigned long long& n_expanded) {
  const int n = min(w.top, 32);
  uint32_t e = lane < n ? ws.stack[w.top - 1 - lane] : kNoEntry;
  w.top -= n;
  __syncwarp();
  if (p.unique) {  // identical entries in one step are expanded once (--unique)
    const unsigned peers = __match_any_sync(kFull, e);
    if ((__ffs(peers) - 1) != lane) e = kNoEntry;
  }
  const uint32_t v = e >> kEntryPosBits;
  const int r = (int)(e & ((1u << kEntryPosBits) - 1));
  const int64_t q = c.wb + r;
  const bool go = e != kNoEntry && q + 1 < c.hi;
  uint4 sc = make_uint4(kNoSucc, kNoSucc, kNoSucc, kNoSucc);
  uint4 sm = make_uint4(0u, 0u, 0u, 0u);
  uint32_t s = 0;
  if (go) {
    sc = load_succ(tv, v);
    if (tv.fused) sm = load_smask(tv, v);
    s = c.in[r + 1];
  }
  n_expanded += go;
  const uint32_t u[4] = {sc.x, sc.y, sc.z, sc.w};
  const uint32_t um[4] = {sm.x, sm.y, sm.z, sm.w};
  bool ok[4];
  int cnt = 0;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    ok[j] = go && succ_accepts(tv, u[j], um[j], s);
    cnt += ok[j];
  }
  report4(p, ws, w, tv, lane, ok, u, q + 1, q + 1 >= c.emit_lo);
  const bool need = go && q + 2 < c.hi;        // the successors have a next symbol
  const bool at_end = r + 1 == c.wlen;         // successors sit at the next window's start
  if (tv.sticky) {  // matched sticky states are registered instead of pushed
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const bool stk = ok[j] && need && is_sticky(tv, u[j] & kIdMask);
      // positions injected so far: [wb, wb + min(cursor, wlen)) (a batch may end past the window)
      if (register_each(p, ws, w, tv, c, lane, stk, u[j] & kIdMask, q + 1,
                        c.wb + min(cursor, c.wlen))) {
        ok[j] = false;
        cnt--;
      }
    }
  }
  if (__any_sync(kFull, need && at_end)) {
#pragma unroll
    for (int j = 0; j < 4; j++) carry_state(p, w, lane, need && at_end && ok[j], u[j] & kIdMask);
  }
  const bool privatize = PRIV > 0 && !tv.sticky &&
                         __popc(__ballot_sync(kFull, go)) > p.active_threshold;
  if (!privatize) {
    const int pc = (need && !at_end) ? cnt : 0;
    int total;
    const int ex = warp_excl<3>(pc, lane, total);
    if (pc) {
      int pos = w.top + ex;
      const uint32_t tag = (uint32_t)(r + 1);
#pragma unroll
      for (int j = 0; j < 4; j++)
        if (ok[j]) store_entry(p, ws, w, pos++, ((u[j] & kIdMask) << kEntryPosBits) | tag);
    }
    grow_stack(p, w, total);
    __syncwarp();
    return;
  }
  // privatization (kernel_ngap_OA.cu:96-138): expand the matched successors in
  // registers one more level instead of pushing them
  const bool inner = need && !at_end;  // successors' successors read in[r + 2] <= window end
  const uint32_t s2 = inner ? c.in[r + 2] : 0u;
  uint32_t u2[4][4];
  bool ok2[4][4];
  int cnt2 = 0;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    uint4 sc2 = make_uint4(kNoSucc, kNoSucc, kNoSucc, kNoSucc);
    uint4 sm2 = make_uint4(0u, 0u, 0u, 0u);
    if (inner && ok[j]) {
      sc2 = load_succ(tv, u[j] & kIdMask);
      if (tv.fused) sm2 = load_smask(tv, u[j] & kIdMask);
    }
    u2[j][0] = sc2.x;
    u2[j][1] = sc2.y;
    u2[j][2] = sc2.z;
    u2[j][3] = sc2.w;
    const uint32_t um2[4] = {sm2.x, sm2.y, sm2.z, sm2.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      ok2[j][k] = succ_accepts(tv, u2[j][k], um2[k], s2);
      cnt2 += ok2[j][k];
    }
  }
#pragma unroll
  for (int j = 0; j < 4; j++) report4(p, ws, w, tv, lane, ok2[j], u2[j], q + 2, q + 2 >= c.emit_lo);
  const bool need2 = inner && q + 3 < c.hi;
  const bool at_end2 = r + 2 == c.wlen;
  if (__any_sync(kFull, need2 && at_end2)) {
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int k = 0; k < 4; k++)
        carry_state(p, w, lane, need2 && at_end2 && ok2[j][k], u2[j][k] & kIdMask);
  }
  const int pc = (need2 && !at_end2) ? cnt2 : 0;
  int total;
  const int ex = warp_excl<5>(pc, lane, total);
  if (pc) {
    int pos = w.top + ex;
    const uint32_t tag = (uint32_t)(r + 2);
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int k = 0; k < 4; k++)
        if (ok2[j][k]) store_entry(p, ws, w, pos++, ((u2[j][k] & kIdMask) << kEntryPosBits) | tag);
  }
  grow_stack(p, w, total);
  __syncwarp();
}

// One worklist step over up to 64 entries, two per lane, for tiles without
// sticky states and without privatization: both entries' successor records
// are requested before either is used, so a warp keeps two L2 round trips in
// flight per lane instead of one. Same results as two expand_step calls.
// FUSED: the tile's records carry the successors' class masks (one 32-byte
// record per state); the window arithmetic is 32-bit (UnitCtx::lim, elo)
// and the rare report and carry paths are entered on one vote each.
template <bool FUSED>
__device__ __forceinline__ void expand_step2(const MatchParams& p, WarpSmem& ws, WarpRun& w,
                                             const TileView& tv, const UnitCtx& c, int lane,
                                             unsigned long long& n_expanded) {
  const int n = min(w.top, 64);
  uint32_t e[2];
  e[0] = lane < n ? ws.stack[w.top - 1 - lane] : kNoEntry;
  e[1] = lane + 32 < n ? ws.stack[w.top - 33 - lane] : kNoEntry;
  w.top -= n;
  __syncwarp();
  if (p.unique) {  // identical entries in one half-step are expanded once (--unique)
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const unsigned peers = __match_any_sync(kFull, e[k]);
      if ((__ffs(peers) - 1) != lane) e[k] = kNoEntry;
    }
  }
  uint4 sc[2], sm[2];
  uint32_t s[2];
  int r[2];
  bool go[2];
#pragma unroll
  for (int k = 0; k < 2; k++) {
    r[k] = (int)(e[k] & ((1u << kEntryPosBits) - 1));
    go[k] = e[k] != kNoEntry && r[k] + 1 < c.lim;
    sc[k] = make_uint4(kNoSucc, kNoSucc, kNoSucc, kNoSucc);
    sm[k] = make_uint4(0u, 0u, 0u, 0u);
    s[k] = 0u;
    if (go[k]) {
      const uint32_t v = e[k] >> kEntryPosBits;
      if (FUSED) {
        sc[k] = tv.succ[(size_t)v * 2];
        sm[k] = tv.succ[(size_t)v * 2 + 1];
      } else {
        sc[k] = load_succ(tv, v);
      }
      s[k] = c.in[r[k] + 1];
    }
  }
  n_expanded += (unsigned)go[0] + (unsigned)go[1];
  bool ok[2][4], need[2], at_end[2];
  bool rep = false, carry = false;
  int cnt = 0;
#pragma unroll
  for (int k = 0; k < 2; k++) {
    const uint32_t u[4] = {sc[k].x, sc[k].y, sc[k].z, sc[k].w};
    const uint32_t um[4] = {sm[k].x, sm[k].y, sm[k].z, sm[k].w};
    bool rk = false;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      ok[k][j] = go[k] && (FUSED ? ((um[j] >> s[k]) & 1u) != 0u : succ_accepts(tv, u[j], um[j], s[k]));
      rk |= ok[k][j] && (u[j] >> 31);
    }
    rep |= rk && r[k] + 1 >= c.elo;
    need[k] = go[k] && r[k] + 2 < c.lim;
    at_end[k] = r[k] + 1 == c.wlen;
    carry |= need[k] && at_end[k];
    if (need[k] && !at_end[k]) {
#pragma unroll
      for (int j = 0; j < 4; j++) cnt += ok[k][j];
    }
  }
  if (__any_sync(kFull, rep)) {  // reports (rare): the warp-collective path per half
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const uint32_t u[4] = {sc[k].x, sc[k].y, sc[k].z, sc[k].w};
      const int64_t q = c.wb + r[k];
      report4(p, ws, w, tv, lane, ok[k], u, q + 1, r[k] + 1 >= c.elo);
    }
  }
  if (__any_sync(kFull, carry)) {  // states landing on the next window's first position
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const uint32_t u[4] = {sc[k].x, sc[k].y, sc[k].z, sc[k].w};
#pragma unroll
      for (int j = 0; j < 4; j++)
        carry_state(p, w, lane, need[k] && at_end[k] && ok[k][j], u[j] & kIdMask);
    }
  }
  int total;
  const int ex = warp_excl<4>(cnt, lane, total);
  if (cnt) {
    int pos = w.top + ex;
#pragma unroll
    for (int k = 0; k < 2; k++) {
      if (!(need[k] && !at_end[k])) continue;
      const uint32_t u[4] = {sc[k].x, sc[k].y, sc[k].z, sc[k].w};
      const uint32_t tag = (uint32_t)(r[k] + 1);
#pragma unroll
      for (int j = 0; j < 4; j++)
        if (ok[k][j]) store_entry(p, ws, w, pos++, ((u[j] & kIdMask) << kEntryPosBits) | tag);
    }
  }
  grow_stack(p, w, total);
  __syncwarp();
}

// A warp's view of one tile and the knobs derived from it.
struct TileRun {
  TileView tv;
  int depth, batch, defer;
  bool layered, wide_inject;
};

// Builds the view of tile t whose image is at ib (shared-memory copy or the
// global image), prefix-table descriptors at pt and byte classes at cls.
template <bool LEAN>
__device__ __forceinline__ void tile_run(const MatchParams& p, const TileDev* t, const uint8_t* ib,
                                         const PrefixTableDev* pt, const uint8_t* cls,
                                         TileRun& tr) {
  TileView& tv = tr.tv;
  tv.succ = reinterpret_cast<const uint4*>(ib);
  tv.cmask = reinterpret_cast<const uint32_t*>(ib + t->off_cmask);
  tv.rep = reinterpret_cast<const uint32_t*>(ib + t->off_rep);
  tv.sticky = !LEAN && t->nsticky > 0 ? reinterpret_cast<const uint32_t*>(ib + t->off_sticky)
                                        : nullptr;
  tv.cls = cls;
  tv.t = t;
  tv.pt = pt;
  tv.cw = t->cw;
  tv.narrow = t->narrow;
  tv.fused = t->fused;
  tv.nlive = (uint32_t)t->nlive;
  tv.rep_levels = 0u;
  for (int d = 0; d < kMaxDepth; d++) tv.rep_levels |= (pt[d].has_reports ? 1u : 0u) << d;
  tr.depth = p.depth == 0 || t->naas == 0 ? 0 : min(p.depth, t->depth);
  tr.batch = tr.depth == 0 ? t->inj_batch0 : t->inj_batch;
  // short table lists, no sticky states: two positions per lane per injection
  tr.wide_inject = tr.depth > 0 && !tv.sticky && tr.batch == 32;
  // Without sticky states registered during the window (plain tiles
  // without them, layered tiles), the last depth - 1 positions of a window
  // are injected at the start of the next one (from look-behind bytes), so
  // that every position but the unit's last ones gets the full table depth.
  tr.layered = !LEAN && t->phase == 2;
  tr.defer = (tr.depth > 1 && (!tv.sticky || tr.layered)) ? tr.depth - 1 : 0;
}

// Two kinds of work per launch:
//  * tasks (consecutive units of one tile whose image fits shared memory):
//    a CTA stages the image once and its warps take the task's units; the
//    CTA waits for all of them before the next task replaces the image;
//  * free units (tiles read in place through L2): every warp takes the next
//    unit from a global cursor on its own and reads the tile's descriptors
//    from global memory, so no warp waits for another.
// CTAs take tasks until none is left, then free units. LEAN kernels serve
// launches whose tiles have no sticky states and are plain (no activation or
// layered pass): that code is compiled out, for a smaller hot loop.
template <int PRIV, bool LEAN>
__global__ void __launch_bounds__(kCtaThreads, 1) match_kernel(MatchParams p) {
  extern __shared__ __align__(128) uint8_t smem_raw[];
  __shared__ int s_task;
  __shared__ unsigned s_next;
  __shared__ __align__(16) PrefixTableDev s_pt[kMaxDepth];
  __shared__ __align__(16) uint8_t s_cls[256];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int W = p.window;
  uint8_t* image = smem_raw;
  uint8_t* base = smem_raw + p.image_region + (size_t)warp * warp_smem_bytes(W);
  WarpSmem ws;
  ws.stack = reinterpret_cast<uint32_t*>(base);
  ws.in[0] = base + kStackCap * 4;
  ws.in[1] = ws.in[0] + window_buf_bytes(W);
  ws.rbuf = reinterpret_cast<unsigned long long*>(ws.in[1] + window_buf_bytes(W));
  ws.inj = reinterpret_cast<uint32_t*>(ws.rbuf + kReportBuf);
  ws.bar = reinterpret_cast<uint64_t*>(ws.inj + 3 * 32);
  ws.stk_s = reinterpret_cast<uint32_t*>(ws.bar + 2);
  ws.stk_q = ws.stk_s + kStickyCap;
  ws.pend_s = ws.stk_q + kStickyCap;
  ws.pend_q = ws.pend_s + kPendCap;
  ws.pend_n = ws.pend_q + kPendCap;
  if (lane == 0) *ws.pend_n = 0u;
  const int slot = blockIdx.x * kWarpsPerCta + warp;
  WarpRun w;
  w.top = w.ovf_n = w.ncarry = w.nrep = w.nstk = 0;
  w.base = 0;
  w.key_hi = 0ull;
  w.ovf = p.ovf + (size_t)slot * p.ovf_cap;
  w.carry = p.carry + (size_t)slot * p.carry_cap;
  w.marks = p.marks + (size_t)slot * p.mark_words;
  w.act = nullptr;
  w.stk_cap = kStickyCap;
  w.stk_rep = false;
  uint32_t* const stk_smem = ws.stk_s;
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
  int staged = -1;  // tile whose image is in shared memory

  // loads window [wb, min(wb + W, hi)) plus one look-ahead byte and `lb`
  // look-behind bytes into buffer buf; returns the byte count, and in `skip`
  // the offset of wb's byte in the buffer
  auto issue = [&](int buf, int64_t wb, int64_t hi, int lb, uint32_t& skip) {
    const int64_t we = min(wb + (int64_t)W, hi);
    const int64_t end = min(we + 1, hi);
    const int64_t a0 = (wb - lb) & ~(int64_t)15;
    const uint32_t bytes = (uint32_t)(((end - a0) + 15) & ~(int64_t)15);
    skip = (uint32_t)(wb - a0);
    if (lane == 0) {
      mbar_expect_tx(&ws.bar[buf], bytes);
      bulk_g2s(ws.in[buf], p.input + a0, bytes, &ws.bar[buf]);
    }
    pending[buf] = true;
    return bytes;
  };

  // sticky list of a unit: shared memory, or global memory for layered units
  // with more activations (n) than that holds. (Global stores are not
  // cached in L1: a list there costs an L2 round trip per read.)
  auto sticky_lists = [&](const TileDev* t, bool layered, uint32_t n) {
    if (layered && n > (uint32_t)kStickyCap && p.stk_g_cap >= t->nact) {
      ws.stk_s = p.stk_g + (size_t)slot * 2 * p.stk_g_cap;
      ws.stk_q = ws.stk_s + p.stk_g_cap;
      w.stk_cap = p.stk_g_cap;
    } else {
      ws.stk_s = stk_smem;
      ws.stk_q = stk_smem + kStickyCap;
      w.stk_cap = kStickyCap;
    }
  };

  // matches unit uid of tile t (warp-collective)
  auto run_unit = [&](unsigned uid, const TileDev* t, const TileRun& tr) {
    const TileView& tv = tr.tv;
    const int depth = tr.depth, batch = tr.batch, defer = tr.defer;
    const bool layered = tr.layered, wide_inject = tr.wide_inject;
    const UnitDev un = p.units[uid];
    const unsigned long long work0 = n_expanded + n_injected;  // per-unit trace
    if (p.unit_work && lane == 0) p.unit_cycles[uid] = clock64();  // start; the end subtracts
    UnitCtx c;
    c.hi = un.hi;
    c.emit_lo = un.emit_lo;
    w.nstk = 0;  // sticky states are per unit
    w.key_hi = un.key_hi;
    w.base = (uint32_t)un.base;
    w.act = !LEAN && t->phase == 1 ? p.act + un.act_row : nullptr;
    if (layered) {
      // sticky states whose first match (from the activation pass; the
      // segment's matched slots are listed at act_list) comes before the
      // unit's end: active from there on; a reporting one also reports at
      // its first match
      const uint32_t n = p.act_cnt[un.act_rowid];
      sticky_lists(t, true, n);
      bool rep_any = false;
      for (uint32_t i0 = 0; i0 < n; i0 += 32) {
        const uint32_t i = i0 + lane;
        const uint32_t sl = i < n ? p.act_list[un.act_row + i] : 0u;
        const uint32_t f = i < n ? p.act[un.act_row + sl] : kNoAct;
        const int64_t q = un.base + (int64_t)f;
        const bool ok = f != kNoAct && q < c.hi;
        const unsigned m = __ballot_sync(kFull, ok);
        const uint32_t sv = ok ? __ldg(t->act_local + sl) & kActIdMask : 0u;
        if (ok) {
          const int k = w.nstk + __popc(m & lanemask_lt(lane));
          if (k < w.stk_cap) {
            ws.stk_s[k] = sl;
            ws.stk_q[k] = (uint32_t)q;
          } else {
            atomicOr(p.err, kErrQueue);
          }
        }
        w.nstk = min(w.nstk + __popc(m), w.stk_cap);
        const bool rs = ok && is_report(tv, sv);
        rep_any |= rs;
        const bool rep = rs && q >= c.emit_lo;
        emit_report(p, ws, w, lane, rep, rep ? __ldg(t->sid + sv) : 0u, (uint32_t)q);
      }
      w.stk_rep = __any_sync(kFull, rep_any);
      __syncwarp();
    }
    // nothing can become active in a layered unit without sticky states,
    // always-active states or start-of-data states at its first position
    // (such a unit runs no window: its end is moved to its start)
    if (layered && w.nstk == 0 && t->naas == 0 && !((un.flags & 1u) && t->nstart > 0))
      c.hi = un.lo;
    int cur = 0;
    uint32_t nbytes[2], skip[2];
    if (c.hi > un.lo && (int32_t)uid != p.skip_copy_unit) {
      nbytes[0] = issue(0, un.lo, c.hi, 0, skip[0]);
    } else {  // idle, or the test hook: nothing is in flight (the hook's first wait gives up)
      nbytes[0] = 0u;
      skip[0] = 0u;
    }
    int64_t inj_pos = un.lo;  // next position for always-active injection
    for (int64_t wb = un.lo; wb < c.hi; wb += W) {
      const int64_t we = min(wb + (int64_t)W, c.hi);
      c.wb = wb;
      c.wlen = (int)(we - wb);
      c.iend = we == c.hi ? c.wlen : c.wlen - defer;
      c.lim = (int)min(c.hi - wb, (int64_t)1 << 30);
      c.elo = (int)max(min(c.emit_lo - wb, (int64_t)1 << 30), -((int64_t)1 << 30));
      if (!mbar_wait(&ws.bar[cur], phase[cur], p.wait_rounds)) {
        if (lane == 0) atomicOr(p.err, kErrTimeout);
        dead = true;
        break;
      }
      phase[cur] ^= 1u;
      pending[cur] = false;
      // bytes -> class ids, in place (every tile keys its tables by its own
      // classes); a window whose bytes (look-behind and look-ahead included)
      // are all of the dead class, which no state of the tile accepts, has
      // nothing to inject and no sticky work
      bool live = false;
      for (uint32_t i = lane; i < nbytes[cur]; i += 32) {
        const uint8_t k = tv.cls[ws.in[cur][i]];
        ws.in[cur][i] = k;
        live |= k < tv.nlive;
      }
      live = __any_sync(kFull, live);
      __syncwarp();
      if (we < c.hi)
        nbytes[cur ^ 1] = issue(cur ^ 1, we, c.hi, (int)min((int64_t)defer, we - un.lo), skip[cur ^ 1]);
      c.in = ws.in[cur] + skip[cur];
      // carried states: matched at wb
      w.top = 0;
      if (w.ncarry > 0) {
        for (int i = lane; i < w.ncarry; i += 32) {
          const uint32_t u = w.carry[i];
          w.marks[u >> 5] = 0u;
          store_entry(p, ws, w, i, u << kEntryPosBits);
        }
        const int nc = w.ncarry;
        w.ncarry = 0;
        grow_stack(p, w, nc);
        __syncwarp();
      }
      // start-of-data states at the unit's first position (ngap_buffer.cu:613-631)
      if (wb == un.lo && (un.flags & 1u)) {
        const uint32_t s0 = c.in[0];
        for (int i0 = 0; i0 < t->nstart; i0 += 32) {
          const int i = i0 + lane;
          const uint32_t v = i < t->nstart ? __ldg(t->start + i) : 0u;
          const bool ok = i < t->nstart && accepts(tv, v, s0);
          const bool rep = ok && is_report(tv, v) && un.lo >= c.emit_lo;
          emit_report(p, ws, w, lane, rep, rep ? (__ldg(t->sid + v)) : 0u, (uint32_t)un.lo);
          const bool need = ok && un.lo + 1 < c.hi;
          bool reg = false;
          if (layered)  // already registered from the activation pass
            reg = is_sticky(tv, v);
          else if (tv.sticky)
            reg = register_each(p, ws, w, tv, c, lane, need && is_sticky(tv, v), v, un.lo, wb);
          push_entry(p, ws, w, lane, need && !reg, v << kEntryPosBits);
        }
      }
      // next window offset to inject: negative for positions deferred from
      // the previous window (at most `defer` of them)
      // (without always-active states only plain sticky tiles have injection
      // work: their registered sticky states, batch by batch)
      int cursor = !live || (t->naas == 0 && (LEAN || layered || !tv.sticky))
                       ? c.iend
                       : (int)(inj_pos - wb);
      InjAhead ahead;  // table words of the next batch, read ahead (this window only)
      // layered tiles: next window offset of the sticky states' work
      int scur = live && layered && w.nstk > 0 ? 0 : c.wlen;
      while (true) {
        // inject only when the overflow stack is empty, so that it holds at
        // most one batch's excess
        if (w.top < kInjectLow && w.ovf_n == 0) {
          if (cursor < c.iend) {
            if (wide_inject) {
              inject_aas2<LEAN && PRIV == 0>(p, ws, w, tv, c, lane, cursor, 2 * batch, depth,
                                             n_injected, ahead);
              cursor += 2 * batch;
            } else if (LEAN) {
              inject_aas(p, ws, w, tv, c, lane, cursor, batch, depth, n_injected);
              cursor += batch;
            } else {
              inject(p, ws, w, tv, c, lane, cursor, batch, depth, n_injected);
              cursor += batch;
            }
            continue;
          }
          if (!LEAN && scur < c.wlen) {
            layered_sticky_positions(p, ws, w, tv, c, lane, scur);
            scur += 32;
            continue;
          }
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
          if (cursor < c.iend || (!LEAN && scur < c.wlen)) continue;
          break;
        }
        // (layered tiles have no edge into a sticky state: no successor to register)
        if (PRIV == 0 && (LEAN || !tv.sticky || layered)) {
          if (tv.fused)
            expand_step2<true>(p, ws, w, tv, c, lane, n_expanded);
          else
            expand_step2<false>(p, ws, w, tv, c, lane, n_expanded);
        } else {
          expand_step<PRIV>(p, ws, w, tv, c, lane, cursor, n_expanded);
        }
      }
      inj_pos = max(inj_pos, wb + c.iend);  // a batch may end past iend
      cur ^= 1;
    }
    if (p.unit_work) {  // worklist work of this unit (all lanes)
      unsigned long long d = n_expanded + n_injected - work0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(kFull, d, o);
      if (lane == 0) {
        p.unit_work[uid] = d;
        p.unit_cycles[uid] = clock64() - p.unit_cycles[uid];
      }
    }
    if (dead) {
      for (int i = lane; i < w.ncarry; i += 32) w.marks[w.carry[i] >> 5] = 0u;
      w.ncarry = w.top = w.ovf_n = 0;
      // wait (bounded) for any copy still in flight before giving up on this warp
      for (int b = 0; b < 2; b++)
        if (pending[b]) {
          mbar_wait(&ws.bar[b], phase[b], p.wait_rounds);
          pending[b] = false;
        }
      __syncwarp();
    }
  };

  // One loop, one call of run_unit: the next unit comes from the CTA's
  // current task (staged tiles; a new task after a CTA barrier once the
  // current one is exhausted) until no task is left, then from the free
  // units, warp by warp. Every warp of a CTA takes the same barriers: a warp
  // that gave up (dead) still waits for its CTA's tasks to end.
  bool tasks_left = p.ntasks > 0;
  bool free_ready = false;
  bool need_task = true;
  bool task_fits = false;
  int task_end = 0;
  const TileDev* task_tile = nullptr;
  while (true) {
    unsigned uid = 0;
    const TileDev* t = nullptr;
    if (tasks_left) {
      if (need_task) {
        __syncthreads();  // every warp is done with the last task before its image is replaced
        if (threadIdx.x == 0) s_task = (int)atomicAdd(p.task_counter, 1u);
        __syncthreads();
        const int task = s_task;
        if (task >= p.ntasks) {
          tasks_left = false;
          continue;
        }
        const TaskDev tk = p.tasks[task];
        t = &p.tiles[tk.tile];
        const bool fits = t->image_bytes <= p.image_region;
        if (fits && staged != tk.tile) {  // stage the tile image
          const uint4* src = reinterpret_cast<const uint4*>(t->image);
          uint4* dst = reinterpret_cast<uint4*>(image);
          for (int i = threadIdx.x; i < t->image_bytes / 16; i += kCtaThreads) dst[i] = __ldg(src + i);
          staged = tk.tile;
        }
        {  // the tile's prefix-table descriptors, read at every injection, and its byte classes
          const uint32_t* src = reinterpret_cast<const uint32_t*>(t->pt);
          uint32_t* dst = reinterpret_cast<uint32_t*>(s_pt);
          for (int i = threadIdx.x; i < (int)(sizeof(s_pt) / 4); i += kCtaThreads) dst[i] = src[i];
          if (threadIdx.x < 64)
            reinterpret_cast<uint32_t*>(s_cls)[threadIdx.x] =
                __ldg(reinterpret_cast<const uint32_t*>(t->image + t->off_cls) + threadIdx.x);
        }
        if (threadIdx.x == 0) s_next = (unsigned)tk.ubegin;
        __syncthreads();
        task_tile = t;
        task_fits = fits;
        task_end = tk.uend;
        need_task = false;
      }
      if (dead) {
        need_task = true;
        continue;
      }
      if (lane == 0) uid = atomicAdd(&s_next, 1u);
      uid = __shfl_sync(kFull, uid, 0);
      if (uid >= (unsigned)task_end) {
        need_task = true;
        continue;
      }
      t = task_tile;
    } else {
      if (!free_ready) {  // CTA-uniform: every warp of the CTA has left the tasks
        if (p.free_tile >= 0) {  // one tile for all free units: its descriptors in shared memory
          const TileDev* ft = &p.tiles[p.free_tile];
          const uint32_t* src = reinterpret_cast<const uint32_t*>(ft->pt);
          uint32_t* dst = reinterpret_cast<uint32_t*>(s_pt);
          for (int i = threadIdx.x; i < (int)(sizeof(s_pt) / 4); i += kCtaThreads) dst[i] = src[i];
          if (threadIdx.x < 64)
            reinterpret_cast<uint32_t*>(s_cls)[threadIdx.x] =
                __ldg(reinterpret_cast<const uint32_t*>(ft->image + ft->off_cls) + threadIdx.x);
          __syncthreads();
        }
        free_ready = true;
      }
      if (dead || p.nfree <= 0) break;
      unsigned k = 0;
      if (lane == 0) k = atomicAdd(p.free_cursor, 1u);
      k = __shfl_sync(kFull, k, 0);
      if (k >= (unsigned)p.nfree) break;
      uid = (unsigned)p.free_begin + k;
      t = &p.tiles[p.units[uid].tile];
    }
    // the unit's view of its tile (rebuilt per unit, so that it is not live
    // across units): the staged image and shared descriptors of the task, or
    // for free units the global image and descriptors, read in place
    TileRun tr;
    if (tasks_left)
      tile_run<LEAN>(p, t, task_fits ? image : t->image, s_pt, s_cls, tr);
    else if (p.free_tile >= 0 && t == p.tiles + p.free_tile)
      tile_run<LEAN>(p, t, t->image, s_pt, s_cls, tr);
    else
      tile_run<LEAN>(p, t, t->image, t->pt, t->image + t->off_cls, tr);
    sticky_lists(t, false, 0u);  // layered units choose theirs by their activation count
    run_unit(uid, t, tr);
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
