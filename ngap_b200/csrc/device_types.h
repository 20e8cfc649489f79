// Structures shared by host table building and device kernels.
#pragma once

#include <vector_types.h>

#include <cstdint>

namespace ngap {

constexpr uint32_t kNoSucc = 0xffffffffu;
// act_local of layered tiles: local id of the slot's sticky state in the low
// 28 bits; bit 28 + j set when the state enables its successor j from its
// first match on (a shortcut) rather than from the next position
constexpr uint32_t kActIdMask = 0x0fffffffu;
constexpr int kMaxDepth = 12;        // prefix-memoization depth limit (the reference stops at 3)
constexpr int kEntryPosBits = 13;    // worklist entry = local_state << 13 | window offset
constexpr int kMaxWindow = (1 << kEntryPosBits) - 2;
constexpr int kMaxTileStates = 1 << (32 - kEntryPosBits);
constexpr uint64_t kDenseKeys = 1ull << 18;     // prefix tables with <= 2^18 keys are dense
constexpr uint64_t kMaxDenseKeys = 1ull << 26;  // larger ones are dense when that is smaller

constexpr uint32_t kHashEmpty = 0xffffffffu;

// One prefix-memoization table of depth d for a tile (precompute_table.h:8-101).
// The key is the live class ids c_0 .. c_{d-1} of the next d input bytes as a
// base-L number (L = TileDev::nlive): ((c_0 * L + c_1) * L + ...) + c_{d-1}.
// A byte of the dead class (accepted by no state of the tile) ends every path,
// so keys never contain it. dense: offsets indexed by the key (key space
// <= kDenseKeys); otherwise an open-addressing hash table (linear probing,
// capacity a power of two, at least twice the keys) whose slots hold
// {key, state-list begin, report-list begin, state-list length << 16 |
// report-list length}; the reference binary-searches a sorted key array
// (precompute_table.h:59-100).
// inline1 (dense tables without report lists): voff holds one word per key
// [space]: kHashEmpty for an empty list, the state itself (bit 31 clear) for
// a list of one, else bit 31 | begin << 6 | length (2..63) into vlist; most
// keys of a deep table have at most one state, so a lookup is one read.
struct PrefixTableDev {
  int32_t dense = 0;
  uint32_t hmask = 0;               // hash capacity - 1
  int32_t cutoff = 0;
  int32_t has_reports = 0;          // any report list non-empty
  int32_t inline1 = 0;
  int32_t pad = 0;
  const uint32_t* voff = nullptr;   // dense: state-list offsets [space + 1], or inline1 words
  const uint32_t* roff = nullptr;   // dense: report-list offsets [space + 1] (if reports)
  const uint4* slots = nullptr;     // hashed: [hmask + 1]
  const uint32_t* vlist = nullptr;  // local states reached after d symbols
  const uint32_t* rlist = nullptr;  // local report states reached after d symbols
};

__host__ __device__ inline uint32_t prefix_hash(uint32_t key) {
  return (key * 0x9E3779B1u) ^ (key >> 15);
}

// A tile: a set of whole CCs (of one group, or of several for a global tile),
// matched by one warp per unit. Its hot tables form one contiguous image,
// staged into shared memory by the CTA that works on the tile when it fits
// (global tiles are read in place, through L2):
//   [succ][cmask: nstates x cw x u32][rep: ceil(nstates/32) x u32][cls: 256 B]
// succ: up to 4 tile-local successors per state; narrow tiles (< 32767
// states) store 4 x u16 (bit 15 = report successor, 0xffff = none), wide
// ones 4 x u32 (bit 31 = report successor, kNoSucc = none); fused wide tiles
// (one class word) follow each state's 4 x u32 with its successors' class
// masks (4 x u32, 0 for none), a 32-byte record. cmask: bit c of
// word c/32 = the state accepts byte class c. cls: byte -> class id, live
// classes first, the dead class (bytes no state accepts) last.
struct TileDev {
  int32_t group = 0;        // group of the first CC (report ids are in sid)
  int32_t nstates = 0;
  int32_t naas = 0;
  int32_t nstart = 0;
  int32_t depth = 0;        // prefix depth built for this tile (>= 1)
  int32_t max_path = -1;    // longest path in states if acyclic, else -1
  int32_t ncls = 0;         // byte classes
  int32_t cw = 8;           // class-mask words per state: ceil(classes / 32), 1..8
  int32_t nlive = 0;        // live classes: key base; class id nlive = dead
  int32_t narrow = 1;       // 16-bit successors
  int32_t fused = 0;        // wide, one class word: records of 2 x uint4 (successors, their masks)
  int32_t image_bytes = 0;  // multiple of 16
  int32_t off_cmask = 0, off_rep = 0, off_cls = 0;
  int32_t inj_batch = 32;   // positions injected per worklist refill (prefix tables)
  int32_t inj_batch0 = 32;  // the same when the always-active list is scanned
  int32_t nsticky = 0;      // sticky states (bitmap at off_sticky in the image)
  int32_t off_sticky = 0;
  int32_t phase = 0;        // 0 plain; 1 activation pass; 2 layered (sticky states pre-registered)
  int32_t nact = 0;         // activation slots per segment (phase 1 and 2)
  const uint32_t* act_local = nullptr;  // phase 2: [nact] each slot's sticky state (kActIdMask)
  const uint32_t* stk_union = nullptr;  // phase 2: [nact][cw] classes any successor accepts
  const uint8_t* image = nullptr;   // global copy of the image (16-byte aligned)
  const uint32_t* sid = nullptr;    // [nstates] local -> report id (sid | group << 22)
  const uint32_t* aas = nullptr;    // [naas] local ids
  const uint32_t* start = nullptr;  // [nstart] local ids
  PrefixTableDev pt[kMaxDepth];
};

// A unit of work: one tile over input positions [lo, hi); reports are kept for
// positions >= emit_lo (the positions before are warm-up of a chunk). A report
// at position q is stored as key_hi | (q - base) << off_shift | id, where
// key_hi carries the stream index in batched matching (0 otherwise). Units of
// activation tiles record the first match of sticky state slot i of their
// segment as atomicMin(act[act_row + i], q - base); units of the paired
// layered tile read those slots.
struct UnitDev {
  int32_t tile;
  uint32_t flags;  // bit0: inject start-of-data states at lo
  int64_t lo, hi, emit_lo;
  int64_t base;      // first byte of the unit's stream
  uint64_t key_hi;   // stream index, already shifted into the report key
  int64_t act_row;   // phase 1 and 2 tiles: first activation slot of the unit's segment
  int32_t act_rowid; // its row (pair, segment) in the compacted activation lists
  int32_t stream;    // segment (plain matching) or stream (batched matching) index
};

// A CTA-level task: consecutive units [ubegin, uend) of one tile.
struct TaskDev {
  int32_t tile;
  int32_t ubegin, uend;
  int32_t pad;
};

}  // namespace ngap
