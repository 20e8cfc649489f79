// Structures shared by host table building and device kernels.
#pragma once

#include <vector_types.h>

#include <cstdint>

namespace ngap {

constexpr uint32_t kNoSucc = 0xffffffffu;
constexpr int kMaxDepth = 3;         // prefix-memoization depth limit (reference: 0..3)
constexpr int kEntryPosBits = 13;    // worklist entry = local_state << 13 | window offset
constexpr int kMaxWindow = (1 << kEntryPosBits) - 2;
constexpr int kMaxTileStates = 1 << (32 - kEntryPosBits);

// One prefix-memoization table of depth d for a tile (precompute_table.h:8-101).
// Key = d input bytes in base 256. dense: offsets indexed by key; otherwise
// keys[] holds the sorted non-empty keys and offsets are indexed by rank.
struct PrefixTableDev {
  int32_t dense = 0;
  int32_t nkeys = 0;
  int32_t nrkeys = 0;
  int32_t cutoff = 0;
  const uint32_t* keys = nullptr;   // state-list keys (compressed)
  const uint32_t* voff = nullptr;   // state-list offsets
  const uint32_t* vlist = nullptr;  // local states reached after d bytes
  const uint32_t* rkeys = nullptr;  // report-list keys (compressed)
  const uint32_t* roff = nullptr;   // report-list offsets
  const uint32_t* rlist = nullptr;  // local report states reached after d bytes
};

// A tile: a set of whole CCs of one group, matched by one warp per unit.
struct TileDev {
  int32_t group = 0;
  int32_t nstates = 0;
  int32_t naas = 0;
  int32_t nstart = 0;
  int32_t depth = 0;       // prefix depth used by this tile (0 = scan the AAS list)
  int32_t max_path = -1;   // longest path in states if acyclic, else -1
  const uint4* succ = nullptr;      // [nstates] local successors (edges into AAS removed)
  const uint32_t* bits = nullptr;   // [nstates * 8] symbol classes
  const uint32_t* rep = nullptr;    // [ceil(nstates / 32)] report bitmap
  const uint32_t* sid = nullptr;    // [nstates] local -> group-local sid
  const uint32_t* aas = nullptr;    // [naas] local ids
  const uint32_t* start = nullptr;  // [nstart] local ids
  PrefixTableDev pt[kMaxDepth];
};

// A unit of work: one tile over input positions [lo, hi); reports are kept for
// positions >= emit_lo (the positions before are warm-up of a chunk).
struct UnitDev {
  int32_t tile;
  uint32_t flags;  // bit0: inject start-of-data states at lo
  int64_t lo, hi, emit_lo;
};

}  // namespace ngap
