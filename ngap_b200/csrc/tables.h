// Host-side construction of the matching tables: tiles of CCs and their
// prefix-memoization tables.
#pragma once

#include <vector>

#include "device_types.h"
#include "nfa.h"

namespace ngap {

struct PrefixTableHost {
  bool dense = false;
  int32_t cutoff = 0;
  std::vector<uint32_t> keys, voff, vlist;
  std::vector<uint32_t> rkeys, roff, rlist;
  int64_t entries() const { return (int64_t)vlist.size() + (int64_t)rlist.size(); }
};

struct TileHost {
  int32_t group = 0;
  int32_t nstates = 0;
  int32_t depth = 0;
  int32_t max_path = -1;
  int32_t num_ccs = 0;
  std::vector<uint32_t> succ;  // nstates * 4
  std::vector<uint32_t> bits;  // nstates * 8
  std::vector<uint32_t> rep;   // ceil(nstates / 32)
  std::vector<uint32_t> sid;   // nstates
  std::vector<uint32_t> aas, start;
  PrefixTableHost pt[kMaxDepth];
};

struct TableOpts {
  int precompute_depth = 0;
  int precompute_cutoff = -1;
  int tile_states = 0;              // 0 = automatic
  int64_t max_table_entries = 0;    // 0 = automatic
  int max_warmup = 2048;            // longest acyclic path that still allows chunking
};

// Splits every group into tiles and builds each tile's tables.
int build_tiles(const GroupSet& gs, const TableOpts& opts, std::vector<TileHost>& tiles);

}  // namespace ngap
