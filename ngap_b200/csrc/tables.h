// Host-side construction of the matching tables: tiles of CCs, their byte
// classes, shared-memory images and prefix-memoization tables.
#pragma once

#include <vector>

#include "device_types.h"
#include "nfa.h"

namespace ngap {

struct PrefixTableHost {
  bool dense = false;
  bool inline1 = false;               // dense, one word per key (see PrefixTableDev::inline1)
  int32_t cutoff = 0;
  uint32_t hmask = 0;
  std::vector<uint32_t> voff, roff;   // dense
  std::vector<uint32_t> slots;        // hashed: 4 words per slot
  std::vector<uint32_t> vlist, rlist;
  int64_t entries = 0;                // state-list entries over all keys
  int32_t max_len = 0;                // longest state list
};

struct TileHost {
  int32_t group = 0;
  int32_t nstates = 0;
  int32_t depth = 0;
  int32_t max_path = -1;
  int32_t num_ccs = 0;
  int32_t ncls = 0, cw = 8, nlive = 0;
  bool narrow = true;                // 16-bit successor ids in the image
  bool fused = false;                // wide tile of <= 32 classes: each state's successor ids and
                                     // their class masks in one 32-byte record
  int32_t inj_batch = 32;            // positions injected per worklist refill
  int32_t inj_batch0 = 32;           // the same without prefix tables (AAS scan)
  bool global = false;               // tables read through L2, never staged in shared memory
  int32_t phase = 0;                 // 0 plain, 1 activation pass, 2 layered (stickies from pass 1)
  int32_t pair = -1;                 // activation/layered tiles: index of their pair
  int32_t nact = 0;                  // activation slots (sticky states) of the pair
  std::vector<uint32_t> act_local;   // layered: sticky state of each slot and its shortcut bits (kActIdMask)
  std::vector<uint32_t> stk_union;   // layered: [nact][cw] classes any successor of the slot accepts
  std::vector<uint8_t> cls;          // 256: byte -> class, live classes first
  std::vector<uint32_t> succ;        // nstates * 4, bit 31 = report successor
  std::vector<uint32_t> bits;        // nstates * 8 raw symbol classes
  std::vector<uint32_t> cmask;       // nstates * cw
  int64_t plan_bytes = 0;            // the image's size for planning decisions (tile packing,
                                     // staging): with 1, 2 or 8 mask words, as the planner was
                                     // tuned, though the image holds ceil(classes / 32)
  std::vector<uint32_t> rep;         // ceil(nstates / 32)
  std::vector<uint32_t> sid;         // nstates: report id, group-local sid | group << 22
  std::vector<uint32_t> aas, start;
  std::vector<uint32_t> sticky;      // ceil(nstates / 32): self-loop + every byte, not always-active
  int32_t nsticky = 0;
  std::vector<uint8_t> image;        // succ | cmask | rep | sticky | cls, 16-byte aligned parts
  int32_t off_cmask = 0, off_rep = 0, off_sticky = 0, off_cls = 0;
  PrefixTableHost pt[kMaxDepth];
};

struct TableOpts {
  int precompute_depth = 0;
  int precompute_cutoff = -1;
  int tile_states = 0;              // max states per tile; 0 = fill the image budget
  int64_t max_table_entries = 0;    // 0 = automatic
  int image_budget = 128 * 1024;    // bytes of shared memory for one tile's image
  int unbounded_tile_states = 256;  // cap for tiles of cyclic CCs (one unit per segment)
  int64_t auto_table_bytes = 12 << 20;  // automatic depth: prefix-table bytes per tile
  int max_warmup = 2048;            // longest acyclic path that still allows chunking
  int tile_mode = 0;                // 0 automatic, 1 shared-memory tiles, 2 global tiles
  bool layered = true;              // chunk CCs that are cyclic only through sticky self-loops
  int64_t auto_global_table_bytes = 192 << 20;  // automatic depth, global tiles
  int64_t global_table_entries = 32 << 20;     // list entries per table, global tiles
};

constexpr int32_t kNarrowMaxStates = 32767;  // 15-bit tile-local ids

// Bytes of a tile image with n states and cw class words.
// Mask words per state in the planner's size rule (1, 2 or 8).
inline int plan_class_words(int ncls) { return ncls <= 32 ? 1 : (ncls <= 64 ? 2 : 8); }

inline int64_t image_bytes(int64_t n, int cw) {
  auto r16 = [](int64_t x) { return (x + 15) & ~(int64_t)15; };
  const int64_t succ = n <= kNarrowMaxStates ? n * 8 : n * 16;
  return r16(succ) + r16(n * cw * 4) + 2 * r16(((n + 31) / 32) * 4) + 256;
}

// Splits every group into tiles and builds each tile's tables.
int build_tiles(const GroupSet& gs, const TableOpts& opts, std::vector<TileHost>& tiles);

// Checks the public table options (NULL = the defaults) and converts them;
// `fn` names the entry point in the error message. *device gets the device.
int table_opts_from(const ngap_table_opts* opts, const char* fn, TableOpts& out, int* device);

}  // namespace ngap
