// NFA preprocessing: connected-component split, out-degree limiting and
// grouping. Produces the per-group graphs whose state numbering is the one
// that appears in reports: report id = sid | group << 22.
#pragma once

#include <string>
#include <vector>

#include "anml.h"

namespace ngap {

struct GroupOpts {
  int group_num = 10;       // --group-num
  int max_nfa_size = -1;    // --max-nfa-size
  bool quit_degree = true;  // --quit-degree
  bool remove_degree = false;  // --remove-degree
  int degree_limit = 4;     // fixed at 4 by the reference (ngap.cu:70-71)
};

// One group graph, in the layout of Graph::ReadNFA + Csr::fromCoo
// (code/src/commons/graph.cu:169-206, code/include/commons/graph.h:184-219).
struct GroupGraph {
  int32_t V = 0, E = 0;
  std::vector<int32_t> row_offsets;  // V + 1
  std::vector<int32_t> cols;         // E, sorted by (src, dst)
  std::vector<uint32_t> bits;        // V * 8, bit s of word s/32 => accepts byte s
  std::vector<uint8_t> attrs;        // bit0 always-active, bit1 report
  std::vector<int32_t> aas;          // always-active (all-input) states, ascending
  std::vector<int32_t> starts;       // start-of-data states, ascending
  std::vector<int32_t> cc_begin;     // first sid of each CC, plus V at the end
  std::vector<int32_t> orig_node;    // sid -> index of the ANML STE it was cloned from
};

struct GroupSet {
  int group_num = 0;                 // after clamping to the CC count
  int64_t num_ccs_total = 0;         // CCs before limiting
  int64_t num_ccs_failed = 0;        // CCs dropped because the degree limit failed
  int64_t num_ccs_too_big = 0;       // CCs dropped by max_nfa_size
  std::vector<GroupGraph> groups;
};

int build_groups(const AnmlNfa& nfa, const GroupOpts& opts, GroupSet& out);

}  // namespace ngap
