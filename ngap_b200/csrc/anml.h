// ANML reader: homogeneous NFA as written in the file (ids, symbol classes,
// start kinds, report flags, ordered activate-on-match edges).
#pragma once

#include <string>
#include <vector>

#include "common.h"

namespace ngap {

struct AnmlNode {
  std::string str_id;
  std::string symbol_set_str;
  Bits256 symbols;
  uint8_t start = kStartNone;
  bool report = false;
  std::string report_code;
};

// Nodes in file order (that order is the reference's integer id); adj[i] lists
// the targets of node i in activate-on-match order, duplicates removed.
struct AnmlNfa {
  std::vector<AnmlNode> nodes;
  std::vector<std::vector<int>> adj;
  int64_t num_edges() const {
    int64_t e = 0;
    for (auto& a : adj) e += (int64_t)a.size();
    return e;
  }
};

// VASim symbol-set grammar (code/src/commons/vasim_helper.cpp:40).
bool parse_symbol_set(const std::string& ss, Bits256& col, std::string& err);

int parse_anml(const char* xml, size_t len, AnmlNfa& out);
int load_anml_file(const char* path, AnmlNfa& out);

}  // namespace ngap
