// Shared host-side definitions: status codes, error reporting, small helpers.
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/ngap_b200.h"

namespace ngap {

// Records the message returned by ngap_last_error() for the calling thread.
void set_error(const char* fmt, ...) __attribute__((format(printf, 1, 2)));
const std::string& last_error();

// 256-bit symbol class of one STE; bit s set <=> the STE accepts byte s.
struct Bits256 {
  uint32_t w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  void set(int s) { w[s >> 5] |= 1u << (s & 31); }
  void reset(int s) { w[s >> 5] &= ~(1u << (s & 31)); }
  bool test(int s) const { return (w[s >> 5] >> (s & 31)) & 1u; }
  void set_all() {
    for (auto& x : w) x = 0xffffffffu;
  }
  void flip() {
    for (auto& x : w) x = ~x;
  }
  int count() const {
    int n = 0;
    for (auto x : w) n += __builtin_popcount(x);
    return n;
  }
  bool operator==(const Bits256& o) const {
    for (int i = 0; i < 8; i++)
      if (w[i] != o.w[i]) return false;
    return true;
  }
};

// Start attribute of an STE (NFALoader.cpp:24-35, node.h NODE_START_ENUM).
enum StartKind : uint8_t { kStartNone = 0, kStartOfData = 1, kStartAllInput = 2 };

}  // namespace ngap
