// Definitions of the opaque C ABI handles shared by the translation units.
#pragma once

#include "anml.h"
#include "nfa.h"

struct ngap_nfa {
  ngap::AnmlNfa nfa;
};

struct ngap_groups {
  ngap::GroupSet gs;
};
