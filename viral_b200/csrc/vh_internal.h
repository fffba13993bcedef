// Internal hooks shared by the translation units of libvh (not exported in
// include/vh.h).
#pragma once
#include <vector>

#include "vh.h"

// configuration of a handle and its EOS table (4 x n: e, P, cs2, T)
int vh_internal_config(const vh_handle* h, vh_config* out, std::vector<double>* eos4);
