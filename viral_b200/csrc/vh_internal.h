// Internal hooks shared by the translation units of libvh (not exported in
// include/vh.h).
#pragma once
#include <vector>

#include "vh.h"

// configuration of a handle and its EOS table (4 x n: e, P, cs2, T)
int vh_internal_config(const vh_handle* h, vh_config* out, std::vector<double>* eos4);
// record msg as the handle's last error and return code
int vh_internal_error(vh_handle* h, int code, const char* msg);
