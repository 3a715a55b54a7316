// Host-side container of a compiled device program (see plan.h).
#pragma once
#include <stdint.h>
#include <string>
#include <vector>

#include "plan.h"

namespace wm {

struct HostProgram {
  int nside = 0, lmax = 0, mmax = 0;
  int32_t max_rows = 0;                 // largest intermediate buffer over all matrices
  std::vector<DevMatrix> mats;          // (m, odd) in file order: index 2m + odd
  std::vector<DevDBlock> dblocks;
  std::vector<DevStrip> strips;
  std::vector<DevLevel> levels;
  std::vector<DevPair> pairs;
  std::vector<double> f64;
  std::vector<int32_t> i32;
  std::vector<int64_t> element_count;   // header element_count per (2m + odd)
};

// Parses a rev1 file image.  nside_expect < 0 accepts any nside.
bool compile_resource(const char *data, size_t len, int nside_expect, int lmax_expect,
                      int mmax_expect, HostProgram &P, std::string &err);

}  // namespace wm
