// Host-side hierarchy planning for the uniform pressure multigrid.
#pragma once

namespace fpp {

constexpr int kMaxLevels = 24;

struct HierarchyPlan {
  int levels = 0;
  int dims[kMaxLevels][3] = {};
  int stride[kMaxLevels][3] = {};  // per-axis coarsening factor from level l-1 (1 or 2)
  int coarsest_haloed = 0;
  bool semi = false;       // reference semi-coarsening schedule
  bool extended = false;   // ceil-halving schedule for lattices the reference rejects
  bool ok = false;
  const char* rejection = nullptr;
};

HierarchyPlan plan_hierarchy(int nx, int ny, int nz);

}  // namespace fpp
