// Hierarchy planner of the uniform pressure multigrid.
//
// Follows planUniformCM11aHierarchy (lib/methods/uniform/
// webgpu-uniform-pressure-multigrid.ts:149-169): halve all axes in lockstep when
// the thinnest axis is a power of two and every axis divides evenly, else halve
// each even axis above two cells on its own schedule; the coarsest lattice plus
// its one-cell halo must fit 256 cells.  Where the reference rejects a lattice
// (odd edges such as 37x50x99), this planner continues with ceil-halving of
// every axis above two cells; a coarse cell then covers fine cells {2c, 2c+1}
// clipped to the grid.  Level maps of accepted lattices are identical to the
// reference's.
#include "plan.h"

#include <algorithm>

namespace fpp {
namespace {

constexpr long kCoarsestLimit = 256;  // UNIFORM_CM11A_COARSEST_LANES

long with_halo(const int* d) { return long(d[0] + 2) * long(d[1] + 2) * long(d[2] + 2); }

// Lockstep rule: levelCount = floor(log2(min)); every axis divisible by 2^(levelCount-1).
int lockstep(const int* d, int (*out)[3]) {
  const int thinnest = std::min(d[0], std::min(d[1], d[2]));
  if (thinnest & (thinnest - 1)) return 0;
  int count = 0;
  for (int v = thinnest; v > 1; v >>= 1) ++count;
  const int factor = 1 << (count - 1);
  if (d[0] % factor || d[1] % factor || d[2] % factor) return 0;
  if (count > kMaxLevels) return 0;
  for (int l = 0; l < count; ++l)
    for (int a = 0; a < 3; ++a) out[l][a] = d[a] >> l;
  return with_halo(out[count - 1]) <= kCoarsestLimit ? count : 0;
}

// Semi-coarsening rule: an axis halves while it is even and above two cells.
int semi_coarsened(const int* d, int (*out)[3]) {
  int count = 1;
  for (int a = 0; a < 3; ++a) out[0][a] = d[a];
  while (count < kMaxLevels) {
    bool changed = false;
    for (int a = 0; a < 3; ++a) {
      const int v = out[count - 1][a];
      const int next = (v % 2 == 0 && v > 2) ? v / 2 : v;
      changed |= next != v;
      out[count][a] = next;
    }
    if (!changed) break;
    ++count;
  }
  return count;
}

int ceil_halving(const int* d, int (*out)[3]) {
  int count = 1;
  for (int a = 0; a < 3; ++a) out[0][a] = d[a];
  while (with_halo(out[count - 1]) > kCoarsestLimit) {
    if (count >= kMaxLevels) return 0;
    bool changed = false;
    for (int a = 0; a < 3; ++a) {
      const int v = out[count - 1][a];
      out[count][a] = v > 2 ? (v + 1) / 2 : v;
      changed |= out[count][a] != v;
    }
    if (!changed) return 0;
    ++count;
  }
  return count;
}

}  // namespace

HierarchyPlan plan_hierarchy(int nx, int ny, int nz) {
  HierarchyPlan p;
  const int d[3] = {nx, ny, nz};
  if (nx < 2 || ny < 2 || nz < 2) {
    p.rejection = "CM11a dense hierarchy requires positive integral dimensions of at least two cells";
    return p;
  }
  int levels[kMaxLevels][3];
  int count = lockstep(d, levels);
  p.semi = false;
  if (!count) {
    count = semi_coarsened(d, levels);
    p.semi = true;
  }
  if (with_halo(levels[count - 1]) > kCoarsestLimit) {
    count = ceil_halving(d, levels);
    p.semi = false;
    p.extended = true;
    if (!count) {
      p.rejection = "CM11a coarsest grid must be integral and fit its 256-lane high-precision solve";
      return p;
    }
  }
  p.levels = count;
  for (int l = 0; l < count; ++l)
    for (int a = 0; a < 3; ++a) {
      p.dims[l][a] = levels[l][a];
      p.stride[l][a] = (l > 0 && levels[l][a] < levels[l - 1][a]) ? 2 : 1;
    }
  p.coarsest_haloed = (int)with_halo(levels[count - 1]);
  p.ok = true;
  return p;
}

}  // namespace fpp
