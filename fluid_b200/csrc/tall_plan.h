// Host-side layout planning for the restricted tall-cell grid: per-column tall
// cell height ("base") and the coarse tall grids of its multigrid hierarchy.
#pragma once
#include <vector>

#include "plan.h"

namespace fpp {

// chooseTallCellBase (lib/core/tall-cell-grid.ts:61-82).
int tall_choose_base(int lowest_surface, int highest_surface, int fine_ny, int regular_layers, int liquid_halo,
                     int air_halo);

// limitNeighboringTallCellBases (lib/core/tall-cell-grid.ts:84-106): `passes`
// Jacobi passes of base <= neighbour + max_delta over the 4-neighbourhood of
// an nx x nz column grid (index x + nx * z), rounded like Math.round.
void tall_limit_bases(float* bases, int nx, int nz, int max_delta, int passes);

// One tall grid of the hierarchy: columns, world rows, band rows, bases.
struct TallLevel {
  int nx = 0, nz = 0, fine_ny = 0, band = 0;
  std::vector<int> bases;   // x + nx * z
  int P() const { return band + 2; }
  long long samples() const { return (long long)nx * P() * nz; }
};

struct TallPlan {
  std::vector<TallLevel> levels;
  bool ok = false;
  const char* rejection = nullptr;
};

// Level 0 from the caller's bases; each coarser level halves nx, nz (ceil),
// the world rows (ceil) and the band (down to 2), and its column base covers
// every child's tall cell: base = max(2, ceil(max child base / 2)), clamped so
// the band stays inside the domain (the coarse tall grid covers the finer one,
// docs/papers/tallCells.txt Eq. 8-9 with no terrain).  Coarsening stops once a
// level has at most kMaxCoarse samples.
TallPlan plan_tall(int nx, int nz, int fine_ny, int band, const int* bases);

}  // namespace fpp
