// Host-side tall-cell layout planning (see tall_plan.h).
#include "tall_plan.h"

#include <algorithm>
#include <cmath>

#include "types.h"

namespace fpp {

namespace {
// Math.round: nearest integer, halves toward +infinity.
double js_round(double v) { return std::floor(v + 0.5); }
}  // namespace

int tall_choose_base(int lowest_surface, int highest_surface, int fine_ny, int regular_layers, int liquid_halo,
                     int air_halo) {
  const int maximum_base = std::max(0, fine_ny - regular_layers);
  const int lower = highest_surface + 1 + air_halo - regular_layers;
  const int upper = lowest_surface + 1 - liquid_halo;
  const int desired = lower <= upper ? int(js_round((lower + upper) / 2.0)) : lower;
  const int clamped = std::max(0, std::min(maximum_base, desired));
  return maximum_base >= 2 ? std::max(2, clamped) : 0;
}

void tall_limit_bases(float* bases, int nx, int nz, int max_delta, int passes) {
  std::vector<float> cur(bases, bases + (size_t)nx * nz), next(cur.size());
  for (int pass = 0; pass < passes; ++pass) {
    next = cur;
    for (int z = 0; z < nz; ++z)
      for (int x = 0; x < nx; ++x) {
        const int i = x + nx * z;
        float upper = cur[i];
        if (x > 0) upper = std::min(upper, cur[i - 1] + float(max_delta));
        if (x + 1 < nx) upper = std::min(upper, cur[i + 1] + float(max_delta));
        if (z > 0) upper = std::min(upper, cur[i - nx] + float(max_delta));
        if (z + 1 < nz) upper = std::min(upper, cur[i + nx] + float(max_delta));
        next[i] = float(js_round(upper));
      }
    cur.swap(next);
  }
  std::copy(cur.begin(), cur.end(), bases);
}

TallPlan plan_tall(int nx, int nz, int fine_ny, int band, const int* bases) {
  TallPlan plan;
  if (nx < 1 || nz < 1 || band < 2 || fine_ny < band + 2) {
    plan.rejection = "tall grid needs a band of at least 2 rows and a tall cell of at least 2 rows";
    return plan;
  }
  TallLevel l0;
  l0.nx = nx;
  l0.nz = nz;
  l0.fine_ny = fine_ny;
  l0.band = band;
  l0.bases.assign(bases, bases + (size_t)nx * nz);
  for (int b : l0.bases)
    if (b < 2 || b + band > fine_ny) {
      plan.rejection = "every column needs base >= 2 and its band inside the domain";
      return plan;
    }
  plan.levels.push_back(l0);
  while ((int)plan.levels.size() < kMaxLevels && plan.levels.back().samples() > kMaxCoarse) {
    const TallLevel& f = plan.levels.back();
    if (f.nx == 1 && f.nz == 1 && f.band == 2) break;
    TallLevel c;
    c.nx = (f.nx + 1) / 2;
    c.nz = (f.nz + 1) / 2;
    c.fine_ny = (f.fine_ny + 1) / 2;
    c.band = std::max(2, f.band / 2);
    if (c.fine_ny < c.band + 2) c.fine_ny = c.band + 2;
    c.bases.resize((size_t)c.nx * c.nz);
    for (int Z = 0; Z < c.nz; ++Z)
      for (int X = 0; X < c.nx; ++X) {
        int m = 0;
        for (int dz = 0; dz < 2; ++dz)
          for (int dx = 0; dx < 2; ++dx) {
            const int x = 2 * X + dx, z = 2 * Z + dz;
            if (x < f.nx && z < f.nz) m = std::max(m, f.bases[x + f.nx * z]);
          }
        const int b = std::min(std::max(2, (m + 1) / 2), c.fine_ny - c.band);
        c.bases[X + c.nx * Z] = b;
      }
    plan.levels.push_back(c);
  }
  if (plan.levels.back().samples() > kMaxCoarse) {
    plan.rejection = "coarsest tall grid exceeds the dense coarse solve";
    return plan;
  }
  plan.ok = true;
  return plan;
}

}  // namespace fpp
