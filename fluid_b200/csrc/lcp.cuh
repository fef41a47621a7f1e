// The CM11a LCP variant: a standalone projected multigrid solve of
// A p = b subject to p >= p_min (Chentanez & Mueller 2011, the reference's
// uniform GPU method: webgpu-uniform-pressure-multigrid.ts:419-576 and
// webgpu-uniform-pressure-multigrid.wgsl.ts:155-166, 267-344, 404-471).
//
// The bound lives on solid cells that are pressure unknowns (open fraction <=
// 1e-5, liquid by the continued density): p >= 0 there, so a solid can push the
// liquid but not pull it (a separating boundary); elsewhere p_min = -inf
// (mgBuildFinestRhs, mg.wgsl.ts:155-166).  A domain wall the host wants
// separating is a layer of solid cells at the lattice's edge, the reference's
// one-cell halo.  The schedule is the reference's: full cycles, then V-cycles,
// each smoothing with projected red-black Gauss-Seidel (mgSmoothColour); a
// V-cycle's coarse correction is bounded by max over the children of
// (p_min - p) on the first `constraint_levels` coarse levels and unbounded
// below them (mgDownsampleSubtract / mgClearMinimum); a full cycle solves for
// the correction e of p with bound p_min - p (mgShiftMinimum), restricting the
// bound down by the children's maximum (mgDownsampleMinimum); the coarsest
// level runs projected Gauss-Seidel sweeps until its projected residual
// (mgSolveCoarsest's fixed-point residual) falls below the tolerance or the
// sweep cap is reached.
#pragma once

#include "solids.cuh"

namespace fpp {

constexpr float kNoBound = -3.402823e38f;   // p_min of an unbounded cell (the reference's -FLT_MAX)

// Level-0 lower bound of cell i: 0 on a solid cell that is a liquid unknown.
__device__ __forceinline__ float lcp_base_bound(const InstDev& I, long long i) {
  return (I.lv[0].label[i] && !(clamp01(I.open[i]) > kSolidCell)) ? 0.0f : kNoBound;
}

// (A v)_i on level 0 (face-weighted, unit axis weights), v zero on air.
__device__ __forceinline__ float lcp_apply0(const LevelDev& L, const float* v, int x, int y, int z, long long i) {
  const int sy = L.nx, sz = L.nx * L.ny;
  const float* ff = L.ff;
  const long long n = L.n;
  const float s = d4sum6(x > 0 ? face_w(ff, n, 0, i - 1, 1.0f) * v[i - 1] : 0.0f,
                         x + 1 < L.nx ? face_w(ff, n, 0, i, 1.0f) * v[i + 1] : 0.0f,
                         y > 0 ? face_w(ff, n, 1, i - sy, 1.0f) * v[i - sy] : 0.0f,
                         y + 1 < L.ny ? face_w(ff, n, 1, i, 1.0f) * v[i + sy] : 0.0f,
                         z > 0 ? face_w(ff, n, 2, i - sz, 1.0f) * v[i - sz] : 0.0f,
                         z + 1 < L.nz ? face_w(ff, n, 2, i, 1.0f) * v[i + sz] : 0.0f);
  return L.diag[i] * v[i] - s;
}

// Start of the solve: rhs0 = b, the base bound, z0 = the previous pressure
// (warm) or 0; the CG scalars are not used (sigma 1: no rescaling between
// levels), and the solve runs unless the input was not finite.
__global__ void k_lcp_init(const InstDev* insts, const Tile* tiles, int ntiles, int warm) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    const LevelDev& L = I.lv[0];
    float* z = static_cast<float*>(L.z);
    float* r = static_cast<float*>(L.rhs);
    int x, y, zz, i;
    for (TileIt it(tl.tile, L.nx, L.ny, L.nz, L.depth); it.next(x, y, zz, i);) {
      const bool liq = L.label[i] != 0;
      r[i] = liq ? I.b[i] : 0.0f;
      L.pmin[i] = lcp_base_bound(I, i);
      z[i] = (warm && liq) ? fmaxf(I.x[i] + I.xlo[i], L.pmin[i]) : 0.0f;
    }
    if (t == 0 && threadIdx.x == 0) {
      Ctrl* c = I.ctrl;
      c->sigma = 1.0;
      c->done = c->status == FLUID_PP_NONFINITE ? 1 : 0;
    }
  }
}

// Full cycle, begin (fullCycle mg.ts:539-549): keep p in x, rhs0 = b - A p,
// bound of the correction p_min - p.
__global__ void k_lcp_fc_begin(const InstDev* insts, const Tile* tiles, int ntiles) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    if (I.ctrl->done) continue;
    const LevelDev& L = I.lv[0];
    const float* z = static_cast<const float*>(L.z);
    float* r = static_cast<float*>(L.rhs);
    int x, y, zz, i;
    for (TileIt it(tl.tile, L.nx, L.ny, L.nz, L.depth); it.next(x, y, zz, i);) {
      const bool liq = L.label[i] != 0;
      const float p = z[i];
      I.x[i] = p;
      r[i] = liq ? I.b[i] - lcp_apply0(L, z, x, y, zz, i) : 0.0f;
      const float base = lcp_base_bound(I, i);
      L.pmin[i] = base == kNoBound ? kNoBound : base - p;
    }
  }
}

// Full cycle, end (mgAddPressure): p = kept p + correction; rhs0 = b and the
// base bound again.
__global__ void k_lcp_fc_end(const InstDev* insts, const Tile* tiles, int ntiles) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    if (I.ctrl->done) continue;
    const LevelDev& L = I.lv[0];
    float* z = static_cast<float*>(L.z);
    float* r = static_cast<float*>(L.rhs);
    int x, y, zz, i;
    for (TileIt it(tl.tile, L.nx, L.ny, L.nz, L.depth); it.next(x, y, zz, i);) {
      const bool liq = L.label[i] != 0;
      z[i] = liq ? I.x[i] + z[i] : 0.0f;
      r[i] = liq ? I.b[i] : 0.0f;
      L.pmin[i] = lcp_base_bound(I, i);
    }
  }
}

// Bound of level l + 1 from level l: mode 0 max over the children of
// (p_min - z) (mgDownsampleSubtract), 1 max of the children's p_min
// (mgDownsampleMinimum), 2 unbounded (mgClearMinimum).  The children are the
// fine-child map of the level-set coarsening.
template <class TZ>
__global__ void k_lcp_bound_down(const InstDev* insts, const Tile* tiles, int ntiles, int level, int mode) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    if (I.ctrl->done) continue;
    const LevelDev& F = I.lv[level];
    const LevelDev& C = I.lv[level + 1];
    const TZ* zf = static_cast<const TZ*>(F.z);
    int x, y, z, i;
    for (TileIt it(tl.tile, C.nx, C.ny, C.nz, C.depth); it.next(x, y, z, i);) {
      float b = kNoBound;
      if (mode != 2) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const int ox = c & 1, oy = (c >> 1) & 1, oz = (c >> 2) & 1;
          const int fx = min(C.sx * x + ox * (C.sx - 1), F.nx - 1);
          const int fy = min(C.sy * y + oy * (C.sy - 1), F.ny - 1);
          const int fz = min(C.sz * z + oz * (C.sz - 1), F.nz - 1);
          const long long f = fx + (long long)F.nx * (fy + (long long)F.ny * fz);
          const float pm = F.pmin[f];
          b = fmaxf(b, mode == 0 && pm != kNoBound ? pm - tof(zf[f]) : pm);
        }
      }
      C.pmin[i] = b;
    }
  }
}

// The coarsest level (mgSolveCoarsest, mg.wgsl.ts:404-471): projected red-black
// Gauss-Seidel from z = 0 in float64, one CTA per instance, until the largest
// projected fixed-point residual is at most tol times the largest |rhs| or
// after `cap` sweeps.  A row's projected residual is |r| away from the bound
// and gap * diag where the projection to the bound absorbs r (r < 0 and
// -r >= gap * diag, gap = p - p_min).
template <class T>
__global__ void __launch_bounds__(kMaxCoarse) k_lcp_coarse(const InstDev* insts, const int* list, int cap, double tol) {
  const InstDev& I = insts[list[blockIdx.x]];
  if (I.ctrl->done) return;
  const LevelDev& L = I.lv[I.nlev - 1];
  const int m = int(L.n);
  __shared__ double zs[kMaxCoarse], rs[kMaxCoarse], dg[kMaxCoarse], pm[kMaxCoarse], w[6][kMaxCoarse];
  __shared__ int nb[6][kMaxCoarse];
  __shared__ unsigned char lab[kMaxCoarse];
  __shared__ double worst, bmax;
  const int i = threadIdx.x;
  int x = 0, y = 0, z = 0;
  if (i < m) {
    decode(i, L.nx, L.ny, x, y, z);
    lab[i] = L.label[i];
    rs[i] = tof(static_cast<const T*>(L.rhs)[i]);
    dg[i] = tof(static_cast<const T*>(L.diagT)[i]);
    pm[i] = L.pmin[i];
    zs[i] = 0.0;
    const int sy = L.nx, sz = L.nx * L.ny;
    const bool in[6] = {x > 0, x + 1 < L.nx, y > 0, y + 1 < L.ny, z > 0, z + 1 < L.nz};
    const int j[6] = {i - 1, i + 1, i - sy, i + sy, i - sz, i + sz};
    const int f[6] = {i - 1, i, i - sy, i, i - sz, i};
    const float wa[3] = {L.wx, L.wy, L.wz};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      nb[k][i] = in[k] ? j[k] : i;
      w[k][i] = in[k] ? double(face_w(L.ff, L.n, k / 2, f[k], wa[k / 2])) : 0.0;
    }
  }
  if (i == 0) bmax = 0.0;
  __syncthreads();
  if (i < m && lab[i]) atomicMax(reinterpret_cast<unsigned long long*>(&bmax), __double_as_longlong(fabs(rs[i])));
  __syncthreads();
  const double limit = tol * bmax;
  auto nsum = [&](int c) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) s += lab[nb[k][c]] && nb[k][c] != c ? w[k][c] * zs[nb[k][c]] : 0.0;
    return s;
  };
  for (int sweep = 0; sweep < cap; ++sweep) {
    for (int colour = 0; colour < 2; ++colour) {
      if (i < m && lab[i] && ((x + y + z) & 1) == colour && dg[i] > 0.0) zs[i] = fmax((rs[i] + nsum(i)) / dg[i], pm[i]);
      __syncthreads();
    }
    if (i == 0) worst = 0.0;
    __syncthreads();
    if (i < m && lab[i] && dg[i] > 0.0) {
      const double r = rs[i] - (dg[i] * zs[i] - nsum(i));
      const double gap = fmax(0.0, zs[i] - pm[i]);
      const double proj = (r < 0.0 && -r >= gap * dg[i]) ? gap * dg[i] : fabs(r);
      atomicMax(reinterpret_cast<unsigned long long*>(&worst), __double_as_longlong(proj));
    }
    __syncthreads();
    const bool stop = worst <= limit;   // non-negative doubles order like their bits
    __syncthreads();
    if (stop) break;
  }
  if (i < m) static_cast<T*>(L.z)[i] = fromf<T>(lab[i] ? float(zs[i]) : 0.0f);
}

// End of the solve: the pressure in x (xlo = 0), and the projected fixed-point
// residual of level 0 against b (mgMeasureFineResidual): per tile its sum of
// squares and maximum; the instance's last tile publishes them as the
// receipt's true residual.
__global__ void __launch_bounds__(kThreads) k_lcp_measure(const InstDev* insts, const Tile* tiles, int ntiles,
                                                          int cycles) {
  __shared__ double sh[32];
  __shared__ int flag;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    Ctrl* c = I.ctrl;
    const LevelDev& L = I.lv[0];
    const float* z = static_cast<const float*>(L.z);
    const bool run = !c->done;
    double ss = 0.0, mx = 0.0;
    int x, y, zz, i;
    for (TileIt it(tl.tile, L.nx, L.ny, L.nz, L.depth); it.next(x, y, zz, i);) {
      if (!run) continue;
      const bool liq = L.label[i] != 0;
      I.x[i] = liq ? z[i] : 0.0f;
      I.xlo[i] = 0.0f;
      if (!liq || !(L.diag[i] > 0.0f)) continue;
      const double r = double(I.b[i]) - double(lcp_apply0(L, z, x, y, zz, i));
      const double gap = fmax(0.0, double(z[i]) - double(L.pmin[i]));
      const double d = L.diag[i];
      const double proj = (r < 0.0 && -r >= gap * d) ? gap * d : fabs(r);
      ss += proj * proj;
      mx = fmax(mx, proj);
    }
    const double a0 = block_sum(ss, sh), a1 = block_max(mx, sh);
    const int nt0 = I.ntiles0;
    if (threadIdx.x == 0) {
      I.partial[tl.tile] = a0;
      I.partial[nt0 + tl.tile] = a1;
    }
    if (arrive_last(&c->arrive[kStTrue], nt0, &flag)) {
      const double s = gather_slot(I.partial, 0, nt0, 0, sh);
      const double m = gather_slot(I.partial, 1, nt0, 1, sh);
      if (threadIdx.x == 0 && run) {
        c->rr_true = s;
        c->rr = s;
        c->rmax = m;
        c->iter = cycles;
        c->done = 1;
        c->converged = 1;
        c->status = FLUID_PP_OK;
      }
    }
  }
}

}  // namespace fpp
