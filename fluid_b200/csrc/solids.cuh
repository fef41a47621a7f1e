// Embedded solids on the uniform grid (cut cells).
//
// A handle with embedded solids carries, on the finest level, each cell's open
// (non-solid) volume fraction V_i, the open fraction V_f of each MAC face's
// dual cell (the geometric quantity CM11a's V_{i+1/2} names,
// webgpu-uniform-reference.wgsl.ts:530-556) and the solids' normal velocity on
// each face.  The system stays A = G^T W G / theta with the face weight W_f =
// V_f (the atlas's pressureDualOpenFraction, sparse-atlas-composite-
// projection.ts:506-526 and 1075-1080), zero for a closed face (V_f <= 1e-6,
// mgCoefficientRaw mg.wgsl.ts:108):
//  * density rho' = rho / V_i, continued by the maximum of the open neighbours'
//    rho' into cells with V_i <= 1e-5 (pressureDensity, reference.wgsl.ts:
//    213-233); phi = 0.5 - rho' (finest-cell units); a cell is a liquid unknown
//    when rho' > 0.5 and at least one of its faces is open (a cell with every
//    face closed has an empty row; the reference's smoother keeps it at p = 0,
//    mg.wgsl.ts:341); on coarse levels a liquid cell whose faces are all
//    closed is dropped from the system the same way (k_bake_diag);
//  * b_i = -(sum over axes of (W+ u+ - W- u-) + (W+ - V_i) us+ - (W- - V_i) us-)
//    + q(rho') (divergenceAt, reference.wgsl.ts:1010-1024, Eqs. 8-10 of CM11a,
//    in finest-cell units; the volume correction of cm12-numerics.ts:127-138 on
//    rho');
//  * coarse levels: each face fraction is the mean of the eight children's
//    (mgDownsampleTopology, mg.wgsl.ts:170-183), folded in mgD4Sum8 order;
//  * projection: u_f -= (p_j - p_i) / theta on open faces with a liquid side,
//    u_f = us_f on closed faces (project, reference.wgsl.ts:1052-1099).
// Domain walls stay closed as everywhere else in this library.
#pragma once

#include "kernels.cuh"

namespace fpp {

__device__ __forceinline__ float clamp01(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }

// The weight a face's open fraction gives it (closed faces weigh nothing).
__device__ __forceinline__ float open_weight(float f) { return f > kClosedFace ? f : 0.0f; }

// rho' of cell i at (x, y, z): rho / V for an open cell, else the largest rho'
// of its open neighbours (0 when none).
__device__ __forceinline__ float solid_density(const InstDev& I, int x, int y, int z, long long i) {
  const float* __restrict__ open = I.open;
  const float* __restrict__ vof = I.vof;
  const float v = clamp01(open[i]);
  if (v > kSolidCell) return __fdiv_rn(vof[i], v);
  const int nx = I.nx, ny = I.ny, nz = I.nz;
  const long long sy = nx, sz = (long long)nx * ny;
  float best = 0.0f;
  auto take = [&](bool inside, long long j) {
    if (!inside) return;
    const float vj = clamp01(open[j]);
    if (vj > kSolidCell) best = fmaxf(best, __fdiv_rn(vof[j], vj));
  };
  take(x > 0, i - 1);
  take(x + 1 < nx, i + 1);
  take(y > 0, i - sy);
  take(y + 1 < ny, i + sy);
  take(z > 0, i - sz);
  take(z + 1 < nz, i + sz);
  return best;
}

// The weighted flux divergence of cell i (W-weighted face velocities plus the
// solids' terms) for the velocity arrays U, V, W.
__device__ __forceinline__ float solid_divergence(const InstDev& I, int x, int y, int z, long long i, const float* U,
                                                  const float* V, const float* W) {
  const int nx = I.nx, ny = I.ny, nz = I.nz;
  const long long uS = nx + 1, vS = ny + 1, sz = (long long)nx * ny;
  const float vi = clamp01(I.open[i]);
  const float* const* fv = I.fv;
  const float* const* us = I.us;
  auto solid_v = [&](int a, long long f) { return us[a] ? us[a][f] : 0.0f; };
  // one axis: faces fm (low) and fp (high); a missing face (wall) has weight 0
  auto axis = [&](int a, bool hm, long long fm, bool hp, long long fp, const float* vel) {
    const float wm = hm ? open_weight(clamp01(fv[a][fm])) : 0.0f;
    const float wp = hp ? open_weight(clamp01(fv[a][fp])) : 0.0f;
    const float um = hm ? vel[fm] : 0.0f, up = hp ? vel[fp] : 0.0f;
    const float sm = hm ? solid_v(a, fm) : 0.0f, sp = hp ? solid_v(a, fp) : 0.0f;
    return (wp * up - wm * um) + ((wp - vi) * sp - (wm - vi) * sm);
  };
  const long long urow = uS * (y + (long long)ny * z);
  const long long vcol = x + (long long)nx * vS * z;
  const float fx = axis(0, x > 0, urow + x, x + 1 < nx, urow + x + 1, U);
  const float fy = axis(1, y > 0, vcol + (long long)nx * y, y + 1 < ny || I.open_top, vcol + (long long)nx * (y + 1), V);
  const float fz = axis(2, z > 0, i, z + 1 < nz, i + sz, W);
  return (fx + fz) + fy;
}

// Whether cell i has an open face (a pressure unknown needs one: with every face
// closed its row is empty, and the reference's smoother leaves such a cell at
// p = 0, mgSmoothColour mg.wgsl.ts:341).
__device__ __forceinline__ bool has_open_face(const InstDev& I, int x, int y, int z, long long i) {
  const int nx = I.nx, ny = I.ny, nz = I.nz;
  const long long uS = nx + 1, vS = ny + 1, sz = (long long)nx * ny;
  const long long urow = uS * (y + (long long)ny * z), vcol = x + (long long)nx * vS * z;
  auto open = [&](int a, long long f) { return open_weight(clamp01(I.fv[a][f])) > 0.0f; };
  return (x > 0 && open(0, urow + x)) || (x + 1 < nx && open(0, urow + x + 1)) ||
         (y > 0 && open(1, vcol + (long long)nx * y)) ||
         ((y + 1 < ny || I.open_top) && open(1, vcol + (long long)nx * (y + 1))) || (z > 0 && open(2, i)) ||
         (z + 1 < nz && open(2, i + sz));
}

// Volume correction (cm12VolumeCorrectionDivergence * h, cm12-numerics.ts:127-138).
__device__ __forceinline__ float volume_correction(float rho, float hdt) {
  return rho > 1.0f ? fminf(fminf(0.5f * (rho - 1.0f), 1.0f), hdt) : 0.0f;
}

// Level 0 with embedded solids: labels, level set and right-hand side.
__global__ void __launch_bounds__(kThreads) k_label_rhs_solid(const InstDev* insts, const Tile* tiles, int ntiles,
                                                              int warm) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    const LevelDev& L = I.lv[0];
    int liquid = 0, air = 0, top = 0, bad = 0;
    const int nx = I.nx, ny = I.ny, nz = I.nz;
    const long long uS = nx + 1, vS = ny + 1, sz = (long long)nx * ny;
    const float hdt = I.h / I.dt;
    int x, y, z, i;
    for (TileIt it(tl.tile, nx, ny, nz, L.depth); it.next(x, y, z, i);) {
      const float r = solid_density(I, x, y, z, i);
      const bool dense = r > 0.5f;
      const bool liq = dense && has_open_face(I, x, y, z, i);   // a liquid cell with every face closed is no unknown
      L.label[i] = liq ? 1 : 0;
      L.phi[i] = 0.5f - r;
      const long long urow = uS * (y + (long long)ny * z), vcol = x + (long long)nx * vS * z;
      bad |= !(isfinite(I.vof[i]) && isfinite(I.open[i]) && isfinite(I.u[urow + x]) && isfinite(I.u[urow + x + 1]) &&
               isfinite(I.v[vcol + (long long)nx * y]) && isfinite(I.v[vcol + (long long)nx * (y + 1)]) &&
               isfinite(I.w[i]) && isfinite(I.w[i + sz]));
      float b = 0.0f;
      if (liq) {
        b = -(solid_divergence(I, x, y, z, i, I.u, I.v, I.w) - volume_correction(r, hdt));
        ++liquid;
        top += (y == ny - 1);
      } else if (!dense) {
        ++air;
      }
      I.b[i] = b;
      if (!(warm && liq)) {
        I.x[i] = 0.0f;
        I.xlo[i] = 0.0f;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      liquid += __shfl_xor_sync(0xffffffffu, liquid, o);
      air += __shfl_xor_sync(0xffffffffu, air, o);
      top += __shfl_xor_sync(0xffffffffu, top, o);
      bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if ((threadIdx.x & 31) == 0) {
      if (liquid) atomicAdd(&I.ctrl->liquid, liquid);
      if (air) atomicAdd(&I.ctrl->air, air);
      if (top) atomicAdd(&I.ctrl->top_liquid, top);
      if (bad) atomicOr(&I.ctrl->nonfinite, 1);
    }
  }
}

// Level-0 face fractions in the level layout (planar +x, +y, +z faces of each
// cell) from the MAC-face arrays: a domain-wall face keeps fraction 1 (it has
// no coupling; the value only enters the coarse levels' means), the open top
// its given fraction.
__global__ void k_solid_faces(InstDev* I) {
  const int nx = I->nx, ny = I->ny, nz = I->nz;
  const long long n = (long long)nx * ny * nz, uS = nx + 1, vS = ny + 1;
  float* ff = const_cast<float*>(I->lv[0].ff);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = int(i % nx);
    const long long yz = i / nx;
    const int y = int(yz % ny), z = int(yz / ny);
    const float fx = x + 1 < nx ? clamp01(I->fv[0][uS * (y + (long long)ny * z) + x + 1]) : 1.0f;
    const long long ftop = x + (long long)nx * (y + 1 + vS * z);
    const float fy = (y + 1 < ny || I->open_top) ? clamp01(I->fv[1][ftop]) : 1.0f;
    const float fz = z + 1 < nz ? clamp01(I->fv[2][i + (long long)nx * ny]) : 1.0f;
    ff[i] = fx;
    ff[n + i] = fy;
    ff[2 * n + i] = fz;
  }
}

// Coarse face fractions of level l: the mean of the eight children's fractions
// per axis (mgDownsampleTopology, mg.wgsl.ts:170-183), folded in mgD4Sum8 order.
__global__ void k_coarsen_faces(InstDev* I, int l) {
  const LevelDev& C = I->lv[l];
  const LevelDev& F = I->lv[l - 1];
  const long long n = C.n;
  float* cf = const_cast<float*>(C.ff);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = int(i % C.nx);
    const long long yz = i / C.nx;
    const int y = int(yz % C.ny), z = int(yz / C.ny);
    long long child[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int ox = c & 1, oy = (c >> 1) & 1, oz = (c >> 2) & 1;
      const int fx = min(C.sx * x + ox * (C.sx - 1), F.nx - 1);
      const int fy = min(C.sy * y + oy * (C.sy - 1), F.ny - 1);
      const int fz = min(C.sz * z + oz * (C.sz - 1), F.nz - 1);
      child[c] = fx + (long long)F.nx * (fy + (long long)F.ny * fz);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float v[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) v[c] = F.ff[a * F.n + child[c]];
      const float y0 = __fadd_rn(__fadd_rn(v[0], v[5]), __fadd_rn(v[1], v[4]));
      const float y1 = __fadd_rn(__fadd_rn(v[2], v[7]), __fadd_rn(v[3], v[6]));
      cf[a * n + i] = __fdiv_rn(__fadd_rn(y0, y1), 8.0f);
    }
  }
}

// Gradient subtract with embedded solids: each cell's +x, +y, +z faces (and the
// low walls).  An open face with a liquid side takes u -= (p_j - p_i) / theta, a
// closed face the solids' velocity, a face with no liquid side 0; pressure in Pa.
__global__ void __launch_bounds__(kThreads) k_grad_solid(const InstDev* insts, const Tile* tiles, int ntiles) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    if (I.ctrl->status == FLUID_PP_NONFINITE) continue;   // fail closed: keep the previous state
    const LevelDev& L = I.lv[0];
    const int nx = I.nx, ny = I.ny, nz = I.nz;
    const long long uS = nx + 1, vS = ny + 1, sz = (long long)nx * ny;
    const double pscale = double(I.pscale);
    auto P = [&](long long j) { return L.label[j] ? double(I.x[j]) + double(I.xlo[j]) : 0.0; };
    // face f of axis a between cells i and j (j < 0: the open top, exterior phi 0.5)
    auto face = [&](int a, long long f, long long i, long long j, float* vel) {
      const float w = open_weight(clamp01(I.fv[a][f]));
      if (w == 0.0f) {
        vel[f] = I.us[a] ? I.us[a][f] : 0.0f;
        return;
      }
      if (j < 0) {
        vel[f] = L.label[i] ? float(double(vel[f]) + P(i) / double(ghost_theta(L.phi[i], 0.5f))) : 0.0f;
        return;
      }
      vel[f] = face_value(L.label[i], L.label[j], L.phi[i], L.phi[j], P(i), P(j), vel[f]);
    };
    int x, y, z, i;
    for (TileIt it(tl.tile, nx, ny, nz, L.depth); it.next(x, y, z, i);) {
      const long long urow = uS * (y + (long long)ny * z), vcol = x + (long long)nx * vS * z;
      if (x + 1 < nx) face(0, urow + x + 1, i, i + 1, I.u);
      else I.u[urow + x + 1] = 0.0f;
      if (x == 0) I.u[urow] = 0.0f;
      if (y + 1 < ny) face(1, vcol + (long long)nx * (y + 1), i, i + nx, I.v);
      else if (I.open_top) face(1, vcol + (long long)nx * (y + 1), i, -1, I.v);
      else I.v[vcol + (long long)nx * (y + 1)] = 0.0f;
      if (y == 0) I.v[vcol] = 0.0f;
      if (z + 1 < nz) face(2, i + sz, i, i + sz, I.w);
      else I.w[i + sz] = 0.0f;
      if (z == 0) I.w[i] = 0.0f;
      I.p_si[i] = float(P(i) * pscale);
    }
  }
}

// Receipts with embedded solids: the weighted divergence (the quantity b
// measures) before and after the projection, per liquid cell.
__global__ void __launch_bounds__(kThreads) k_receipt_solid(const InstDev* insts, const Tile* tiles, int ntiles) {
  __shared__ double sh[4 * 32];
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    const LevelDev& L = I.lv[0];
    const int nx = I.nx, ny = I.ny, nz = I.nz;
    const float hdt = I.h / I.dt;
    double sums[2] = {0, 0}, maxes[2] = {0, 0};   // after, before
    int x, y, z, i;
    for (TileIt it(tl.tile, nx, ny, nz, L.depth); it.next(x, y, z, i);) {
      if (!L.label[i]) continue;
      const float r = solid_density(I, x, y, z, i);
      const double after = double(solid_divergence(I, x, y, z, i, I.u, I.v, I.w)) - double(volume_correction(r, hdt));
      const double before = -double(I.b[i]);
      maxes[0] = fmax(maxes[0], fabs(after));
      sums[0] += after * after;
      maxes[1] = fmax(maxes[1], fabs(before));
      sums[1] += before * before;
    }
    block_folds<2, 2>(sums, maxes, sh);
    if (threadIdx.x == 0) {
      I.partial[0 * I.ntiles0 + tl.tile] = maxes[0];
      I.partial[1 * I.ntiles0 + tl.tile] = sums[0];
      I.partial[2 * I.ntiles0 + tl.tile] = maxes[1];
      I.partial[3 * I.ntiles0 + tl.tile] = sums[1];
    }
  }
}

}  // namespace fpp
