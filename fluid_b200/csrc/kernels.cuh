// Device kernels of the uniform-grid pressure projection (sm_100a).
//
// Every kernel walks a list of work tiles (instance, level, tile) so that the
// same launch serves one solve or a batch of uneven solves.  A tile is kTile
// consecutive cells of one level (x fastest).  Reductions are deterministic:
// each tile writes its float64 partial to its own slot and the last tile of an
// instance to arrive sums the slots in tile order and finalises the scalars.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "../../include/fluid_pp.h"
#include "types.h"

namespace fpp {

struct Tile {
  int inst;
  int level;
  int tile;
  int pad;
};

// ------------------------------------------------------------ storage types
template <class T>
struct St;
template <>
struct St<float> {
  static __device__ __forceinline__ float ld(const void* p, long long i) { return static_cast<const float*>(p)[i]; }
  static __device__ __forceinline__ void st(void* p, long long i, float v) { static_cast<float*>(p)[i] = v; }
};
template <>
struct St<__half> {
  static __device__ __forceinline__ float ld(const void* p, long long i) {
    return __half2float(static_cast<const __half*>(p)[i]);
  }
  static __device__ __forceinline__ void st(void* p, long long i, float v) {
    static_cast<__half*>(p)[i] = __float2half_rn(v);
  }
};
template <>
struct St<__nv_bfloat16> {
  static __device__ __forceinline__ float ld(const void* p, long long i) {
    return __bfloat162float(static_cast<const __nv_bfloat16*>(p)[i]);
  }
  static __device__ __forceinline__ void st(void* p, long long i, float v) {
    static_cast<__nv_bfloat16*>(p)[i] = __float2bfloat16_rn(v);
  }
};

__device__ __forceinline__ void decode(long long i, int nx, int ny, int& x, int& y, int& z) {
  const long long yz = i / nx;
  x = int(i - yz * nx);
  z = int(yz / ny);
  y = int(yz - (long long)z * ny);
}

// cm12GhostFluidTheta (lib/core/cm12-numerics.ts:37-45), epsilon 1e-12.
__device__ __forceinline__ float ghost_theta(float liquid_phi, float air_phi) {
  const float a = fabsf(liquid_phi);
  return fminf(1.0f, fmaxf(0.05f, a / fmaxf(a + fabsf(air_phi), 1e-12f)));
}

// Canonical fold of the six face terms (mgD4Sum6, mg.wgsl.ts:49).
__device__ __forceinline__ float d4sum6(float xm, float xp, float ym, float yp, float zm, float zp) {
  return ((xm + xp) + (zm + zp)) + (ym + yp);
}

// Deterministic block reductions (fixed shuffle tree).  Result valid in warp 0.
__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0;
  if (w == 0) {
    r = l < int(blockDim.x >> 5) ? sh[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  return r;
}
__device__ __forceinline__ double block_max(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0;
  if (w == 0) {
    r = l < int(blockDim.x >> 5) ? sh[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
  }
  __syncthreads();
  return r;
}

// Publish this tile's partials and report whether it is the instance's last.
__device__ __forceinline__ bool arrive_last(unsigned* counter, int total, int* flag) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(counter, 1u);
    *flag = prev == unsigned(total - 1);
    if (*flag) {
      __threadfence();
      *counter = 0u;   // every tile of this instance has arrived: reset for the next launch
    }
  }
  __syncthreads();
  return *flag != 0;
}

// Sum (op 0) or max (op 1) of one slot over all tiles, in tile order.
__device__ __forceinline__ double gather_slot(const double* partial, int slot, int ntiles, int op, double* sh) {
  const volatile double* p = partial + (long long)slot * ntiles;
  double acc = 0;
  for (int t = threadIdx.x; t < ntiles; t += blockDim.x) acc = op ? fmax(acc, p[t]) : acc + p[t];
  return op ? block_max(acc, sh) : block_sum(acc, sh);
}

// ================================================================= setup
// Level 0: labels, level set and right-hand side from the VOF and MAC velocities
// (ref.wgsl.ts:208-242 labelling; divergenceAt :1010-1024 with closed walls
// carrying no flux; mgBuildFinestRhs mg.wgsl.ts:152-167 in finest-cell units).
__global__ void k_label_rhs(const InstDev* insts, const Tile* tiles, int ntiles, int warm) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    const LevelDev& L = I.lv[0];
    int liquid = 0, air = 0, top = 0, bad = 0;
    const long long base = (long long)tl.tile * kTile;
    for (int k = 0; k < kTile / kThreads; ++k) {
      const long long i = base + k * kThreads + threadIdx.x;
      if (i >= L.n) break;
      int x, y, z;
      decode(i, I.nx, I.ny, x, y, z);
      const float rho = I.vof[i];
      const bool liq = rho > 0.5f;
      L.label[i] = liq ? 1 : 0;
      L.phi[i] = 0.5f - rho;
      const long long uS = I.nx + 1, vS = I.ny + 1;
      const float up = I.u[x + 1 + uS * (y + (long long)I.ny * z)];
      const float um = I.u[x + uS * (y + (long long)I.ny * z)];
      const float vp = I.v[x + (long long)I.nx * (y + 1 + vS * z)];
      const float vm = I.v[x + (long long)I.nx * (y + vS * z)];
      const float wp = I.w[i + (long long)I.nx * I.ny];
      const float wm = I.w[i];
      bad |= !(isfinite(rho) && isfinite(up) && isfinite(um) && isfinite(vp) && isfinite(vm) && isfinite(wp) &&
               isfinite(wm));
      float b = 0.0f;
      if (liq) {
        const float fxp = x + 1 < I.nx ? up : 0.0f, fxm = x > 0 ? um : 0.0f;
        const float fyp = (y + 1 < I.ny || I.open_top) ? vp : 0.0f, fym = y > 0 ? vm : 0.0f;
        const float fzp = z + 1 < I.nz ? wp : 0.0f, fzm = z > 0 ? wm : 0.0f;
        const float div = ((fxp - fxm) + (fzp - fzm)) + (fyp - fym);
        float q = 0.0f;   // cm12VolumeCorrectionDivergence * h (cm12-numerics.ts:127-138)
        if (rho > 1.0f) q = fminf(fminf(0.5f * (rho - 1.0f), 1.0f), I.h / I.dt);
        b = -(div - q);
        ++liquid;
        top += (y == I.ny - 1);
      } else {
        ++air;
      }
      I.b[i] = b;
      if (!(warm && liq)) I.x[i] = 0.0f;
    }
    // integer counts are order independent
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

// Coarse level set (mgDownsampleTopology, mg.wgsl.ts:169-195): mean of the eight
// children, or the mean of the non-negative children when the block is mixed and
// the destination is one of the two finest coarse levels; folded in mgD4Sum8 order.
__global__ void k_coarsen_phi(const InstDev* insts, const Tile* tiles, int ntiles) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    const LevelDev& C = I.lv[tl.level];
    const LevelDev& F = I.lv[tl.level - 1];
    const long long base = (long long)tl.tile * kTile;
    for (int k = 0; k < kTile / kThreads; ++k) {
      const long long i = base + k * kThreads + threadIdx.x;
      if (i >= C.n) break;
      int x, y, z;
      decode(i, C.nx, C.ny, x, y, z);
      float ph[8], ps[8], pf[8], nf[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int ox = c & 1, oy = (c >> 1) & 1, oz = (c >> 2) & 1;
        const int fx = min(C.sx * x + ox * (C.sx - 1), F.nx - 1);
        const int fy = min(C.sy * y + oy * (C.sy - 1), F.ny - 1);
        const int fz = min(C.sz * z + oz * (C.sz - 1), F.nz - 1);
        const float p = F.phi[fx + (long long)F.nx * (fy + (long long)F.ny * fz)];
        ph[c] = p;
        ps[c] = p >= 0.0f ? p : 0.0f;
        pf[c] = p >= 0.0f ? 1.0f : 0.0f;
        nf[c] = p >= 0.0f ? 0.0f : 1.0f;
      }
      auto fold = [](const float* v) {
        const float y0 = __fadd_rn(__fadd_rn(v[0], v[5]), __fadd_rn(v[1], v[4]));
        const float y1 = __fadd_rn(__fadd_rn(v[2], v[7]), __fadd_rn(v[3], v[6]));
        return __fadd_rn(y0, y1);
      };
      const float sum = fold(ph), pos = fold(ps), npos = fold(pf), nneg = fold(nf);
      const bool mixed = npos > 0.0f && nneg > 0.0f;
      const float c = (mixed && tl.level <= 2) ? __fdiv_rn(pos, fmaxf(npos, 1.0f)) : __fdiv_rn(sum, 8.0f);
      C.phi[i] = c;
      C.label[i] = c < 0.0f ? 1 : 0;
    }
  }
}

// Diagonal of every level (mgCoefficientRaw / mgBakeCoefficients, mg.wgsl.ts:93-115,
// 299-307, Neumann walls, no embedded solids): face to liquid w_a, face to air
// w_a / theta, open top w_y / theta(phi, h_y / 2).
template <class T>
__global__ void k_bake_diag(const InstDev* insts, const Tile* tiles, int ntiles) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    const LevelDev& L = I.lv[tl.level];
    const float norm = 1.0f / L.wmax;
    const float wx = L.wx * L.wmax, wy = L.wy * L.wmax, wz = L.wz * L.wmax;
    const long long base = (long long)tl.tile * kTile;
    for (int k = 0; k < kTile / kThreads; ++k) {
      const long long i = base + k * kThreads + threadIdx.x;
      if (i >= L.n) break;
      float d = 0.0f;
      if (L.label[i]) {
        int x, y, z;
        decode(i, L.nx, L.ny, x, y, z);
        const float ph = L.phi[i];
        const long long sy = L.nx, sz = (long long)L.nx * L.ny;
        auto term = [&](bool inside, long long j, float w) -> float {
          if (!inside) return 0.0f;
          return L.label[j] ? w : w / ghost_theta(ph, L.phi[j]);
        };
        const float xm = term(x > 0, i - 1, wx), xp = term(x + 1 < L.nx, i + 1, wx);
        const float ym = term(y > 0, i - sy, wy);
        float yp = term(y + 1 < L.ny, i + sy, wy);
        if (y + 1 == L.ny && I.open_top) yp = wy / ghost_theta(ph, L.ext_phi);
        const float zm = term(z > 0, i - sz, wz), zp = term(z + 1 < L.nz, i + sz, wz);
        d = d4sum6(xm, xp, ym, yp, zm, zp);
      }
      L.diag[i] = d;
      St<T>::st(L.diagT, i, d * norm);
    }
  }
}

// ================================================================= CG scalars
enum Stage { kStInit = 0, kStGamma = 1, kStSpmv = 2, kStUpdate = 3, kStTrue = 4, kStReceipt = 5 };

__device__ __forceinline__ void set_sigma(Ctrl* c, double rr) {
  const double per = rr / double(c->liquid > 0 ? c->liquid : 1);
  c->sigma = per > 1e-300 ? 1.0 / sqrt(per) : 1.0;
}

// r = b - A x (x already masked to liquid), bb, sums for the nullspace.
__global__ void k_cg_init(const InstDev* insts, const Tile* tiles, int ntiles, double rel_tol, double abs_tol,
                          int max_iter, int true_every, int warm) {
  __shared__ double sh[32];
  __shared__ int flag;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    Ctrl* c = I.ctrl;
    const LevelDev& L = I.lv[0];
    float* r = static_cast<float*>(L.rhs);
    double sbb = 0, sb = 0, srr = 0;
    const long long base = (long long)tl.tile * kTile;
    const long long sy = L.nx, sz = (long long)L.nx * L.ny;
    for (int k = 0; k < kTile / kThreads; ++k) {
      const long long i = base + k * kThreads + threadIdx.x;
      if (i >= L.n) break;
      const float b = I.b[i];
      float rv = b;
      if (warm && L.label[i]) {
        int x, y, z;
        decode(i, L.nx, L.ny, x, y, z);
        const float* X = I.x;
        auto nb = [&](bool in, long long j) { return (in && L.label[j]) ? X[j] : 0.0f; };
        const float s = d4sum6(nb(x > 0, i - 1), nb(x + 1 < L.nx, i + 1), nb(y > 0, i - sy),
                               nb(y + 1 < L.ny, i + sy), nb(z > 0, i - sz), nb(z + 1 < L.nz, i + sz));
        rv = float(double(b) - (double(L.diag[i]) * X[i] - double(s)));
      }
      r[i] = rv;
      sbb += double(b) * b;
      sb += b;
      srr += double(rv) * rv;
    }
    double a0 = block_sum(sbb, sh), a1 = block_sum(sb, sh), a2 = block_sum(srr, sh);
    if (threadIdx.x == 0) {
      I.partial[0 * I.ntiles0 + tl.tile] = a0;
      I.partial[1 * I.ntiles0 + tl.tile] = a1;
      I.partial[2 * I.ntiles0 + tl.tile] = a2;
    }
    if (arrive_last(&c->arrive[kStInit], I.ntiles0, &flag)) {
      const double bb = gather_slot(I.partial, 0, I.ntiles0, 0, sh);
      const double bs = gather_slot(I.partial, 1, I.ntiles0, 0, sh);
      const double rr = gather_slot(I.partial, 2, I.ntiles0, 0, sh);
      if (threadIdx.x == 0) {
        c->anchored = (c->air > 0) || (I.open_top && c->top_liquid > 0);
        const double nliq = double(c->liquid > 0 ? c->liquid : 1);
        c->bmean = c->anchored ? 0.0 : bs / nliq;
        c->bb = bb - (c->anchored ? 0.0 : nliq * c->bmean * c->bmean);
        c->rr = rr - (c->anchored ? 0.0 : nliq * c->bmean * c->bmean);
        if (c->bb < 0) c->bb = 0;
        if (c->rr < 0) c->rr = 0;
        const double thr = fmax(abs_tol, rel_tol * sqrt(c->bb));
        c->thr2 = thr * thr;
        c->iter = 0;
        c->max_iter = max_iter;
        c->true_every = true_every;
        c->first = 1;
        c->candidate = 0;
        c->converged = 0;
        c->done = 0;
        c->status = FLUID_PP_OK;
        c->rr_true = c->rr;
        set_sigma(c, c->rr);
        if (c->nonfinite) {
          c->done = 1;
          c->status = FLUID_PP_NONFINITE;
        } else if (c->liquid == 0 || c->rr <= c->thr2) {
          c->done = 1;   // nothing to solve, or the initial guess already satisfies the tolerance
          c->converged = 1;
        }
      }
    }
  }
}

// Nullspace projection of b and r for a finest system without Dirichlet contact
// (sparse-atlas-composite-projection.ts projectNullspace :1194-1213).
__global__ void k_project_init(const InstDev* insts, const Tile* tiles, int ntiles) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    const Ctrl* c = I.ctrl;
    if (c->anchored || c->done) continue;
    const LevelDev& L = I.lv[0];
    float* r = static_cast<float*>(L.rhs);
    const float m = float(c->bmean);
    const long long base = (long long)tl.tile * kTile;
    for (int k = 0; k < kTile / kThreads; ++k) {
      const long long i = base + k * kThreads + threadIdx.x;
      if (i >= L.n) break;
      if (!L.label[i]) continue;
      I.b[i] -= m;
      r[i] -= m;
    }
  }
}

// ================================================================= V-cycle
// One colour pass of red-black Gauss-Seidel on the normalised level operator
// (mgSmoothColour, mg.wgsl.ts:325-344, without the p_min projection).  With
// zero_init the pass starts from z = 0 and also clears the other colour.
template <class TZ, class TR, class TD>
__global__ void k_smooth(const InstDev* insts, const Tile* tiles, int ntiles, int level, int colour, int zero_init) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    if (I.ctrl->done) continue;
    const LevelDev& L = I.lv[level];
    const long long base = (long long)tl.tile * kTile;
    const long long sy = L.nx, sz = (long long)L.nx * L.ny;
    for (int k = 0; k < kTile / kThreads; ++k) {
      const long long i = base + k * kThreads + threadIdx.x;
      if (i >= L.n) break;
      int x, y, z;
      decode(i, L.nx, L.ny, x, y, z);
      if (((x + y + z) & 1) != colour) {
        if (zero_init) St<TZ>::st(L.z, i, 0.0f);
        continue;
      }
      if (!L.label[i]) {
        St<TZ>::st(L.z, i, 0.0f);
        continue;
      }
      float s = 0.0f;
      if (!zero_init) {
        auto nb = [&](bool in, long long j, float w) { return in ? w * St<TZ>::ld(L.z, j) : 0.0f; };
        s = d4sum6(nb(x > 0, i - 1, L.wx), nb(x + 1 < L.nx, i + 1, L.wx), nb(y > 0, i - sy, L.wy),
                   nb(y + 1 < L.ny, i + sy, L.wy), nb(z > 0, i - sz, L.wz), nb(z + 1 < L.nz, i + sz, L.wz));
      }
      St<TZ>::st(L.z, i, (St<TR>::ld(L.rhs, i) + s) / St<TD>::ld(L.diagT, i));
    }
  }
}

// res = scale * (rhs - A z) on liquid cells (mgResidual, mg.wgsl.ts:197-205).
// On level 0 the residual is scaled by sigma so half-precision levels stay in range.
template <class TZ, class TR, class TD, class TS>
__global__ void k_residual(const InstDev* insts, const Tile* tiles, int ntiles, int level) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    if (I.ctrl->done) continue;
    const LevelDev& L = I.lv[level];
    const float scale = level == 0 ? float(I.ctrl->sigma) : 1.0f;
    const long long base = (long long)tl.tile * kTile;
    const long long sy = L.nx, sz = (long long)L.nx * L.ny;
    for (int k = 0; k < kTile / kThreads; ++k) {
      const long long i = base + k * kThreads + threadIdx.x;
      if (i >= L.n) break;
      float r = 0.0f;
      if (L.label[i]) {
        int x, y, z;
        decode(i, L.nx, L.ny, x, y, z);
        auto nb = [&](bool in, long long j, float w) { return in ? w * St<TZ>::ld(L.z, j) : 0.0f; };
        const float s = d4sum6(nb(x > 0, i - 1, L.wx), nb(x + 1 < L.nx, i + 1, L.wx), nb(y > 0, i - sy, L.wy),
                               nb(y + 1 < L.ny, i + sy, L.wy), nb(z > 0, i - sz, L.wz), nb(z + 1 < L.nz, i + sz, L.wz));
        r = scale * (St<TR>::ld(L.rhs, i) - (St<TD>::ld(L.diagT, i) * St<TZ>::ld(L.z, i) - s));
      }
      St<TS>::st(L.res, i, r);
    }
  }
}

// Weight of coarse cell c in the renormalised trilinear stencil of fine cell f
// (mgTrilinearPressure, mg.wgsl.ts:217-241) along an axis that coarsened by 2.
__device__ __forceinline__ float p1d(int f, int c, int nc) {
  const int d = f - 2 * c;
  if (d == 0) return c == 0 ? 1.0f : 0.75f;
  if (d == 1) return c + 1 == nc ? 1.0f : 0.75f;
  return 0.25f;   // d == -1 or d == 2
}

// rhs_{l+1} = to_coarse * P^T res_l / 2^k (the transpose of the prolongation, so
// the V-cycle is a symmetric preconditioner); coarse air cells get zero.
template <class TS>
__global__ void k_restrict(const InstDev* insts, const Tile* tiles, int ntiles, int level) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    if (I.ctrl->done) continue;
    const LevelDev& F = I.lv[level];
    const LevelDev& C = I.lv[level + 1];
    const float scale = F.to_coarse / float((C.sx == 2 ? 2 : 1) * (C.sy == 2 ? 2 : 1) * (C.sz == 2 ? 2 : 1));
    const long long base = (long long)tl.tile * kTile;
    for (int k = 0; k < kTile / kThreads; ++k) {
      const long long i = base + k * kThreads + threadIdx.x;
      if (i >= C.n) break;
      float acc = 0.0f;
      if (C.label[i]) {
        int X, Y, Z;
        decode(i, C.nx, C.ny, X, Y, Z);
        const int x0 = C.sx == 2 ? max(2 * X - 1, 0) : X, x1 = C.sx == 2 ? min(2 * X + 2, F.nx - 1) : X;
        const int y0 = C.sy == 2 ? max(2 * Y - 1, 0) : Y, y1 = C.sy == 2 ? min(2 * Y + 2, F.ny - 1) : Y;
        const int z0 = C.sz == 2 ? max(2 * Z - 1, 0) : Z, z1 = C.sz == 2 ? min(2 * Z + 2, F.nz - 1) : Z;
        for (int fz = z0; fz <= z1; ++fz) {
          const float wz = C.sz == 2 ? p1d(fz, Z, C.nz) : 1.0f;
          for (int fy = y0; fy <= y1; ++fy) {
            const float wy = wz * (C.sy == 2 ? p1d(fy, Y, C.ny) : 1.0f);
            const long long row = (long long)F.nx * (fy + (long long)F.ny * fz);
            for (int fx = x0; fx <= x1; ++fx) {
              const float wx = C.sx == 2 ? p1d(fx, X, C.nx) : 1.0f;
              acc += wy * wx * St<TS>::ld(F.res, row + fx);
            }
          }
        }
        acc *= scale;
      }
      St<TS>::st(C.rhs, i, acc);
    }
  }
}

__device__ __forceinline__ int taps1d(int f, int stride, int nc, int* c, float* w) {
  if (stride == 1) {
    c[0] = f;
    w[0] = 1.0f;
    return 1;
  }
  const int k = f >> 1;
  int a, b;
  float wa, wb;
  if ((f & 1) == 0) { a = k - 1; wa = 0.25f; b = k; wb = 0.75f; }
  else { a = k; wa = 0.75f; b = k + 1; wb = 0.25f; }
  int n = 0;
  if (a >= 0 && a < nc) { c[n] = a; w[n] = wa; ++n; }
  if (b >= 0 && b < nc) { c[n] = b; w[n] = wb; ++n; }
  if (n == 1) w[0] = 1.0f;
  return n;
}

// z_l += P z_{l+1} on liquid cells (mgProlongateAdd, mg.wgsl.ts:243-246);
// from level 1 into level 0 the sigma scaling is undone.
template <class TZF, class TZC>
__global__ void k_prolong(const InstDev* insts, const Tile* tiles, int ntiles, int level) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    if (I.ctrl->done) continue;
    const LevelDev& F = I.lv[level];
    const LevelDev& C = I.lv[level + 1];
    const float unscale = level == 0 ? float(1.0 / I.ctrl->sigma) : 1.0f;
    const long long base = (long long)tl.tile * kTile;
    for (int k = 0; k < kTile / kThreads; ++k) {
      const long long i = base + k * kThreads + threadIdx.x;
      if (i >= F.n) break;
      if (!F.label[i]) continue;
      int x, y, z;
      decode(i, F.nx, F.ny, x, y, z);
      int cx[2], cy[2], cz[2];
      float wx[2], wy[2], wz[2];
      const int nxx = taps1d(x, C.sx, C.nx, cx, wx);
      const int nyy = taps1d(y, C.sy, C.ny, cy, wy);
      const int nzz = taps1d(z, C.sz, C.nz, cz, wz);
      float s = 0.0f;
      for (int c2 = 0; c2 < nzz; ++c2)
        for (int c1 = 0; c1 < nyy; ++c1)
          for (int c0 = 0; c0 < nxx; ++c0)
            s += wx[c0] * wy[c1] * wz[c2] *
                 St<TZC>::ld(C.z, cx[c0] + (long long)C.nx * (cy[c1] + (long long)C.ny * cz[c2]));
      St<TZF>::st(F.z, i, St<TZF>::ld(F.z, i) + s * unscale);
    }
  }
}

// ================================================================= CG kernels
// gamma = r . (z - zmean) with float64 accumulation; beta from the previous gamma.
__global__ void k_dot_rz(const InstDev* insts, const Tile* tiles, int ntiles) {
  __shared__ double sh[32];
  __shared__ int flag;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    Ctrl* c = I.ctrl;
    if (c->done) continue;
    const LevelDev& L = I.lv[0];
    const float* r = static_cast<const float*>(L.rhs);
    const float* z = static_cast<const float*>(L.z);
    double rz = 0, zs = 0, rs = 0;
    const long long base = (long long)tl.tile * kTile;
    for (int k = 0; k < kTile / kThreads; ++k) {
      const long long i = base + k * kThreads + threadIdx.x;
      if (i >= L.n) break;
      if (!L.label[i]) continue;
      const double zv = z[i], rv = r[i];
      rz += rv * zv;
      zs += zv;
      rs += rv;
    }
    const double a0 = block_sum(rz, sh), a1 = block_sum(zs, sh), a2 = block_sum(rs, sh);
    if (threadIdx.x == 0) {
      I.partial[0 * I.ntiles0 + tl.tile] = a0;
      I.partial[1 * I.ntiles0 + tl.tile] = a1;
      I.partial[2 * I.ntiles0 + tl.tile] = a2;
    }
    if (arrive_last(&c->arrive[kStGamma], I.ntiles0, &flag)) {
      const double g = gather_slot(I.partial, 0, I.ntiles0, 0, sh);
      const double zsum = gather_slot(I.partial, 1, I.ntiles0, 0, sh);
      const double rsum = gather_slot(I.partial, 2, I.ntiles0, 0, sh);
      if (threadIdx.x == 0) {
        double gamma = g;
        c->zmean = 0.0;
        if (!c->anchored) {
          c->zmean = zsum / double(c->liquid);
          gamma = g - c->zmean * rsum;
        }
        if (!(gamma > 0.0) || !isfinite(gamma)) {
          c->done = 1;
          c->status = FLUID_PP_NONCONVERGENCE;
        } else {
          c->beta = c->first ? 0.0 : gamma / c->gamma;
          c->gamma = gamma;
          c->first = 0;
        }
      }
    }
  }
}

// d = (z - zmean) + beta d on liquid cells.
__global__ void k_dir(const InstDev* insts, const Tile* tiles, int ntiles) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    const Ctrl* c = I.ctrl;
    if (c->done) continue;
    const LevelDev& L = I.lv[0];
    const float* z = static_cast<const float*>(L.z);
    const float beta = float(c->beta), zm = float(c->zmean);
    const long long base = (long long)tl.tile * kTile;
    for (int k = 0; k < kTile / kThreads; ++k) {
      const long long i = base + k * kThreads + threadIdx.x;
      if (i >= L.n) break;
      I.d[i] = L.label[i] ? (z[i] - zm) + beta * I.d[i] : 0.0f;
    }
  }
}

// q = A d and delta = d . q (applyLiquidOperator, atlas :1171-1192), alpha = gamma / delta.
__global__ void k_spmv(const InstDev* insts, const Tile* tiles, int ntiles) {
  __shared__ double sh[32];
  __shared__ int flag;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    Ctrl* c = I.ctrl;
    if (c->done) continue;
    const LevelDev& L = I.lv[0];
    const float* D = I.d;
    double dq = 0;
    const long long base = (long long)tl.tile * kTile;
    const long long sy = L.nx, sz = (long long)L.nx * L.ny;
    for (int k = 0; k < kTile / kThreads; ++k) {
      const long long i = base + k * kThreads + threadIdx.x;
      if (i >= L.n) break;
      float q = 0.0f;
      if (L.label[i]) {
        int x, y, z;
        decode(i, L.nx, L.ny, x, y, z);
        const float s = d4sum6(x > 0 ? D[i - 1] : 0.0f, x + 1 < L.nx ? D[i + 1] : 0.0f, y > 0 ? D[i - sy] : 0.0f,
                               y + 1 < L.ny ? D[i + sy] : 0.0f, z > 0 ? D[i - sz] : 0.0f,
                               z + 1 < L.nz ? D[i + sz] : 0.0f);
        q = L.diag[i] * D[i] - s;
        dq += double(D[i]) * q;
      }
      I.q[i] = q;
    }
    const double a0 = block_sum(dq, sh);
    if (threadIdx.x == 0) I.partial[tl.tile] = a0;
    if (arrive_last(&c->arrive[kStSpmv], I.ntiles0, &flag)) {
      const double delta = gather_slot(I.partial, 0, I.ntiles0, 0, sh);
      if (threadIdx.x == 0) {
        c->delta = delta;
        if (!(delta > 0.0) || !isfinite(delta)) {
          c->done = 1;
          c->status = FLUID_PP_NONCONVERGENCE;
        } else {
          c->alpha = c->gamma / delta;
        }
      }
    }
  }
}

// x += alpha d, r -= alpha q, rr = r . r.
__global__ void k_update(const InstDev* insts, const Tile* tiles, int ntiles) {
  __shared__ double sh[32];
  __shared__ int flag;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    Ctrl* c = I.ctrl;
    if (c->done) continue;
    const LevelDev& L = I.lv[0];
    float* r = static_cast<float*>(L.rhs);
    const float alpha = float(c->alpha);
    double rr = 0;
    const long long base = (long long)tl.tile * kTile;
    for (int k = 0; k < kTile / kThreads; ++k) {
      const long long i = base + k * kThreads + threadIdx.x;
      if (i >= L.n) break;
      if (!L.label[i]) continue;
      I.x[i] += alpha * I.d[i];
      const float rv = r[i] - alpha * I.q[i];
      r[i] = rv;
      rr += double(rv) * rv;
    }
    const double a0 = block_sum(rr, sh);
    if (threadIdx.x == 0) I.partial[tl.tile] = a0;
    if (arrive_last(&c->arrive[kStUpdate], I.ntiles0, &flag)) {
      const double s = gather_slot(I.partial, 0, I.ntiles0, 0, sh);
      if (threadIdx.x == 0) {
        c->rr = s;
        c->iter += 1;
        set_sigma(c, s);
        if (!isfinite(s)) {
          c->done = 1;
          c->status = FLUID_PP_NONCONVERGENCE;
        } else if (s <= c->thr2 || c->iter >= c->max_iter) {
          c->candidate = 1;
        }
      }
    }
  }
}

// Float64 true residual r = b - A x, replacing the recursive residual; decides
// convergence for candidates (octree-pipelined-pcg.ts:501-541 acceptance rule).
__global__ void k_true_residual(const InstDev* insts, const Tile* tiles, int ntiles) {
  __shared__ double sh[32];
  __shared__ int flag;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    Ctrl* c = I.ctrl;
    if (c->done) continue;
    if (!c->candidate && !(c->true_every > 0 && c->iter % c->true_every == 0)) continue;
    const LevelDev& L = I.lv[0];
    float* r = static_cast<float*>(L.rhs);
    const float* X = I.x;
    double rr = 0;
    const long long base = (long long)tl.tile * kTile;
    const long long sy = L.nx, sz = (long long)L.nx * L.ny;
    for (int k = 0; k < kTile / kThreads; ++k) {
      const long long i = base + k * kThreads + threadIdx.x;
      if (i >= L.n) break;
      if (!L.label[i]) continue;
      int x, y, z;
      decode(i, L.nx, L.ny, x, y, z);
      double s = 0;
      if (x > 0) s += X[i - 1];
      if (x + 1 < L.nx) s += X[i + 1];
      if (y > 0) s += X[i - sy];
      if (y + 1 < L.ny) s += X[i + sy];
      if (z > 0) s += X[i - sz];
      if (z + 1 < L.nz) s += X[i + sz];
      const double rv = double(I.b[i]) - (double(L.diag[i]) * double(X[i]) - s);
      r[i] = float(rv);
      rr += rv * rv;
    }
    const double a0 = block_sum(rr, sh);
    if (threadIdx.x == 0) I.partial[tl.tile] = a0;
    if (arrive_last(&c->arrive[kStTrue], I.ntiles0, &flag)) {
      const double s = gather_slot(I.partial, 0, I.ntiles0, 0, sh);
      if (threadIdx.x == 0) {
        c->rr_true = s;
        c->rr = s;
        set_sigma(c, s);
        if (c->candidate) {
          if (s <= c->thr2) {
            c->done = 1;
            c->converged = 1;
            c->status = FLUID_PP_OK;
          } else if (c->iter >= c->max_iter) {
            c->done = 1;
            c->status = FLUID_PP_NONCONVERGENCE;
          }
          c->candidate = 0;
        }
      }
    }
  }
}

// ================================================================= projection
__device__ __forceinline__ float face_update(const LevelDev& L, const float* X, long long i, long long j, float u) {
  const bool li = L.label[i], lj = L.label[j];
  if (!li && !lj) return 0.0f;
  float th = 1.0f;
  if (li && !lj) th = ghost_theta(L.phi[i], L.phi[j]);
  if (!li && lj) th = ghost_theta(L.phi[j], L.phi[i]);
  const float pi = li ? X[i] : 0.0f, pj = lj ? X[j] : 0.0f;
  return u - (pj - pi) / th;
}

// Gradient subtract (webgpu-uniform-reference.wgsl.ts:1052-1099 / atlas
// pressureCorrection :1263-1279): each cell owns its three positive faces and,
// on the low domain walls, its negative faces.  Closed walls and faces with no
// liquid side are zero.  Also publishes the pressure in Pa.
__global__ void k_grad(const InstDev* insts, const Tile* tiles, int ntiles) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    const Ctrl* c = I.ctrl;
    if (c->status == FLUID_PP_NONFINITE) continue;   // fail closed: keep the previous state
    const LevelDev& L = I.lv[0];
    const float* X = I.x;
    const long long base = (long long)tl.tile * kTile;
    const long long uS = I.nx + 1, vS = I.ny + 1;
    for (int k = 0; k < kTile / kThreads; ++k) {
      const long long i = base + k * kThreads + threadIdx.x;
      if (i >= L.n) break;
      int x, y, z;
      decode(i, L.nx, L.ny, x, y, z);
      const long long urow = uS * (y + (long long)I.ny * z);
      const long long vcol = x + (long long)I.nx * vS * z;
      const long long sz = (long long)I.nx * I.ny;
      // +x
      {
        const long long f = urow + x + 1;
        I.u[f] = x + 1 < I.nx ? face_update(L, X, i, i + 1, I.u[f]) : 0.0f;
        if (x == 0) I.u[urow] = 0.0f;
      }
      // +y
      {
        const long long f = vcol + (long long)I.nx * (y + 1);
        float nv = 0.0f;
        if (y + 1 < I.ny) nv = face_update(L, X, i, i + I.nx, I.v[f]);
        else if (I.open_top && L.label[i]) nv = I.v[f] - (0.0f - X[i]) / ghost_theta(L.phi[i], 0.5f);
        I.v[f] = nv;
        if (y == 0) I.v[vcol] = 0.0f;
      }
      // +z
      {
        const long long f = i + sz;
        I.w[f] = z + 1 < I.nz ? face_update(L, X, i, i + sz, I.w[f]) : 0.0f;
        if (z == 0) I.w[i] = 0.0f;
      }
      I.p_si[i] = L.label[i] ? X[i] * I.pscale : 0.0f;
    }
  }
}

// Post-projection divergence receipts (atlas divergenceFromEquationResidual,
// :1283-1296): max and sum of squares of (div u - q) before and after.
__global__ void k_receipt(const InstDev* insts, const Tile* tiles, int ntiles) {
  __shared__ double sh[32];
  __shared__ int flag;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    Ctrl* c = I.ctrl;
    const LevelDev& L = I.lv[0];
    double mb = 0, sb = 0, ma = 0, sa = 0;
    const long long base = (long long)tl.tile * kTile;
    const long long uS = I.nx + 1, vS = I.ny + 1;
    for (int k = 0; k < kTile / kThreads; ++k) {
      const long long i = base + k * kThreads + threadIdx.x;
      if (i >= L.n) break;
      if (!L.label[i]) continue;
      int x, y, z;
      decode(i, L.nx, L.ny, x, y, z);
      const long long urow = uS * (y + (long long)I.ny * z);
      const long long vcol = x + (long long)I.nx * vS * z;
      const long long sz = (long long)I.nx * I.ny;
      const double du = double(I.u[urow + x + 1]) - double(I.u[urow + x]);
      const double dv = double(I.v[vcol + (long long)I.nx * (y + 1)]) - double(I.v[vcol + (long long)I.nx * y]);
      const double dw = double(I.w[i + sz]) - double(I.w[i]);
      const float rho = I.vof[i];
      double q = 0.0;
      if (rho > 1.0f) q = fminf(fminf(0.5f * (rho - 1.0f), 1.0f), I.h / I.dt);
      const double after = (du + dw) + dv - q;
      const double before = -double(I.b[i]);
      ma = fmax(ma, fabs(after));
      sa += after * after;
      mb = fmax(mb, fabs(before));
      sb += before * before;
    }
    const double a0 = block_max(ma, sh), a1 = block_sum(sa, sh), a2 = block_max(mb, sh), a3 = block_sum(sb, sh);
    if (threadIdx.x == 0) {
      I.partial[0 * I.ntiles0 + tl.tile] = a0;
      I.partial[1 * I.ntiles0 + tl.tile] = a1;
      I.partial[2 * I.ntiles0 + tl.tile] = a2;
      I.partial[3 * I.ntiles0 + tl.tile] = a3;
    }
    if (arrive_last(&c->arrive[kStReceipt], I.ntiles0, &flag)) {
      const double r0 = gather_slot(I.partial, 0, I.ntiles0, 1, sh);
      const double r1 = gather_slot(I.partial, 1, I.ntiles0, 0, sh);
      const double r2 = gather_slot(I.partial, 2, I.ntiles0, 1, sh);
      const double r3 = gather_slot(I.partial, 3, I.ntiles0, 0, sh);
      if (threadIdx.x == 0) {
        c->red[0] = r0;
        c->red[1] = r1;
        c->red[2] = r2;
        c->red[3] = r3;
      }
    }
  }
}

}  // namespace fpp
