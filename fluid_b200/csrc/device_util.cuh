// Inline device helpers shared by every kernel translation unit: work-tile
// geometry, storage-type access, the canonical stencil fold, deterministic
// block reductions and the last-tile-arrives pattern, trilinear transfer weights.
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

constexpr int kTX = 32, kTY = 8;   // tile extent in x and y; kTX * kTY == kThreads
constexpr int kMaxDepth = 8;       // cells per thread along z: 8 on level 0, 1, 2 or 4 on coarser levels
constexpr int kBlockThreads = 1024;        // coarse-block CTA

__host__ __device__ inline int tiles_of(int nx, int ny, int nz, int depth) {
  return ((nx + kTX - 1) / kTX) * ((ny + kTY - 1) / kTY) * ((nz + depth - 1) / depth);
}

// The cells of tile t owned by this thread: column (x, y), cells z0 .. z0+depth-1.
struct TileIt {
  int x, y, z0, k, nx, ny, nz, depth;
  bool ok;
  __device__ __forceinline__ TileIt(int t, int nx_, int ny_, int nz_, int depth_)
      : k(0), nx(nx_), ny(ny_), nz(nz_), depth(depth_) {
    const int ntx = (nx + kTX - 1) / kTX, nty = (ny + kTY - 1) / kTY;
    const int tx = t % ntx, r = t / ntx, ty = r % nty, tz = r / nty;
    x = tx * kTX + int(threadIdx.x & (kTX - 1));
    y = ty * kTY + int(threadIdx.x / kTX);
    z0 = tz * depth;
    ok = x < nx && y < ny;
  }
  __device__ __forceinline__ bool next(int& cx, int& cy, int& cz, int& i) {
    if (!ok || k >= depth) return false;
    const int z = z0 + k++;
    if (z >= nz) return false;
    cx = x;
    cy = y;
    cz = z;
    i = x + nx * (y + ny * z);
    return true;
  }
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

__device__ __forceinline__ float tof(float v) { return v; }
__device__ __forceinline__ float tof(__half v) { return __half2float(v); }
__device__ __forceinline__ float tof(__nv_bfloat16 v) { return __bfloat162float(v); }
template <class T>
__device__ __forceinline__ T fromf(float v);
template <>
__device__ __forceinline__ float fromf<float>(float v) { return v; }
template <>
__device__ __forceinline__ __half fromf<__half>(float v) { return __float2half_rn(v); }
template <>
__device__ __forceinline__ __nv_bfloat16 fromf<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

__device__ __forceinline__ void decode(int i, int nx, int ny, int& x, int& y, int& z) {
  const int yz = i / nx;
  x = i - yz * nx;
  z = yz / ny;
  y = yz - z * ny;
}

// cm12GhostFluidTheta (lib/core/cm12-numerics.ts:37-45), epsilon 1e-12.
__device__ __forceinline__ float ghost_theta(float liquid_phi, float air_phi) {
  const float a = fabsf(liquid_phi);
  return fminf(1.0f, fmaxf(0.05f, a / fmaxf(a + fabsf(air_phi), 1e-12f)));
}

// Embedded solids: a face's open fraction at or below this is closed
// (mgCoefficientRaw, mg.wgsl.ts:108: vf <= 1e-6 has no coefficient).
constexpr float kClosedFace = 1e-6f;
// Cells with an open fraction at or below this are solid (pressureDensity,
// webgpu-uniform-reference.wgsl.ts:213-233).
constexpr float kSolidCell = 1e-5f;

// Coupling weight of the face between cell i and its +axis neighbour on a level
// with the per-axis weight w: w itself without embedded solids, otherwise w
// times the face's open fraction, zero for a closed face.
__device__ __forceinline__ float face_w(const float* ff, long long n, int axis, long long i, float w) {
  if (!ff) return w;
  const float f = ff[axis * n + i];
  return f > kClosedFace ? w * f : 0.0f;
}

// Canonical fold of the six face terms (mgD4Sum6, mg.wgsl.ts:49).
__device__ __forceinline__ float d4sum6(float xm, float xp, float ym, float yp, float zm, float zp) {
  return ((xm + xp) + (zm + zp)) + (ym + yp);
}

// Deterministic block reductions (fixed shuffle tree).  Result valid in warp 0.
// Three block_sum folds in one pass (each value takes block_sum's tree, so the
// bits are block_sum's); sh holds 3 x 32 doubles.  Results valid in warp 0.
__device__ __forceinline__ void block_sum3(double& a, double& b, double& c, double* sh) {
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sh[w] = a;
    sh[32 + w] = b;
    sh[64 + w] = c;
  }
  __syncthreads();
  if (w == 0) {
    const bool in = l < int(blockDim.x >> 5);
    a = in ? sh[l] : 0.0;
    b = in ? sh[32 + l] : 0.0;
    c = in ? sh[64 + l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      b += __shfl_xor_sync(0xffffffffu, b, o);
      c += __shfl_xor_sync(0xffffffffu, c, o);
    }
  }
  __syncthreads();
}

// block_sum of a and block_max of m in one pass (each keeps its own tree, so
// the bits are those of the separate folds); sh holds 2 x 32 doubles.
__device__ __forceinline__ void block_sum_max(double& a, double& m, double* sh) {
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sh[w] = a;
    sh[32 + w] = m;
  }
  __syncthreads();
  if (w == 0) {
    const bool in = l < int(blockDim.x >> 5);
    a = in ? sh[l] : 0.0;
    m = in ? sh[32 + l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
  }
  __syncthreads();
}

// NS block_sum folds and NM block_max folds in one pass (every value keeps its
// separate fold's tree, so the bits are those folds'); sh holds (NS + NM) x 32
// doubles.  Results valid in warp 0.
template <int NS, int NM>
__device__ __forceinline__ void block_folds(double* s, double* m, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int k = 0; k < NS; ++k) s[k] += __shfl_xor_sync(0xffffffffu, s[k], o);
#pragma unroll
    for (int k = 0; k < NM; ++k) m[k] = fmax(m[k], __shfl_xor_sync(0xffffffffu, m[k], o));
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
#pragma unroll
    for (int k = 0; k < NS; ++k) sh[32 * k + w] = s[k];
#pragma unroll
    for (int k = 0; k < NM; ++k) sh[32 * (NS + k) + w] = m[k];
  }
  __syncthreads();
  if (w == 0) {
    const bool in = l < int(blockDim.x >> 5);
#pragma unroll
    for (int k = 0; k < NS; ++k) s[k] = in ? sh[32 * k + l] : 0.0;
#pragma unroll
    for (int k = 0; k < NM; ++k) m[k] = in ? sh[32 * (NS + k) + l] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
      for (int k = 0; k < NS; ++k) s[k] += __shfl_xor_sync(0xffffffffu, s[k], o);
#pragma unroll
      for (int k = 0; k < NM; ++k) m[k] = fmax(m[k], __shfl_xor_sync(0xffffffffu, m[k], o));
    }
  }
  __syncthreads();
}

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

// Sum (op 0) or max (op 1) of one slot over all tiles.  Thread j owns tiles
// j, j + blockDim, ... and folds them in four interleaved accumulators (a fixed
// order), then the block folds the threads: deterministic for a given tile
// count.  Loads bypass L1 (__ldcg): the partials were written by other CTAs
// before the arrival counter released them.
__device__ __forceinline__ double gather_slot(const double* partial, int slot, int ntiles, int op, double* sh) {
  const double* p = partial + (long long)slot * ntiles;
  double a[4] = {0.0, 0.0, 0.0, 0.0};
  const int stride = blockDim.x;
  int t = threadIdx.x;
  for (; t + 3 * stride < ntiles; t += 4 * stride) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const double v = __ldcg(p + t + u * stride);
      a[u] = op ? fmax(a[u], v) : a[u] + v;
    }
  }
  for (; t < ntiles; t += stride) {
    const double v = __ldcg(p + t);
    a[0] = op ? fmax(a[0], v) : a[0] + v;
  }
  const double acc = op ? fmax(fmax(a[0], a[1]), fmax(a[2], a[3])) : (a[0] + a[1]) + (a[2] + a[3]);
  return op ? block_max(acc, sh) : block_sum(acc, sh);
}

// Cell-centred trilinear prolongation taps along one axis (mgTrilinearPressure,
// mg.wgsl.ts:217-241): taps outside the grid dropped, weights renormalised.
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

// The same taps as taps1d in a fixed pair: a dropped tap repeats a valid index
// with weight zero, so callers can unroll the 2 x 2 x 2 stencil.
__device__ __forceinline__ void taps2(int f, int stride, int nc, int* c, float* w) {
  if (stride == 1) {
    c[0] = c[1] = f;
    w[0] = 1.0f;
    w[1] = 0.0f;
    return;
  }
  const int k = f >> 1;
  int a, b;
  float wa, wb;
  if ((f & 1) == 0) { a = k - 1; wa = 0.25f; b = k; wb = 0.75f; }
  else { a = k; wa = 0.75f; b = k + 1; wb = 0.25f; }
  const bool ia = a >= 0 && a < nc, ib = b >= 0 && b < nc;
  c[0] = ia ? a : b;
  c[1] = ib ? b : a;
  w[0] = ia ? (ib ? wa : 1.0f) : 0.0f;
  w[1] = ib ? (ia ? wb : 1.0f) : 0.0f;
}

// Weight of coarse cell c in the stencil of fine cell f along an axis that
// coarsened by two (the transpose entries of taps1d).
__device__ __forceinline__ float p1d(int f, int c, int nc) {
  const int d = f - 2 * c;
  if (d == 0) return c == 0 ? 1.0f : 0.75f;
  if (d == 1) return c + 1 == nc ? 1.0f : 0.75f;
  return 0.25f;   // d == -1 or d == 2
}

// ------------------------------------------------------------ CG scalars
// The per-solve scalar logic shared by every CG kernel family; each runs in the
// thread that finished a reduction.

// Preconditioner input scale: 1 / rms of the residual over liquid cells.
__device__ __forceinline__ void set_sigma(Ctrl* c, double rr) {
  const double per = rr / double(c->liquid > 0 ? c->liquid : 1);
  c->sigma = per > 1e-300 ? 1.0 / sqrt(per) : 1.0;
}

// gamma = r . (z - zmean) from its three sums; beta from the previous gamma.
// With the full-cycle preconditioner (not symmetric) beta is flexible CG's
// Polak-Ribiere form r_k+1 . (z_k+1 - z_k) / (r_k . z_k); rzp = r_k+1 . z_k
// (raw, before the previous step's mean removal).  A non-positive or
// non-finite gamma ends the solve (the preconditioned system lost definiteness).
__device__ __forceinline__ void finish_gamma(Ctrl* c, double rz, double zsum, double rsum, double rzp = 0.0) {
  double gamma = rz;
  c->zmean = 0.0;
  if (!c->anchored) {
    c->zmean = zsum / double(c->liquid);
    gamma = rz - c->zmean * rsum;
  }
  if (!(gamma > 0.0) || !isfinite(gamma)) {
    c->done = 1;
    c->status = FLUID_PP_NONCONVERGENCE;
  } else {
    const double num = (c->fcg && !c->first) ? gamma - (rzp - c->zmean_prev * rsum) : gamma;
    c->beta = c->first ? 0.0 : num / c->gamma;
    c->gamma = gamma;
    c->zmean_prev = c->zmean;
    c->first = 0;
  }
}

// delta = d . A d and alpha = gamma / delta (direct curvature).
__device__ __forceinline__ void finish_delta(Ctrl* c, double delta) {
  c->delta = delta;
  if (!(delta > 0.0) || !isfinite(delta)) {
    c->done = 1;
    c->status = FLUID_PP_NONCONVERGENCE;
  } else {
    c->alpha = c->gamma / delta;
  }
}

// x += alpha d, r -= alpha q finished: ||r||^2 = s, max |r| = m.  Below the
// tolerance (or at the iteration cap) the solve becomes a candidate for the
// float64 acceptance check.
__device__ __forceinline__ void finish_update(Ctrl* c, double s, double m) {
  c->rr = s;
  c->rmax = m;
  c->iter += 1;
  set_sigma(c, s);
  if (!isfinite(s)) {
    c->done = 1;
    c->status = FLUID_PP_NONCONVERGENCE;
  } else if ((s <= c->thr2 && (c->thr_inf <= 0 || m <= c->thr_inf)) || c->iter >= c->max_iter) {
    c->candidate = 1;
  }
}

// Float64 true residual finished (octree-pipelined-pcg.ts:501-541 acceptance rule).
__device__ __forceinline__ void finish_true(Ctrl* c, double s, double m) {
  c->rr_true = s;
  c->rr = s;
  c->rmax = m;
  set_sigma(c, s);
  if (c->candidate) {
    if (s <= c->thr2 && (c->thr_inf <= 0 || m <= c->thr_inf)) {
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

// In-place Gauss-Jordan inverse of an SPD m x m matrix in shared memory (no
// pivoting needed), all threads of the CTA; prow/pcol hold m doubles each.
// Rows go to warps and columns to lanes, so no thread divides an index.
__device__ __forceinline__ void gauss_jordan_inplace(double* A, int m, double* prow, double* pcol) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int k = 0; k < m; ++k) {
    const double piv = A[k * m + k];
    for (int j = threadIdx.x; j < m; j += blockDim.x) {
      prow[j] = (j == k ? 1.0 : A[k * m + j]) / piv;
      pcol[j] = A[j * m + k];
    }
    __syncthreads();
    for (int i = warp; i < m; i += nwarps) {
      double* row = A + i * m;
      if (i == k) {
        for (int j = lane; j < m; j += 32) row[j] = prow[j];
      } else {
        const double pc = pcol[i];
        for (int j = lane; j < m; j += 32) row[j] = ((j == k) ? 0.0 : row[j]) - pc * prow[j];
      }
    }
    __syncthreads();
  }
}

}  // namespace fpp
