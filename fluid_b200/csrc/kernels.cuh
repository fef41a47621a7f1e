// Device kernels of the uniform-grid pressure projection (sm_100a).
//
// Every grid kernel walks a list of work tiles (instance, level, tile) so the
// same launch serves one solve or a batch of uneven solves.  A tile is a
// 32 x 8 x 4 block of cells of one level (x fastest): thread (lx, ly) of the
// 256-thread CTA owns column (x0 + lx, y0 + ly) and marches its four z cells.
// Reductions are deterministic: each tile writes its float64 partial to its
// own slot and the last tile of an instance to arrive sums the slots in tile
// order and finalises the scalars.
#pragma once
#include "device_util.cuh"

namespace fpp {

// Column helper: calls f(k, z, i) for the thread's valid cells of its tile
// column (TileIt's cells, in the same order), fully unrolled so the loads of
// all the column's cells are in flight together.
template <class F>
__device__ __forceinline__ void for_column(const TileIt& it, int nx, int ny, int nz, F f) {
  if (!it.ok) return;
  const int sz = nx * ny;
  const int i0 = it.x + nx * (it.y + ny * it.z0);
#pragma unroll
  for (int k = 0; k < kMaxDepth; ++k)
    if (k < it.depth && it.z0 + k < nz) f(k, it.z0 + k, i0 + k * sz);
}

// Grid-stride walk over a tile list that visits only the tiles whose instance
// passes `active`: the CTA reads the flags of up to blockDim.x of its tiles at
// once (one dependent read chain per round instead of one per tile) and runs
// body(t) for the active ones in increasing t, uniformly across the CTA.  A
// skipped tile costs no pass of its own; results are those of the plain walk.
template <class P, class F>
__device__ __forceinline__ void for_active_tiles(const InstDev* insts, const Tile* tiles, int ntiles, P active,
                                                 F body) {
  __shared__ int act[kThreads];
  __shared__ int wcnt[kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int base = blockIdx.x; base < ntiles; base += gridDim.x * blockDim.x) {
    const int mt = base + threadIdx.x * gridDim.x;
    const bool a = mt < ntiles && active(insts[tiles[mt].inst]);
    const unsigned m = __ballot_sync(0xffffffffu, a);
    if (lane == 0) wcnt[warp] = __popc(m);
    __syncthreads();
    int off = 0, n = 0;
    for (int w = 0; w < nwarps; ++w) {
      off += w < warp ? wcnt[w] : 0;
      n += wcnt[w];
    }
    if (a) act[off + __popc(m & ((1u << lane) - 1u))] = mt;
    __syncthreads();
    for (int j = 0; j < n; ++j) body(act[j]);
    __syncthreads();
  }
}

// ================================================================= setup
// Level 0: labels, level set and right-hand side from the VOF and MAC velocities
// (ref.wgsl.ts:208-242 labelling; divergenceAt :1010-1024 with closed walls
// carrying no flux; mgBuildFinestRhs mg.wgsl.ts:152-167 in finest-cell units).
__global__ void __launch_bounds__(kThreads, 2) k_label_rhs(const InstDev* insts, const Tile* tiles, int ntiles,
                                                         int warm) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    const LevelDev& L = I.lv[0];
    int liquid = 0, air = 0, top = 0, bad = 0;
    const int nx = I.nx, ny = I.ny, nz = I.nz;
    const long long uS = nx + 1, vS = ny + 1, sz = (long long)nx * ny;
    const float* __restrict__ vof = I.vof;
    const float* __restrict__ U = I.u;
    const float* __restrict__ V = I.v;
    const float* __restrict__ W = I.w;
    uint8_t* __restrict__ lab = L.label;
    float* __restrict__ phi = L.phi;
    float* __restrict__ B = I.b;
    float* __restrict__ X = I.x;
    float* __restrict__ Xlo = I.xlo;
    const bool open_top = I.open_top;
    const float hdt = I.h / I.dt;
    const TileIt it(tl.tile, nx, ny, nz, L.depth);
    const int x = it.x, y = it.y;
    // every load of the column first, then the arithmetic and the stores
    float rho[kMaxDepth], up[kMaxDepth], um[kMaxDepth], vp[kMaxDepth], vm[kMaxDepth], wp[kMaxDepth], wm[kMaxDepth];
    for_column(it, nx, ny, nz, [&](int k, int z, int i) {
      const long long ur = uS * (y + (long long)ny * z);
      rho[k] = vof[i];
      up[k] = U[x + 1 + ur];
      um[k] = U[x + ur];
      vp[k] = V[x + (long long)nx * (y + 1 + vS * z)];
      vm[k] = V[x + (long long)nx * (y + vS * z)];
      wp[k] = W[i + sz];
      wm[k] = W[i];
    });
    for_column(it, nx, ny, nz, [&](int k, int z, int i) {
      const float r = rho[k];
      const bool liq = r > 0.5f;
      lab[i] = liq ? 1 : 0;
      phi[i] = 0.5f - r;
      bad |= !(isfinite(r) && isfinite(up[k]) && isfinite(um[k]) && isfinite(vp[k]) && isfinite(vm[k]) &&
               isfinite(wp[k]) && isfinite(wm[k]));
      float b = 0.0f;
      if (liq) {
        const float fxp = x + 1 < nx ? up[k] : 0.0f, fxm = x > 0 ? um[k] : 0.0f;
        const float fyp = (y + 1 < ny || open_top) ? vp[k] : 0.0f, fym = y > 0 ? vm[k] : 0.0f;
        const float fzp = z + 1 < nz ? wp[k] : 0.0f, fzm = z > 0 ? wm[k] : 0.0f;
        const float div = ((fxp - fxm) + (fzp - fzm)) + (fyp - fym);
        float q = 0.0f;   // cm12VolumeCorrectionDivergence * h (cm12-numerics.ts:127-138)
        if (r > 1.0f) q = fminf(fminf(0.5f * (r - 1.0f), 1.0f), hdt);
        b = -(div - q);
        ++liquid;
        top += (y == ny - 1);
      } else {
        ++air;
      }
      B[i] = b;
      if (!(warm && liq)) {
        X[i] = 0.0f;
        Xlo[i] = 0.0f;
      }
    });
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
    int x, y, z, i;
    for (TileIt it(tl.tile, C.nx, C.ny, C.nz, C.depth); it.next(x, y, z, i);) {
      float ph[8], ps[8], pf[8], nf[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int ox = c & 1, oy = (c >> 1) & 1, oz = (c >> 2) & 1;
        const int fx = min(C.sx * x + ox * (C.sx - 1), F.nx - 1);
        const int fy = min(C.sy * y + oy * (C.sy - 1), F.ny - 1);
        const int fz = min(C.sz * z + oz * (C.sz - 1), F.nz - 1);
        const float p = F.phi[fx + F.nx * (fy + F.ny * fz)];
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
// 299-307, Neumann walls): face to liquid w_a, face to air w_a / theta, open top
// w_y / theta(phi, h_y / 2); with embedded solids each face's w_a is scaled by its
// open fraction (a closed face adds nothing).
template <class T>
__global__ void k_bake_diag(const InstDev* insts, const Tile* tiles, int ntiles) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    const LevelDev& L = I.lv[tl.level];
    const float norm = 1.0f / L.wmax;
    const float wx = L.wx * L.wmax, wy = L.wy * L.wmax, wz = L.wz * L.wmax;
    const int sy = L.nx, sz = L.nx * L.ny;
    int x, y, z, i;
    for (TileIt it(tl.tile, L.nx, L.ny, L.nz, L.depth); it.next(x, y, z, i);) {
      float d = 0.0f;
      if (L.label[i]) {
        const float ph = L.phi[i];
        const float* ff = L.ff;
        const long long n = L.n;
        // the face between cells f and f + stride of `axis` (j is the neighbour)
        auto term = [&](bool inside, int j, int axis, int f, float w) -> float {
          if (!inside) return 0.0f;
          const float wf = face_w(ff, n, axis, f, w);
          return L.label[j] ? wf : wf / ghost_theta(ph, L.phi[j]);
        };
        const float xm = term(x > 0, i - 1, 0, i - 1, wx), xp = term(x + 1 < L.nx, i + 1, 0, i, wx);
        const float ym = term(y > 0, i - sy, 1, i - sy, wy);
        float yp = term(y + 1 < L.ny, i + sy, 1, i, wy);
        if (y + 1 == L.ny && I.open_top) yp = face_w(ff, n, 1, i, wy) / ghost_theta(ph, L.ext_phi);
        const float zm = term(z > 0, i - sz, 2, i - sz, wz), zp = term(z + 1 < L.nz, i + sz, 2, i, wz);
        d = d4sum6(xm, xp, ym, yp, zm, zp);
        // embedded solids: a liquid cell whose faces are all closed has an empty
        // row and leaves the system (its neighbours see it through closed faces only)
        if (ff && d == 0.0f) L.label[i] = 0;
      }
      L.diag[i] = d;
      St<T>::st(L.diagT, i, d * norm);
    }
  }
}

// Dense inverse of the coarsest (normalised) operator, one CTA per instance.
// Air cells are identity rows; a level without Dirichlet contact gets the
// rank-one term mean(diag)/m * 1 1^T so the inverse is SPD.
template <class TD>
__global__ void __launch_bounds__(kBlockThreads) k_coarse_factor(const InstDev* insts, const int* list) {
  extern __shared__ double A[];
  const InstDev& I = insts[list[blockIdx.x]];
  const LevelDev& L = I.lv[I.nlev - 1];
  const int m = int(L.n);
  __shared__ int anchored;
  __shared__ double diag_mean;
  __shared__ double pivot_row[kMaxCoarse];
  __shared__ double pivot_col[kMaxCoarse];
  if (threadIdx.x == 0) {
    anchored = 0;
    diag_mean = 0.0;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < m * m; e += blockDim.x) A[e] = 0.0;
  __syncthreads();
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    int x, y, z;
    decode(i, L.nx, L.ny, x, y, z);
    if (!L.label[i]) {
      A[i * m + i] = 1.0;
      atomicOr(&anchored, 1);
      continue;
    }
    if (I.open_top && y == L.ny - 1) atomicOr(&anchored, 1);
    A[i * m + i] = St<TD>::ld(L.diagT, i);
    const int sy = L.nx, sz = L.nx * L.ny;
    const float* ff = L.ff;
    const long long n = L.n;
    if (x > 0 && L.label[i - 1]) A[i * m + i - 1] = -face_w(ff, n, 0, i - 1, L.wx);
    if (x + 1 < L.nx && L.label[i + 1]) A[i * m + i + 1] = -face_w(ff, n, 0, i, L.wx);
    if (y > 0 && L.label[i - sy]) A[i * m + i - sy] = -face_w(ff, n, 1, i - sy, L.wy);
    if (y + 1 < L.ny && L.label[i + sy]) A[i * m + i + sy] = -face_w(ff, n, 1, i, L.wy);
    if (z > 0 && L.label[i - sz]) A[i * m + i - sz] = -face_w(ff, n, 2, i - sz, L.wz);
    if (z + 1 < L.nz && L.label[i + sz]) A[i * m + i + sz] = -face_w(ff, n, 2, i, L.wz);
  }
  __syncthreads();
  if (!anchored) {
    if (threadIdx.x == 0) {
      double s = 0;
      for (int i = 0; i < m; ++i) s += A[i * m + i];
      diag_mean = s / double(m);
    }
    __syncthreads();
    const double add = diag_mean / double(m);
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) A[e] += add;
    __syncthreads();
  }
  gauss_jordan_inplace(A, m, pivot_row, pivot_col);
  for (int e = threadIdx.x; e < m * m; e += blockDim.x) I.coarse_inv[e] = A[e];
}

// ================================================================= CG scalars
enum Stage { kStInit = 0, kStGamma = 1, kStSpmv = 2, kStUpdate = 3, kStTrue = 4, kStReceipt = 5 };


// r = b - A x (x already masked to liquid) and the tile's partials of b.b,
// sum b, r.r, max|b|, max|r|; k_cg_init_finish folds them per instance in tile
// order afterwards.
__global__ void __launch_bounds__(kThreads) k_cg_init_part(const InstDev* insts, const Tile* tiles, int ntiles,
                                                            int warm) {
  __shared__ double sh[5 * 32];
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    const LevelDev& L = I.lv[0];
    float* __restrict__ r = static_cast<float*>(L.rhs);
    const float* __restrict__ B = I.b;
    const uint8_t* __restrict__ lab = L.label;
    const int nx = L.nx, ny = L.ny, nz = L.nz, sy = nx, sz = nx * ny;
    double sums[3] = {0, 0, 0}, maxes[2] = {0, 0};   // bb, b, rr; max|b|, max|r|
    const TileIt it(tl.tile, nx, ny, nz, L.depth);
    const int x = it.x, y = it.y;
    float bv[kMaxDepth];
    uint8_t lb[kMaxDepth];
    for_column(it, nx, ny, nz, [&](int k, int, int i) {
      bv[k] = B[i];
      lb[k] = warm ? lab[i] : 0;
    });
    for_column(it, nx, ny, nz, [&](int k, int z, int i) {
      const float b = bv[k];
      float rv = b;
      if (lb[k]) {
        auto X = [&](int j) { return double(I.x[j]) + double(I.xlo[j]); };
        const float* ff = L.ff;
        const long long n = L.n;
        // neighbour j across the face between cells f and f + stride of `axis`
        auto nb = [&](bool in, int j, int axis, int f) {
          return (in && lab[j]) ? double(face_w(ff, n, axis, f, 1.0f)) * X(j) : 0.0;
        };
        const double s = ((nb(x > 0, i - 1, 0, i - 1) + nb(x + 1 < nx, i + 1, 0, i)) +
                          (nb(z > 0, i - sz, 2, i - sz) + nb(z + 1 < nz, i + sz, 2, i))) +
                         (nb(y > 0, i - sy, 1, i - sy) + nb(y + 1 < ny, i + sy, 1, i));
        rv = float(double(b) - (double(L.diag[i]) * X(i) - s));
      }
      r[i] = rv;
      sums[0] += double(b) * b;
      sums[1] += b;
      sums[2] += double(rv) * rv;
      maxes[0] = fmax(maxes[0], fabs(double(b)));
      maxes[1] = fmax(maxes[1], fabs(double(rv)));
    });
    block_folds<3, 2>(sums, maxes, sh);
    if (threadIdx.x == 0) {
      I.partial[0 * I.ntiles0 + tl.tile] = sums[0];
      I.partial[1 * I.ntiles0 + tl.tile] = sums[1];
      I.partial[2 * I.ntiles0 + tl.tile] = sums[2];
      I.partial[3 * I.ntiles0 + tl.tile] = maxes[0];
      I.partial[4 * I.ntiles0 + tl.tile] = maxes[1];
    }
  }
}

// CG scalars of each listed instance from its k_cg_init_part partials (one CTA
// each): nullspace shift, thresholds, and the done flag for an instance with
// nothing to solve.
__global__ void __launch_bounds__(kThreads) k_cg_init_finish(const InstDev* insts, const int* ilist, double rel_tol,
                                                              double abs_tol, int max_iter, int true_every,
                                                              double rel_tol_inf, int fcg) {
  __shared__ double sh[32];
  const InstDev& I = insts[ilist[blockIdx.x]];
  Ctrl* c = I.ctrl;
  const int nt0 = I.ntiles0;
  const double bb = gather_slot(I.partial, 0, nt0, 0, sh);
  const double bs = gather_slot(I.partial, 1, nt0, 0, sh);
  const double rr = gather_slot(I.partial, 2, nt0, 0, sh);
  const double bmax = gather_slot(I.partial, 3, nt0, 1, sh);
  const double rmax = gather_slot(I.partial, 4, nt0, 1, sh);
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
    c->bmax = bmax;
    c->rmax = rmax;
    c->thr_inf = rel_tol_inf > 0 ? rel_tol_inf * bmax : 0.0;
    c->iter = 0;
    c->max_iter = max_iter;
    c->true_every = true_every;
    c->first = 1;
    c->fcg = fcg;
    c->zmean_prev = 0.0;
    c->dsel = 0;
    c->candidate = 0;
    c->converged = 0;
    c->done = 0;
    c->status = FLUID_PP_OK;
    c->rr_true = c->rr;
    set_sigma(c, c->rr);
    if (c->nonfinite) {
      c->done = 1;
      c->status = FLUID_PP_NONFINITE;
    } else if (c->liquid == 0 || (c->rr <= c->thr2 && (c->thr_inf <= 0 || c->rmax <= c->thr_inf))) {
      c->done = 1;   // nothing to solve, or the initial guess already satisfies the tolerance
      c->converged = 1;
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
    int x, y, z, i;
    for (TileIt it(tl.tile, L.nx, L.ny, L.nz, L.depth); it.next(x, y, z, i);) {
      if (!L.label[i]) continue;
      I.b[i] -= m;
      r[i] -= m;
    }
  }
}

// ================================================================= V-cycle
// The grid kernels below are written in two phases: every load of a thread's
// column of kTZ cells is issued first (descriptor fields are copied to
// registers up front), stores follow, so a launch costs about one memory round
// trip per dependency level instead of one per cell.

// One colour pass of red-black Gauss-Seidel on the normalised level operator
// (mgSmoothColour, mg.wgsl.ts:325-344, without the p_min projection).  With
// zero_init the pass starts from z = 0 and also clears the other colour.
//
// project = 1 (the LCP solve, CM11a Eq. 18 as mgSmoothColour applies it): every
// updated value is raised to the level's lower bound pmin, and the liquid cells
// of the other colour are projected too (z = max(z, pmin)).
template <class TZ, class TR, class TD>
__global__ void __launch_bounds__(kThreads) k_smooth(const InstDev* insts, const Tile* tiles, int ntiles, int level,
                                                     int colour, int zero_init, int project = 0) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    const int done = I.ctrl->done;
    const LevelDev L = I.lv[level];
    const TileIt it(tl.tile, L.nx, L.ny, L.nz, L.depth);
    if (done || !it.ok) continue;
    const TZ* z = static_cast<const TZ*>(L.z);
    TZ* zo = static_cast<TZ*>(L.z);
    const TR* __restrict__ rhs = static_cast<const TR*>(L.rhs);
    const TD* __restrict__ dg = static_cast<const TD*>(L.diagT);
    const uint8_t* __restrict__ lab = L.label;
    const int sy = L.nx, sz = L.nx * L.ny;
    const int x = it.x, y = it.y;
    const int i0 = x + L.nx * (y + L.ny * it.z0);
    float val[kMaxDepth];
    bool wr[kMaxDepth];
#pragma unroll
    for (int k = 0; k < kMaxDepth; ++k) {
      if (k >= it.depth) break;
      const int zz = it.z0 + k, i = i0 + k * sz;
      wr[k] = false;
      val[k] = 0.0f;
      if (zz < L.nz) {
        if (((x + y + zz) & 1) == colour) {
          float s = 0.0f;
          if (!zero_init) {
            const float* ff = L.ff;
            const long long n = L.n;
            const float xm = x > 0 ? face_w(ff, n, 0, i - 1, L.wx) * tof(z[i - 1]) : 0.0f;
            const float xp = x + 1 < L.nx ? face_w(ff, n, 0, i, L.wx) * tof(z[i + 1]) : 0.0f;
            const float ym = y > 0 ? face_w(ff, n, 1, i - sy, L.wy) * tof(z[i - sy]) : 0.0f;
            const float yp = y + 1 < L.ny ? face_w(ff, n, 1, i, L.wy) * tof(z[i + sy]) : 0.0f;
            const float zm = zz > 0 ? face_w(ff, n, 2, i - sz, L.wz) * tof(z[i - sz]) : 0.0f;
            const float zp = zz + 1 < L.nz ? face_w(ff, n, 2, i, L.wz) * tof(z[i + sz]) : 0.0f;
            s = d4sum6(xm, xp, ym, yp, zm, zp);
          }
          val[k] = lab[i] ? (tof(rhs[i]) + s) / tof(dg[i]) : 0.0f;
          if (project && lab[i]) val[k] = fmaxf(val[k], L.pmin[i]);
          wr[k] = true;
        } else if (zero_init) {
          wr[k] = true;
        } else if (project && lab[i]) {
          val[k] = fmaxf(tof(z[i]), L.pmin[i]);
          wr[k] = true;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kMaxDepth; ++k)
      if (k < it.depth && wr[k]) zo[i0 + k * sz] = fromf<TZ>(val[k]);
  }
}

// Residual and restriction fused, one CTA per coarse tile of kRX x kRY x kRZ
// cells.  The CTA computes the fine residual scale * (rhs - A z) of its fine
// footprint (the tile's children plus a one-cell halo on coarsened axes) into
// shared memory, then applies R = P^T / 2^k separably: a 4-tap x pass, a y pass
// and a z pass, without the residual's round trip through memory.
constexpr int kRX = 16, kRY = 4, kRZ = 4;
constexpr int kRFX = 2 * kRX + 2, kRFY = 2 * kRY + 2, kRFZ = 2 * kRZ + 2;

__host__ __device__ inline int rtiles_of(int nx, int ny, int nz) {
  return ((nx + kRX - 1) / kRX) * ((ny + kRY - 1) / kRY) * ((nz + kRZ - 1) / kRZ);
}

// Fine index range [f0, f0 + fn) feeding coarse cells [c0, c0 + cn) along one axis.
__device__ __forceinline__ void fine_span(int stride, int c0, int cn, int nf, int& f0, int& fn) {
  if (stride == 1) {
    f0 = c0;
    fn = cn;
    return;
  }
  const int lo = max(2 * c0 - 1, 0), hi = min(2 * (c0 + cn) + 1, nf);
  f0 = lo;
  fn = hi - lo;
}

// 4-tap restriction along one axis from a shared-memory line: coarse index c,
// fine values v[(f - f0) * step].
__device__ __forceinline__ float rline(int stride, int c, int nc, int nf, int f0, const float* v, int step) {
  if (stride == 1) return v[(c - f0) * step];
  float s = 0.0f;
#pragma unroll
  for (int d = -1; d <= 2; ++d) {
    const int f = 2 * c + d;
    if (f >= 0 && f < nf) s += p1d(f, c, nc) * v[(f - f0) * step];
  }
  return s;
}

template <class TZ, class TR, class TD, class TS>
__global__ void __launch_bounds__(kThreads) k_residual_restrict(const InstDev* insts, const Tile* tiles, int ntiles,
                                                                int level) {
  __shared__ float res_s[kRFZ * kRFY * kRFX];
  __shared__ float xs[kRFZ * kRFY * kRX];
  __shared__ float ys[kRFZ * kRY * kRX];
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    const int done = I.ctrl->done;
    const double sigma = I.ctrl->sigma;
    const LevelDev F = I.lv[level];
    const LevelDev C = I.lv[level + 1];
    if (done) continue;   // uniform per CTA
    const float scale = level == 0 ? float(sigma) : 1.0f;
    const int ntx = (C.nx + kRX - 1) / kRX, nty = (C.ny + kRY - 1) / kRY;
    const int tx = tl.tile % ntx, tr = tl.tile / ntx, ty = tr % nty, tz = tr / nty;
    const int cx0 = tx * kRX, cy0 = ty * kRY, cz0 = tz * kRZ;
    const int cnx = min(kRX, C.nx - cx0), cny = min(kRY, C.ny - cy0), cnz = min(kRZ, C.nz - cz0);
    int fx0, fnx, fy0, fny, fz0, fnz;
    fine_span(C.sx, cx0, cnx, F.nx, fx0, fnx);
    fine_span(C.sy, cy0, cny, F.ny, fy0, fny);
    fine_span(C.sz, cz0, cnz, F.nz, fz0, fnz);
    const TZ* __restrict__ z = static_cast<const TZ*>(F.z);
    const TR* __restrict__ rhs = static_cast<const TR*>(F.rhs);
    const TD* __restrict__ dg = static_cast<const TD*>(F.diagT);
    const uint8_t* __restrict__ lab = F.label;
    const int sy = F.nx, sz = F.nx * F.ny;
    // fine residual of the footprint
    const int fcount = fnx * fny * fnz;
    for (int e = threadIdx.x; e < fcount; e += blockDim.x) {
      const int lx = e % fnx, lr = e / fnx, ly = lr % fny, lz = lr / fny;
      const int x = fx0 + lx, y = fy0 + ly, zz = fz0 + lz;
      const int i = x + F.nx * (y + F.ny * zz);
      float r = 0.0f;
      if (lab[i]) {
        const float* ff = F.ff;
        const long long n = F.n;
        const float xm = x > 0 ? face_w(ff, n, 0, i - 1, F.wx) * tof(z[i - 1]) : 0.0f;
        const float xp = x + 1 < F.nx ? face_w(ff, n, 0, i, F.wx) * tof(z[i + 1]) : 0.0f;
        const float ym = y > 0 ? face_w(ff, n, 1, i - sy, F.wy) * tof(z[i - sy]) : 0.0f;
        const float yp = y + 1 < F.ny ? face_w(ff, n, 1, i, F.wy) * tof(z[i + sy]) : 0.0f;
        const float zm = zz > 0 ? face_w(ff, n, 2, i - sz, F.wz) * tof(z[i - sz]) : 0.0f;
        const float zp = zz + 1 < F.nz ? face_w(ff, n, 2, i, F.wz) * tof(z[i + sz]) : 0.0f;
        r = scale * (tof(rhs[i]) - (tof(dg[i]) * tof(z[i]) - d4sum6(xm, xp, ym, yp, zm, zp)));
      }
      res_s[(lz * kRFY + ly) * kRFX + lx] = r;
    }
    __syncthreads();
    // x pass: (fine z, fine y, coarse x)
    for (int e = threadIdx.x; e < fnz * fny * cnx; e += blockDim.x) {
      const int cx = e % cnx, lr = e / cnx, ly = lr % fny, lz = lr / fny;
      xs[(lz * kRFY + ly) * kRX + cx] = rline(C.sx, cx0 + cx, C.nx, F.nx, fx0, &res_s[(lz * kRFY + ly) * kRFX], 1);
    }
    __syncthreads();
    // y pass: (fine z, coarse y, coarse x)
    for (int e = threadIdx.x; e < fnz * cny * cnx; e += blockDim.x) {
      const int cx = e % cnx, lr = e / cnx, cy = lr % cny, lz = lr / cny;
      ys[(lz * kRY + cy) * kRX + cx] = rline(C.sy, cy0 + cy, C.ny, F.ny, fy0, &xs[lz * kRFY * kRX + cx], kRX);
    }
    __syncthreads();
    // z pass and store
    const float out_scale = F.to_coarse / float((C.sx == 2 ? 2 : 1) * (C.sy == 2 ? 2 : 1) * (C.sz == 2 ? 2 : 1));
    TS* __restrict__ out = static_cast<TS*>(C.rhs);
    for (int e = threadIdx.x; e < cnz * cny * cnx; e += blockDim.x) {
      const int cx = e % cnx, lr = e / cnx, cy = lr % cny, cz = lr / cny;
      const int X = cx0 + cx, Y = cy0 + cy, Z = cz0 + cz;
      const int ci = X + C.nx * (Y + C.ny * Z);
      float acc = 0.0f;
      if (C.label[ci]) acc = out_scale * rline(C.sz, Z, C.nz, F.nz, fz0, &ys[cy * kRX + cx], kRY * kRX);
      out[ci] = fromf<TS>(acc);
    }
    __syncthreads();   // shared buffers are reused by the next tile of this CTA
  }
}

// z_l += P z_{l+1} on liquid cells (mgProlongateAdd, mg.wgsl.ts:243-246);
// from level 1 into level 0 the sigma scaling is undone.
template <class TZF, class TZC>
__global__ void __launch_bounds__(kThreads) k_prolong(const InstDev* insts, const Tile* tiles, int ntiles,
                                                      int level) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    const int done = I.ctrl->done;
    const double sigma = I.ctrl->sigma;
    const LevelDev F = I.lv[level];
    const LevelDev C = I.lv[level + 1];
    const TileIt it(tl.tile, F.nx, F.ny, F.nz, F.depth);
    if (done || !it.ok) continue;
    const float unscale = level == 0 ? float(1.0 / sigma) : 1.0f;
    const TZC* __restrict__ zc = static_cast<const TZC*>(C.z);
    TZF* __restrict__ zf = static_cast<TZF*>(F.z);
    const uint8_t* __restrict__ lab = F.label;
    int cx[2], cy[2];
    float wx[2], wy[2];
    taps2(it.x, C.sx, C.nx, cx, wx);
    taps2(it.y, C.sy, C.ny, cy, wy);
    const int sz = F.nx * F.ny;
    const int i0 = it.x + F.nx * (it.y + F.ny * it.z0);
#pragma unroll
    for (int k = 0; k < kMaxDepth; ++k) {
      if (k >= it.depth) break;
      const int zz = it.z0 + k, i = i0 + k * sz;
      if (zz >= F.nz || !lab[i]) continue;
      int cz[2];
      float wz[2];
      taps2(zz, C.sz, C.nz, cz, wz);
      float s = 0.0f;
#pragma unroll
      for (int c2 = 0; c2 < 2; ++c2)
#pragma unroll
        for (int c1 = 0; c1 < 2; ++c1) {
          const int row = C.nx * (cy[c1] + C.ny * cz[c2]);
#pragma unroll
          for (int c0 = 0; c0 < 2; ++c0) s += wx[c0] * wy[c1] * wz[c2] * tof(zc[row + cx[c0]]);
        }
      zf[i] = fromf<TZF>(tof(zf[i]) + s * unscale);
    }
  }
}

// The small levels of the V-cycle in one CTA per instance, in shared memory:
// levels first..nlev-1 (each at most kCoarseBlockCells) are loaded, smoothed,
// restricted, solved densely at the coarsest, prolongated and smoothed again
// with the same operators as the grid kernels, then z of level `first` is
// written back for the prolongation into the finer grid level.  Each level
// keeps packed cell coordinates, a red-then-black cell order (a colour pass
// touches only its own cells) and the reciprocal diagonal, so a pass is a few
// shared-memory loads and FMAs per cell.
struct BlockLevel {
  int nx, ny, nz, n, nred, sx, sy, sz;
  float wx, wy, wz, to_coarse;
  float* z;
  float* rhs;
  float* res;
  float* diag;
  float* inv;
  unsigned* xyz;       // x | y << 10 | z << 20
  unsigned short* ord; // red cells first, then black
  uint8_t* lab;
};

__host__ __device__ inline long long block_level_bytes(long long n) {
  return 20 * n + 4 * n + 2 * ((n + 1) & ~1LL) + ((n + 3) & ~3LL);
}

// Red cells ((x + y + z) even) among the row-major predecessors of (x, y, z)
// in an nx * ny * nz box: a run of len cells starting on parity p holds
// (len + 1 - p) / 2 red cells, and consecutive rows and planes alternate their
// starting parity.
__device__ __forceinline__ int red_runs(int k, int len, int p0) {
  const int even = p0 ? k / 2 : (k + 1) / 2;   // runs that start red
  return even * ((len + 1) / 2) + (k - even) * (len / 2);
}
__device__ __forceinline__ int red_before(int x, int y, int z, int nx, int ny) {
  return red_runs(z, nx * ny, 0) + red_runs(y, nx, z & 1) + red_runs(1, x, (y + z) & 1);
}

template <class T>
__global__ void __launch_bounds__(kBlockThreads) k_coarse_block(const InstDev* insts, const int* list, int pre,
                                                                int post) {
  extern __shared__ float smem[];
  __shared__ BlockLevel B[kMaxLevels];
  __shared__ LevelDev sl[kMaxLevels];
  __shared__ int s_first, s_last, s_done;
  const InstDev* __restrict__ Ip = insts + list[blockIdx.x];
  if (threadIdx.x == 0) {
    s_done = Ip->ctrl->done;
    s_first = Ip->first_block;
    s_last = Ip->nlev - 1;
  }
  __syncthreads();
  if (s_done) return;
  const int first = s_first, last = s_last;
  // The block levels' descriptors, copied cooperatively into shared memory
  // first: one round trip instead of one per field.
  {
    static_assert(sizeof(LevelDev) % 4 == 0, "LevelDev is copied as 32-bit words");
    const int nw = (last - first + 1) * int(sizeof(LevelDev) / 4);
    const unsigned* src = reinterpret_cast<const unsigned*>(&Ip->lv[first]);
    unsigned* dst = reinterpret_cast<unsigned*>(&sl[first]);
    for (int w = threadIdx.x; w < nw; w += blockDim.x) dst[w] = __ldg(src + w);
  }
  __syncthreads();
  if (threadIdx.x <= last - first) {   // one thread per level lays out its arrays
    const int l = first + int(threadIdx.x);
    char* p = reinterpret_cast<char*>(smem);
    for (int k = first; k < l; ++k) p += block_level_bytes(sl[k].n);
    const LevelDev& L = sl[l];
    BlockLevel& b = B[l];
    b.nx = L.nx; b.ny = L.ny; b.nz = L.nz; b.n = int(L.n);
    b.sx = L.sx; b.sy = L.sy; b.sz = L.sz;
    b.wx = L.wx; b.wy = L.wy; b.wz = L.wz; b.to_coarse = L.to_coarse;
    b.z = reinterpret_cast<float*>(p); p += 4 * b.n;
    b.rhs = reinterpret_cast<float*>(p); p += 4 * b.n;
    b.res = reinterpret_cast<float*>(p); p += 4 * b.n;
    b.diag = reinterpret_cast<float*>(p); p += 4 * b.n;
    b.inv = reinterpret_cast<float*>(p); p += 4 * b.n;
    b.xyz = reinterpret_cast<unsigned*>(p); p += 4 * b.n;
    b.ord = reinterpret_cast<unsigned short*>(p); p += 2 * ((b.n + 1) & ~1);
    b.lab = reinterpret_cast<uint8_t*>(p);
    // red cells of a box: ceil(n / 2) when the corner cell is red
    b.nred = (b.n + 1) / 2;
  }
  __syncthreads();
  // All block levels' cells in one flattened loop (cell e of the run
  // first..last), every global load of a thread's cells issued before its first
  // store, so the levels' round trips overlap.
  {
    int total = 0;
    for (int l = first; l <= last; ++l) total += B[l].n;
    constexpr int kU = 4;
    for (int e0 = threadIdx.x; e0 < total; e0 += kU * blockDim.x) {
      float d[kU], r[kU];
      uint8_t lb[kU];
      int lv[kU], ix[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        int e = e0 + u * int(blockDim.x), l = first;
        while (l < last && e >= B[l].n) e -= B[l++].n;
        lv[u] = l;
        ix[u] = e;
        d[u] = 1.0f;
        r[u] = 0.0f;
        lb[u] = 0;
        if (e < B[l].n) {
          d[u] = tof(static_cast<const T*>(sl[l].diagT)[e]);
          lb[u] = sl[l].label[e];
          if (l == first) r[u] = tof(static_cast<const T*>(sl[l].rhs)[e]);
        }
      }
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const BlockLevel& b = B[lv[u]];
        const int i = ix[u];
        if (i >= b.n) continue;
        int x, y, zz;
        decode(i, b.nx, b.ny, x, y, zz);
        b.diag[i] = d[u];
        b.inv[i] = lb[u] ? 1.0f / d[u] : 0.0f;
        b.lab[i] = lb[u];
        b.xyz[i] = unsigned(x) | (unsigned(y) << 10) | (unsigned(zz) << 20);
        const int red = red_before(x, y, zz, b.nx, b.ny);
        b.ord[((x + y + zz) & 1) ? b.nred + (i - red) : red] = (unsigned short)i;
        if (lv[u] == first) b.rhs[i] = r[u];
      }
    }
  }
  __syncthreads();
  auto nbsum = [](const BlockLevel& b, const float* z, int i, unsigned c) {
    const int x = int(c & 1023u), y = int((c >> 10) & 1023u), zz = int(c >> 20);
    const int sy = b.nx, sz = b.nx * b.ny;
    const float xm = x > 0 ? b.wx * z[i - 1] : 0.0f, xp = x + 1 < b.nx ? b.wx * z[i + 1] : 0.0f;
    const float ym = y > 0 ? b.wy * z[i - sy] : 0.0f, yp = y + 1 < b.ny ? b.wy * z[i + sy] : 0.0f;
    const float zm = zz > 0 ? b.wz * z[i - sz] : 0.0f, zp = zz + 1 < b.nz ? b.wz * z[i + sz] : 0.0f;
    return d4sum6(xm, xp, ym, yp, zm, zp);
  };
  // one colour pass; colour 2 clears z
  auto pass = [&](int l, int colour, int zero_init) {
    const BlockLevel& b = B[l];
    if (colour == 2) {
      for (int i = threadIdx.x; i < b.n; i += blockDim.x) b.z[i] = 0.0f;
    } else {
      const int j0 = colour == 0 ? 0 : b.nred, j1 = colour == 0 ? b.nred : b.n;
      for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
        const int i = b.ord[j];
        const float s = zero_init ? 0.0f : nbsum(b, b.z, i, b.xyz[i]);
        b.z[i] = (b.rhs[i] + s) * b.inv[i];
      }
      if (zero_init)   // the other colour starts at zero
        for (int j = (colour == 0 ? b.nred : 0) + threadIdx.x; j < (colour == 0 ? b.n : b.nred); j += blockDim.x)
          b.z[b.ord[j]] = 0.0f;
    }
    __syncthreads();
  };
  // down
  for (int l = first; l < last; ++l) {
    const BlockLevel& F = B[l];
    for (int sw = 0; sw < pre; ++sw) {
      pass(l, 0, sw == 0);
      pass(l, 1, 0);
    }
    if (pre == 0) pass(l, 2, 1);
    for (int i = threadIdx.x; i < F.n; i += blockDim.x)
      F.res[i] = F.lab[i] ? F.rhs[i] - (F.diag[i] * F.z[i] - nbsum(F, F.z, i, F.xyz[i])) : 0.0f;
    __syncthreads();
    const BlockLevel& C = B[l + 1];
    {
      // R = P^T / 2^k as a fixed 4 x 4 x 4 stencil: taps outside the level (or
      // beyond a stride-1 axis' single tap) carry weight 0 at a clamped index.
      const int fnx = F.nx, fny = F.ny, fnz = F.nz, cn = C.n, cnx = C.nx, cny = C.ny, cnz = C.nz;
      const int csx = C.sx, csy = C.sy, csz = C.sz;
      const float scale = F.to_coarse / float((csx == 2 ? 2 : 1) * (csy == 2 ? 2 : 1) * (csz == 2 ? 2 : 1));
      const float* __restrict__ fres = F.res;
      const unsigned* __restrict__ cxyz = C.xyz;
      const uint8_t* __restrict__ clab = C.lab;
      float* __restrict__ crhs = C.rhs;
      auto taps4 = [](int c, int s2, int nc, int nf, int* f, float* w) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int fi = s2 == 2 ? 2 * c - 1 + k : c;
          const bool ok = s2 == 2 ? (fi >= 0 && fi < nf) : k == 0;
          f[k] = min(max(fi, 0), nf - 1);
          w[k] = ok ? (s2 == 2 ? p1d(fi, c, nc) : 1.0f) : 0.0f;
        }
      };
      for (int i = threadIdx.x; i < cn; i += blockDim.x) {
        float acc = 0.0f;
        if (clab[i]) {
          const unsigned cc = cxyz[i];
          int fx[4], fy[4], fz[4];
          float wx[4], wy[4], wz[4];
          taps4(int(cc & 1023u), csx, cnx, fnx, fx, wx);
          taps4(int((cc >> 10) & 1023u), csy, cny, fny, fy, wy);
          taps4(int(cc >> 20), csz, cnz, fnz, fz, wz);
#pragma unroll
          for (int k2 = 0; k2 < 4; ++k2) {
#pragma unroll
            for (int k1 = 0; k1 < 4; ++k1) {
              const int row = fnx * (fy[k1] + fny * fz[k2]);
              const float s = ((wx[0] * fres[row + fx[0]] + wx[1] * fres[row + fx[1]]) +
                               (wx[2] * fres[row + fx[2]] + wx[3] * fres[row + fx[3]]));
              acc += (wz[k2] * wy[k1]) * s;
            }
          }
          acc *= scale;
        }
        crhs[i] = acc;
      }
    }
    __syncthreads();
  }
  // coarsest: dense float64 inverse
  {
    const BlockLevel& b = B[last];
    const int m = b.n;
    const double* __restrict__ inv = Ip->coarse_inv;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
      double s = 0;
      const double* row = inv + (long long)i * m;
      for (int j = 0; j < m; ++j) s += row[j] * (b.lab[j] ? double(b.rhs[j]) : 0.0);
      b.z[i] = b.lab[i] ? float(s) : 0.0f;
    }
    __syncthreads();
  }
  // up
  for (int l = last - 1; l >= first; --l) {
    const BlockLevel& F = B[l];
    const BlockLevel& C = B[l + 1];
    for (int i = threadIdx.x; i < F.n; i += blockDim.x) {
      if (!F.lab[i]) continue;
      const unsigned c = F.xyz[i];
      int cx[2], cy[2], cz[2];
      float wx[2], wy[2], wz[2];
      taps2(int(c & 1023u), C.sx, C.nx, cx, wx);
      taps2(int((c >> 10) & 1023u), C.sy, C.ny, cy, wy);
      taps2(int(c >> 20), C.sz, C.nz, cz, wz);
      float s = 0.0f;
#pragma unroll
      for (int c2 = 0; c2 < 2; ++c2)
#pragma unroll
        for (int c1 = 0; c1 < 2; ++c1)
#pragma unroll
          for (int c0 = 0; c0 < 2; ++c0) s += wx[c0] * wy[c1] * wz[c2] * C.z[cx[c0] + C.nx * (cy[c1] + C.ny * cz[c2])];
      F.z[i] += s;
    }
    __syncthreads();
    for (int sw = 0; sw < post; ++sw) {
      pass(l, 1, 0);
      pass(l, 0, 0);
    }
  }
  const BlockLevel& Bf = B[first];
  T* zo = static_cast<T*>(sl[first].z);
  for (int i = threadIdx.x; i < Bf.n; i += blockDim.x) zo[i] = fromf<T>(Bf.z[i]);
}

// Coarsest solve z = A_c^{-1} rhs in float64 for single-level hierarchies.
template <class TZ, class TR>
__global__ void k_coarse_apply(const InstDev* insts, const int* list) {
  const InstDev& I = insts[list[blockIdx.x]];
  if (I.ctrl->done) return;
  const LevelDev& L = I.lv[I.nlev - 1];
  const int m = int(L.n);
  __shared__ double rhs[kMaxCoarse];
  for (int i = threadIdx.x; i < m; i += blockDim.x) rhs[i] = L.label[i] ? double(St<TR>::ld(L.rhs, i)) : 0.0;
  __syncthreads();
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    double s = 0;
    const double* row = I.coarse_inv + (long long)i * m;
    for (int j = 0; j < m; ++j) s += row[j] * rhs[j];
    St<TZ>::st(L.z, i, L.label[i] ? float(s) : 0.0f);
  }
}

// ================================================================= CG kernels
// The current search direction (the fused path alternates two buffers).
__device__ __forceinline__ float* dir_cur(const InstDev& I) { return I.ctrl->dsel ? I.d2 : I.d; }
// gamma = r . (z - zmean) with float64 accumulation; beta from the previous gamma.
template <bool FCG = false>
__global__ void __launch_bounds__(kThreads) k_dot_rz(const InstDev* insts, const Tile* tiles, int ntiles) {
  __shared__ double sh[96];
  __shared__ int flag;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    Ctrl* c = I.ctrl;
    const int done = c->done;
    const LevelDev L = I.lv[0];
    const int nt0 = I.ntiles0;
    double* partial = I.partial;
    if (done) continue;
    const float* __restrict__ r = static_cast<const float*>(L.rhs);
    const float* __restrict__ z = static_cast<const float*>(L.z);
    const uint8_t* __restrict__ lab = L.label;
    float* __restrict__ zprev = I.d2;   // flexible CG: the previous preconditioned residual (d2 is idle here)
    double rz = 0, zs = 0, rs = 0, rzp = 0;
    const TileIt it(tl.tile, L.nx, L.ny, L.nz, L.depth);
    for_column(it, L.nx, L.ny, L.nz, [&](int, int, int i) {
      if (!lab[i]) return;
      const double zv = z[i], rv = r[i];
      rz += rv * zv;
      zs += zv;
      rs += rv;
      if (FCG) {
        rzp += rv * double(zprev[i]);
        zprev[i] = float(zv);
      }
    });
    const double a0 = block_sum(rz, sh), a1 = block_sum(zs, sh), a2 = block_sum(rs, sh);
    const double a3 = FCG ? block_sum(rzp, sh) : 0.0;
    if (threadIdx.x == 0) {
      partial[0 * nt0 + tl.tile] = a0;
      partial[1 * nt0 + tl.tile] = a1;
      partial[2 * nt0 + tl.tile] = a2;
      if (FCG) partial[3 * nt0 + tl.tile] = a3;
    }
    if (arrive_last(&c->arrive[kStGamma], nt0, &flag)) {
      const double g = gather_slot(partial, 0, nt0, 0, sh);
      const double zsum = gather_slot(partial, 1, nt0, 0, sh);
      const double rsum = gather_slot(partial, 2, nt0, 0, sh);
      const double p = FCG ? gather_slot(partial, 3, nt0, 0, sh) : 0.0;
      if (threadIdx.x == 0) finish_gamma(c, g, zsum, rsum, p);
    }
  }
}

// The same gamma partials as k_dot_rz (per level-0 tile, block_sum's fold)
// without the per-tile arrival: every thread issues its column's label loads,
// then the z / r loads of its liquid cells, then folds in cell order.
// k_dot_rz_finish folds each instance's partials in tile order afterwards.
__global__ void __launch_bounds__(kThreads) k_dot_rz_part(const InstDev* insts, const Tile* tiles, int ntiles) {
  __shared__ double sh[96];
  for_active_tiles(insts, tiles, ntiles, [](const InstDev& I) { return !I.ctrl->done; }, [&](int t) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    if (I.ctrl->done) return;   // uniform per CTA
    const LevelDev& L = I.lv[0];
    const float* __restrict__ r = static_cast<const float*>(L.rhs);
    const float* __restrict__ z = static_cast<const float*>(L.z);
    const uint8_t* __restrict__ lab = L.label;
    double rz = 0, zs = 0, rs = 0;
    const TileIt it(tl.tile, L.nx, L.ny, L.nz, L.depth);
    if (it.ok) {
      const int sz = L.nx * L.ny, i0 = it.x + L.nx * (it.y + L.ny * it.z0);
      uint8_t lb[kMaxDepth];
      float zv[kMaxDepth], rv[kMaxDepth];
#pragma unroll
      for (int k = 0; k < kMaxDepth; ++k)
        lb[k] = (k < it.depth && it.z0 + k < L.nz) ? lab[i0 + k * sz] : 0;
#pragma unroll
      for (int k = 0; k < kMaxDepth; ++k) {
        zv[k] = lb[k] ? z[i0 + k * sz] : 0.0f;
        rv[k] = lb[k] ? r[i0 + k * sz] : 0.0f;
      }
#pragma unroll
      for (int k = 0; k < kMaxDepth; ++k) {
        if (!lb[k]) continue;
        const double zd = zv[k], rd = rv[k];
        rz += rd * zd;
        zs += zd;
        rs += rd;
      }
    }
    block_sum3(rz, zs, rs, sh);
    if (threadIdx.x == 0) {
      const int nt0 = I.ntiles0;
      I.partial[0 * nt0 + tl.tile] = rz;
      I.partial[1 * nt0 + tl.tile] = zs;
      I.partial[2 * nt0 + tl.tile] = rs;
    }
  });
}

// gamma of each listed instance from its k_dot_rz_part partials (one CTA each).
__global__ void __launch_bounds__(kThreads) k_dot_rz_finish(const InstDev* insts, const int* ilist) {
  __shared__ double sh[32];
  const InstDev& I = insts[ilist[blockIdx.x]];
  Ctrl* c = I.ctrl;
  if (c->done) return;
  const int nt0 = I.ntiles0;
  const double g = gather_slot(I.partial, 0, nt0, 0, sh);
  const double zsum = gather_slot(I.partial, 1, nt0, 0, sh);
  const double rsum = gather_slot(I.partial, 2, nt0, 0, sh);
  if (threadIdx.x == 0) finish_gamma(c, g, zsum, rsum);
}

// d = (z - zmean) + beta d on liquid cells.
__global__ void __launch_bounds__(kThreads) k_dir(const InstDev* insts, const Tile* tiles, int ntiles) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    const Ctrl* c = I.ctrl;
    const int done = c->done;
    const float beta = float(c->beta), zm = float(c->zmean);
    const LevelDev L = I.lv[0];
    float* __restrict__ d = dir_cur(I);
    if (done) continue;
    const float* __restrict__ z = static_cast<const float*>(L.z);
    const uint8_t* __restrict__ lab = L.label;
    const TileIt it(tl.tile, L.nx, L.ny, L.nz, L.depth);
    for_column(it, L.nx, L.ny, L.nz, [&](int, int, int i) { d[i] = lab[i] ? (z[i] - zm) + beta * d[i] : 0.0f; });
  }
}

// q = A d and delta = d . q (applyLiquidOperator, atlas :1171-1192), alpha = gamma / delta.
__global__ void __launch_bounds__(kThreads) k_spmv(const InstDev* insts, const Tile* tiles, int ntiles) {
  __shared__ double sh[32];
  __shared__ int flag;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    Ctrl* c = I.ctrl;
    const int done = c->done;
    const LevelDev L = I.lv[0];
    const int nt0 = I.ntiles0;
    double* partial = I.partial;
    const float* __restrict__ D = dir_cur(I);
    float* __restrict__ Q = I.q;
    if (done) continue;
    const float* __restrict__ dg = L.diag;
    const uint8_t* __restrict__ lab = L.label;
    double dq = 0;
    const int sy = L.nx, sz = L.nx * L.ny;
    const TileIt it(tl.tile, L.nx, L.ny, L.nz, L.depth);
    const int x = it.x, y = it.y;
    for_column(it, L.nx, L.ny, L.nz, [&](int, int zz, int i) {
      float q = 0.0f;
      if (lab[i]) {
        const float* ff = L.ff;
        const long long n = L.n;
        const float s = d4sum6(x > 0 ? face_w(ff, n, 0, i - 1, 1.0f) * D[i - 1] : 0.0f,
                               x + 1 < L.nx ? face_w(ff, n, 0, i, 1.0f) * D[i + 1] : 0.0f,
                               y > 0 ? face_w(ff, n, 1, i - sy, 1.0f) * D[i - sy] : 0.0f,
                               y + 1 < L.ny ? face_w(ff, n, 1, i, 1.0f) * D[i + sy] : 0.0f,
                               zz > 0 ? face_w(ff, n, 2, i - sz, 1.0f) * D[i - sz] : 0.0f,
                               zz + 1 < L.nz ? face_w(ff, n, 2, i, 1.0f) * D[i + sz] : 0.0f);
        q = dg[i] * D[i] - s;
        dq += double(D[i]) * q;
      }
      Q[i] = q;
    });
    const double a0 = block_sum(dq, sh);
    if (threadIdx.x == 0) partial[tl.tile] = a0;
    if (arrive_last(&c->arrive[kStSpmv], nt0, &flag)) {
      const double delta = gather_slot(partial, 0, nt0, 0, sh);
      if (threadIdx.x == 0) finish_delta(c, delta);
    }
  }
}

// x += alpha d (double-single), r -= alpha q, rr = r . r, max |r|.
__global__ void __launch_bounds__(kThreads) k_update(const InstDev* insts, const Tile* tiles, int ntiles) {
  __shared__ double sh[32];
  __shared__ int flag;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    Ctrl* c = I.ctrl;
    const int done = c->done;
    const double alpha = c->alpha;
    const LevelDev L = I.lv[0];
    const int nt0 = I.ntiles0;
    double* partial = I.partial;
    float* __restrict__ X = I.x;
    float* __restrict__ Xlo = I.xlo;
    const float* __restrict__ D = dir_cur(I);
    const float* __restrict__ Q = I.q;
    if (done) continue;
    float* __restrict__ r = static_cast<float*>(L.rhs);
    const uint8_t* __restrict__ lab = L.label;
    const float alpha_f = float(alpha);
    double rr = 0, mr = 0;
    const TileIt it(tl.tile, L.nx, L.ny, L.nz, L.depth);
    // every load of the column first (the label does not gate them), then the updates
    float xh[kMaxDepth], xl[kMaxDepth], dv[kMaxDepth], qv[kMaxDepth], rv0[kMaxDepth];
    uint8_t lb[kMaxDepth];
    for_column(it, L.nx, L.ny, L.nz, [&](int k, int, int i) {
      lb[k] = lab[i];
      xh[k] = X[i];
      xl[k] = Xlo[i];
      dv[k] = D[i];
      qv[k] = Q[i];
      rv0[k] = r[i];
    });
    for_column(it, L.nx, L.ny, L.nz, [&](int k, int, int i) {
      if (!lb[k]) return;
      // double-single accumulation: x_hi + x_lo carries the pressure to ~1e-14
      const double xv = double(xh[k]) + double(xl[k]) + alpha * double(dv[k]);
      const float hi = float(xv);
      X[i] = hi;
      Xlo[i] = float(xv - double(hi));
      const float rv = rv0[k] - alpha_f * qv[k];
      r[i] = rv;
      rr += double(rv) * rv;
      mr = fmax(mr, fabs(double(rv)));
    });
    const double a0 = block_sum(rr, sh), a1 = block_max(mr, sh);
    if (threadIdx.x == 0) {
      partial[tl.tile] = a0;
      partial[nt0 + tl.tile] = a1;
    }
    if (arrive_last(&c->arrive[kStUpdate], nt0, &flag)) {
      const double s = gather_slot(partial, 0, nt0, 0, sh);
      const double m = gather_slot(partial, 1, nt0, 1, sh);
      if (threadIdx.x == 0) finish_update(c, s, m);
    }
  }
}

// ||r||^2 and max|r| of each listed instance from its k_cupdate partials (one CTA each).
__global__ void __launch_bounds__(kThreads) k_update_finish(const InstDev* insts, const int* ilist) {
  __shared__ double sh[32];
  const InstDev& I = insts[ilist[blockIdx.x]];
  Ctrl* c = I.ctrl;
  if (c->done) return;
  const int nt0 = I.ntiles0;
  const double s = gather_slot(I.partial, 0, nt0, 0, sh);
  const double m = gather_slot(I.partial, 1, nt0, 1, sh);
  if (threadIdx.x == 0) finish_update(c, s, m);
}

// Float64 true residual r = b - A x, replacing the recursive residual; decides
// convergence for candidates (octree-pipelined-pcg.ts:501-541 acceptance rule).
__global__ void __launch_bounds__(kThreads) k_true_residual(const InstDev* insts, const Tile* tiles, int ntiles) {
  __shared__ double sh[32];
  __shared__ int flag;
  for_active_tiles(insts, tiles, ntiles, [](const InstDev& I) {
    const Ctrl* c = I.ctrl;
    return !c->done && (c->candidate || (c->true_every > 0 && c->iter % c->true_every == 0));
  }, [&](int t) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    Ctrl* c = I.ctrl;
    const int done = c->done, cand = c->candidate, every = c->true_every, iter = c->iter;
    if (done || (!cand && !(every > 0 && iter % every == 0))) return;
    const LevelDev L = I.lv[0];
    const int nt0 = I.ntiles0;
    double* partial = I.partial;
    float* __restrict__ r = static_cast<float*>(L.rhs);
    const float* __restrict__ Xh = I.x;
    const float* __restrict__ Xl = I.xlo;
    const float* __restrict__ B = I.b;
    const float* __restrict__ dg = L.diag;
    const uint8_t* __restrict__ lab = L.label;
    auto X = [&](int j) { return double(Xh[j]) + double(Xl[j]); };
    double rr = 0, mr = 0;
    const int sy = L.nx, sz = L.nx * L.ny;
    const TileIt it(tl.tile, L.nx, L.ny, L.nz, L.depth);
    const int x = it.x, y = it.y;
    // neighbour sums need no label: x is zero on air cells
    double sv[kMaxDepth], av[kMaxDepth];
    float bv[kMaxDepth];
    uint8_t lb[kMaxDepth];
    const float* ff = L.ff;
    const long long n = L.n;
    for_column(it, L.nx, L.ny, L.nz, [&](int k, int zz, int i) {
      double s = 0;
      s += x > 0 ? double(face_w(ff, n, 0, i - 1, 1.0f)) * X(i - 1) : 0.0;
      s += x + 1 < L.nx ? double(face_w(ff, n, 0, i, 1.0f)) * X(i + 1) : 0.0;
      s += y > 0 ? double(face_w(ff, n, 1, i - sy, 1.0f)) * X(i - sy) : 0.0;
      s += y + 1 < L.ny ? double(face_w(ff, n, 1, i, 1.0f)) * X(i + sy) : 0.0;
      s += zz > 0 ? double(face_w(ff, n, 2, i - sz, 1.0f)) * X(i - sz) : 0.0;
      s += zz + 1 < L.nz ? double(face_w(ff, n, 2, i, 1.0f)) * X(i + sz) : 0.0;
      lb[k] = lab[i];
      sv[k] = s;
      av[k] = double(dg[i]) * X(i);
      bv[k] = B[i];
    });
    for_column(it, L.nx, L.ny, L.nz, [&](int k, int, int i) {
      if (!lb[k]) return;
      const double rv = double(bv[k]) - (av[k] - sv[k]);
      r[i] = float(rv);
      rr += rv * rv;
      mr = fmax(mr, fabs(rv));
    });
    const double a0 = block_sum(rr, sh), a1 = block_max(mr, sh);
    if (threadIdx.x == 0) {
      partial[tl.tile] = a0;
      partial[nt0 + tl.tile] = a1;
    }
    if (arrive_last(&c->arrive[kStTrue], nt0, &flag)) {
      const double s = gather_slot(partial, 0, nt0, 0, sh);
      const double m = gather_slot(partial, 1, nt0, 1, sh);
      if (threadIdx.x == 0) finish_true(c, s, m);
    }
  });
}

// ================================================================= projection
// One face of the projected velocity, evaluated in float64 from the double-single
// pressures of its two cells (zero on air cells) and rounded once to the stored
// float32.  li, lj: the cells are liquid; phi_*: their level sets.
__device__ __forceinline__ float face_value(bool li, bool lj, float phi_i, float phi_j, double pi, double pj,
                                            float u) {
  if (!li && !lj) return 0.0f;
  float th = 1.0f;
  if (li && !lj) th = ghost_theta(phi_i, phi_j);
  if (!li && lj) th = ghost_theta(phi_j, phi_i);
  return float(double(u) - (pj - pi) / double(th));
}

// Gradient subtract (webgpu-uniform-reference.wgsl.ts:1052-1099 / atlas
// pressureCorrection :1263-1279): each cell owns its three positive faces and,
// on the low domain walls, its negative faces.  Closed walls and faces with no
// liquid side are zero.  Also publishes the pressure in Pa.  Every load of a
// cell (labels, pressures and level sets of the cell and its +x, +y, +z
// neighbours, the three faces) is issued together; the labels select what is
// used afterwards, so no load waits for another.
__global__ void __launch_bounds__(kThreads, 3) k_grad(const InstDev* insts, const Tile* tiles, int ntiles) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    const Ctrl* c = I.ctrl;
    if (c->status == FLUID_PP_NONFINITE) continue;   // fail closed: keep the previous state
    const LevelDev& L = I.lv[0];
    const int nx = I.nx, ny = I.ny, nz = I.nz, sz = nx * ny;
    const long long uS = nx + 1, vS = ny + 1;
    const uint8_t* __restrict__ lab = L.label;
    const float* __restrict__ phi = L.phi;
    const float* __restrict__ Xh = I.x;
    const float* __restrict__ Xl = I.xlo;
    float* __restrict__ U = I.u;
    float* __restrict__ V = I.v;
    float* __restrict__ W = I.w;
    float* __restrict__ P = I.p_si;
    const bool open_top = I.open_top;
    const double pscale = double(I.pscale);
    const TileIt it(tl.tile, nx, ny, nz, L.depth);
    const int x = it.x, y = it.y;
    const bool hx = x + 1 < nx, hy = y + 1 < ny;
    for_column(it, nx, ny, nz, [&](int, int z, int i) {
      const bool hz = z + 1 < nz;
      const long long urow = uS * (y + (long long)ny * z);
      const long long vcol = x + (long long)nx * vS * z;
      const long long fu_i = urow + x + 1, fv_i = vcol + (long long)nx * (y + 1), fw_i = (long long)i + sz;
      const int jx = hx ? i + 1 : i, jy = hy ? i + nx : i, jz = hz ? i + sz : i;
      const bool l0 = lab[i], lx = hx && lab[jx], ly = hy && lab[jy], lz = hz && lab[jz];
      const float xh0 = Xh[i], xl0 = Xl[i], xhx = Xh[jx], xlx = Xl[jx], xhy = Xh[jy], xly = Xl[jy], xhz = Xh[jz],
                  xlz = Xl[jz];
      const float f0 = phi[i], fx = phi[jx], fy = phi[jy], fz = phi[jz];
      const float u = hx ? U[fu_i] : 0.0f, v = V[fv_i], w = hz ? W[fw_i] : 0.0f;
      const double p0 = l0 ? double(xh0) + double(xl0) : 0.0;
      const double px = lx ? double(xhx) + double(xlx) : 0.0;
      const double py = ly ? double(xhy) + double(xly) : 0.0;
      const double pz = lz ? double(xhz) + double(xlz) : 0.0;
      U[fu_i] = hx ? face_value(l0, lx, f0, fx, p0, px, u) : 0.0f;
      if (x == 0) U[urow] = 0.0f;
      float nv = 0.0f;
      if (hy) nv = face_value(l0, ly, f0, fy, p0, py, v);
      else if (open_top && l0) nv = float(double(v) + p0 / double(ghost_theta(f0, 0.5f)));
      V[fv_i] = nv;
      if (y == 0) V[vcol] = 0.0f;
      W[fw_i] = hz ? face_value(l0, lz, f0, fz, p0, pz, w) : 0.0f;
      if (z == 0) W[i] = 0.0f;
      P[i] = float(p0 * pscale);
    });
  }
}

// Post-projection divergence receipts (atlas divergenceFromEquationResidual,
// :1283-1296): max and sum of squares of (div u - q) before and after.
// k_receipt_part writes each tile's partials; k_receipt_finish folds them per
// instance in tile order.
__global__ void __launch_bounds__(kThreads, 2) k_receipt_part(const InstDev* insts, const Tile* tiles, int ntiles) {
  __shared__ double sh[4 * 32];
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    const LevelDev& L = I.lv[0];
    const int nx = I.nx, ny = I.ny, nz = I.nz;
    const long long uS = nx + 1, vS = ny + 1, sz = (long long)nx * ny;
    const float* __restrict__ U = I.u;
    const float* __restrict__ V = I.v;
    const float* __restrict__ W = I.w;
    const float* __restrict__ vof = I.vof;
    const float* __restrict__ B = I.b;
    const uint8_t* __restrict__ lab = L.label;
    const float hdt = I.h / I.dt;
    double sums[2] = {0, 0}, maxes[2] = {0, 0};   // after, before
    const TileIt it(tl.tile, L.nx, L.ny, L.nz, L.depth);
    const int x = it.x, y = it.y;
    // labels first, then the liquid cells' faces, VOF and right-hand side
    uint8_t lb[kMaxDepth];
    for_column(it, nx, ny, nz, [&](int k, int, int i) { lb[k] = lab[i]; });
    float up[kMaxDepth], um[kMaxDepth], vp[kMaxDepth], vm[kMaxDepth], wp[kMaxDepth], wm[kMaxDepth], rv[kMaxDepth],
        bv[kMaxDepth];
    for_column(it, nx, ny, nz, [&](int k, int z, int i) {
      if (!lb[k]) return;
      const long long urow = uS * (y + (long long)ny * z);
      const long long vcol = x + (long long)nx * vS * z;
      up[k] = U[urow + x + 1];
      um[k] = U[urow + x];
      vp[k] = V[vcol + (long long)nx * (y + 1)];
      vm[k] = V[vcol + (long long)nx * y];
      wp[k] = W[i + sz];
      wm[k] = W[i];
      rv[k] = vof[i];
      bv[k] = B[i];
    });
    for_column(it, nx, ny, nz, [&](int k, int, int) {
      if (!lb[k]) return;
      const double du = double(up[k]) - double(um[k]);
      const double dv = double(vp[k]) - double(vm[k]);
      const double dw = double(wp[k]) - double(wm[k]);
      const float rho = rv[k];
      double q = 0.0;
      if (rho > 1.0f) q = fminf(fminf(0.5f * (rho - 1.0f), 1.0f), hdt);
      const double after = (du + dw) + dv - q;
      const double before = -double(bv[k]);
      maxes[0] = fmax(maxes[0], fabs(after));
      sums[0] += after * after;
      maxes[1] = fmax(maxes[1], fabs(before));
      sums[1] += before * before;
    });
    block_folds<2, 2>(sums, maxes, sh);
    if (threadIdx.x == 0) {
      I.partial[0 * I.ntiles0 + tl.tile] = maxes[0];
      I.partial[1 * I.ntiles0 + tl.tile] = sums[0];
      I.partial[2 * I.ntiles0 + tl.tile] = maxes[1];
      I.partial[3 * I.ntiles0 + tl.tile] = sums[1];
    }
  }
}

// The four receipt norms of each listed instance (one CTA each).
__global__ void __launch_bounds__(kThreads) k_receipt_finish(const InstDev* insts, const int* ilist) {
  __shared__ double sh[32];
  const InstDev& I = insts[ilist[blockIdx.x]];
  Ctrl* c = I.ctrl;
  const int nt0 = I.ntiles0;
  const double r0 = gather_slot(I.partial, 0, nt0, 1, sh);
  const double r1 = gather_slot(I.partial, 1, nt0, 0, sh);
  const double r2 = gather_slot(I.partial, 2, nt0, 1, sh);
  const double r3 = gather_slot(I.partial, 3, nt0, 0, sh);
  if (threadIdx.x == 0) {
    c->red[0] = r0;
    c->red[1] = r1;
    c->red[2] = r2;
    c->red[3] = r3;
  }
}

// End of one CG iteration inside the device-side loop: keep looping while any
// instance is unfinished, never more than `cap` times (the loop counter is
// reset by k_reset_ctrl).
__global__ void k_loop_cond(const InstDev* insts, int n, unsigned* counter, unsigned cap,
                            cudaGraphConditionalHandle handle) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += blockDim.x)
    if (!insts[k].ctrl->done) atomicOr(&any, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned c = *counter + 1;
    *counter = c;
    cudaGraphSetConditional(handle, (any && c < cap) ? 1u : 0u);
  }
}

// Clears the control words a solve accumulates into (counts and done flag).
__global__ void k_reset_ctrl(const InstDev* insts, int n, unsigned* loop_counter) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k == 0 && loop_counter) *loop_counter = 0u;
  if (k >= n) return;
  Ctrl* c = insts[k].ctrl;
  c->liquid = 0;
  c->air = 0;
  c->top_liquid = 0;
  c->nonfinite = 0;
  c->done = 0;
  c->candidate = 0;
  c->status = 0;
  c->converged = 0;
  c->iter = 0;
}

// Test hook: make the solve-loop kernels run with the given scale.
__global__ void k_hook_ctrl(const InstDev* insts, double sigma) {
  Ctrl* c = insts[0].ctrl;
  c->done = 0;
  c->sigma = sigma;
  c->gamma = 1.0;
  c->status = 0;
  c->dsel = 0;
}

}  // namespace fpp
