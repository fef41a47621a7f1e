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
    const long long uS = I.nx + 1, vS = I.ny + 1;
    int x, y, z, i;
    for (TileIt it(tl.tile, I.nx, I.ny, I.nz); it.next(x, y, z, i);) {
      const float rho = I.vof[i];
      const bool liq = rho > 0.5f;
      L.label[i] = liq ? 1 : 0;
      L.phi[i] = 0.5f - rho;
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
      if (!(warm && liq)) {
        I.x[i] = 0.0f;
        I.xlo[i] = 0.0f;
      }
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
    int x, y, z, i;
    for (TileIt it(tl.tile, C.nx, C.ny, C.nz); it.next(x, y, z, i);) {
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
    const int sy = L.nx, sz = L.nx * L.ny;
    int x, y, z, i;
    for (TileIt it(tl.tile, L.nx, L.ny, L.nz); it.next(x, y, z, i);) {
      float d = 0.0f;
      if (L.label[i]) {
        const float ph = L.phi[i];
        auto term = [&](bool inside, int j, float w) -> float {
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

// Dense inverse of the coarsest (normalised) operator, one CTA per instance.
// Air cells are identity rows; a level without Dirichlet contact gets the
// rank-one term mean(diag)/m * 1 1^T so the inverse is SPD.
template <class TD>
__global__ void k_coarse_factor(const InstDev* insts, const int* list) {
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
    if (x > 0 && L.label[i - 1]) A[i * m + i - 1] = -L.wx;
    if (x + 1 < L.nx && L.label[i + 1]) A[i * m + i + 1] = -L.wx;
    if (y > 0 && L.label[i - sy]) A[i * m + i - sy] = -L.wy;
    if (y + 1 < L.ny && L.label[i + sy]) A[i * m + i + sy] = -L.wy;
    if (z > 0 && L.label[i - sz]) A[i * m + i - sz] = -L.wz;
    if (z + 1 < L.nz && L.label[i + sz]) A[i * m + i + sz] = -L.wz;
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
  // In-place Gauss-Jordan inversion (SPD: no pivoting needed).
  for (int k = 0; k < m; ++k) {
    const double piv = A[k * m + k];
    for (int j = threadIdx.x; j < m; j += blockDim.x) {
      pivot_row[j] = (j == k ? 1.0 : A[k * m + j]) / piv;
      pivot_col[j] = A[j * m + k];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
      const int i = e / m, j = e - i * m;
      if (i == k) A[e] = pivot_row[j];
      else A[e] = ((j == k) ? 0.0 : A[e]) - pivot_col[i] * pivot_row[j];
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < m * m; e += blockDim.x) I.coarse_inv[e] = A[e];
}

// ================================================================= CG scalars
enum Stage { kStInit = 0, kStGamma = 1, kStSpmv = 2, kStUpdate = 3, kStTrue = 4, kStReceipt = 5 };

__device__ __forceinline__ void set_sigma(Ctrl* c, double rr) {
  const double per = rr / double(c->liquid > 0 ? c->liquid : 1);
  c->sigma = per > 1e-300 ? 1.0 / sqrt(per) : 1.0;
}

// r = b - A x (x already masked to liquid), bb, sums for the nullspace.
__global__ void k_cg_init(const InstDev* insts, const Tile* tiles, int ntiles, double rel_tol, double abs_tol,
                          int max_iter, int true_every, int warm, double rel_tol_inf) {
  __shared__ double sh[32];
  __shared__ int flag;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const InstDev& I = insts[tl.inst];
    Ctrl* c = I.ctrl;
    const LevelDev& L = I.lv[0];
    float* r = static_cast<float*>(L.rhs);
    double sbb = 0, sb = 0, srr = 0, mb = 0, mr = 0;
    const int sy = L.nx, sz = L.nx * L.ny;
    int x, y, z, i;
    for (TileIt it(tl.tile, L.nx, L.ny, L.nz); it.next(x, y, z, i);) {
      const float b = I.b[i];
      float rv = b;
      if (warm && L.label[i]) {
        auto X = [&](int j) { return double(I.x[j]) + double(I.xlo[j]); };
        auto nb = [&](bool in, int j) { return (in && L.label[j]) ? X(j) : 0.0; };
        const double s = ((nb(x > 0, i - 1) + nb(x + 1 < L.nx, i + 1)) + (nb(z > 0, i - sz) + nb(z + 1 < L.nz, i + sz))) +
                         (nb(y > 0, i - sy) + nb(y + 1 < L.ny, i + sy));
        rv = float(double(b) - (double(L.diag[i]) * X(i) - s));
      }
      r[i] = rv;
      sbb += double(b) * b;
      sb += b;
      srr += double(rv) * rv;
      mb = fmax(mb, fabs(double(b)));
      mr = fmax(mr, fabs(double(rv)));
    }
    const double a0 = block_sum(sbb, sh), a1 = block_sum(sb, sh), a2 = block_sum(srr, sh);
    const double a3 = block_max(mb, sh), a4 = block_max(mr, sh);
    if (threadIdx.x == 0) {
      I.partial[0 * I.ntiles0 + tl.tile] = a0;
      I.partial[1 * I.ntiles0 + tl.tile] = a1;
      I.partial[2 * I.ntiles0 + tl.tile] = a2;
      I.partial[3 * I.ntiles0 + tl.tile] = a3;
      I.partial[4 * I.ntiles0 + tl.tile] = a4;
    }
    if (arrive_last(&c->arrive[kStInit], I.ntiles0, &flag)) {
      const double bb = gather_slot(I.partial, 0, I.ntiles0, 0, sh);
      const double bs = gather_slot(I.partial, 1, I.ntiles0, 0, sh);
      const double rr = gather_slot(I.partial, 2, I.ntiles0, 0, sh);
      const double bmax = gather_slot(I.partial, 3, I.ntiles0, 1, sh);
      const double rmax = gather_slot(I.partial, 4, I.ntiles0, 1, sh);
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
    for (TileIt it(tl.tile, L.nx, L.ny, L.nz); it.next(x, y, z, i);) {
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
    const int sy = L.nx, sz = L.nx * L.ny;
    int x, y, z, i;
    for (TileIt it(tl.tile, L.nx, L.ny, L.nz); it.next(x, y, z, i);) {
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
        auto nb = [&](bool in, int j, float w) { return in ? w * St<TZ>::ld(L.z, j) : 0.0f; };
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
    const int sy = L.nx, sz = L.nx * L.ny;
    int x, y, z, i;
    for (TileIt it(tl.tile, L.nx, L.ny, L.nz); it.next(x, y, z, i);) {
      float r = 0.0f;
      if (L.label[i]) {
        auto nb = [&](bool in, int j, float w) { return in ? w * St<TZ>::ld(L.z, j) : 0.0f; };
        const float s = d4sum6(nb(x > 0, i - 1, L.wx), nb(x + 1 < L.nx, i + 1, L.wx), nb(y > 0, i - sy, L.wy),
                               nb(y + 1 < L.ny, i + sy, L.wy), nb(z > 0, i - sz, L.wz), nb(z + 1 < L.nz, i + sz, L.wz));
        r = scale * (St<TR>::ld(L.rhs, i) - (St<TD>::ld(L.diagT, i) * St<TZ>::ld(L.z, i) - s));
      }
      St<TS>::st(L.res, i, r);
    }
  }
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
    int X, Y, Z, i;
    for (TileIt it(tl.tile, C.nx, C.ny, C.nz); it.next(X, Y, Z, i);) {
      float acc = 0.0f;
      if (C.label[i]) {
        int fx[4], fy[4], fz[4];
        float wx[4], wy[4], wz[4];
        int nxx = 0, nyy = 0, nzz = 0;
        auto axis = [](int stride, int c, int nc, int nf, int* f, float* w) {
          if (stride == 1) {
            f[0] = c;
            w[0] = 1.0f;
            return 1;
          }
          int n = 0;
          for (int q = 2 * c - 1; q <= 2 * c + 2; ++q)
            if (q >= 0 && q < nf) {
              f[n] = q;
              w[n] = p1d(q, c, nc);
              ++n;
            }
          return n;
        };
        nxx = axis(C.sx, X, C.nx, F.nx, fx, wx);
        nyy = axis(C.sy, Y, C.ny, F.ny, fy, wy);
        nzz = axis(C.sz, Z, C.nz, F.nz, fz, wz);
        for (int c2 = 0; c2 < nzz; ++c2) {
          for (int c1 = 0; c1 < nyy; ++c1) {
            const float wyz = wz[c2] * wy[c1];
            const int row = F.nx * (fy[c1] + F.ny * fz[c2]);
            float s = 0.0f;
            for (int c0 = 0; c0 < nxx; ++c0) s += wx[c0] * St<TS>::ld(F.res, row + fx[c0]);
            acc += wyz * s;
          }
        }
        acc *= scale;
      }
      St<TS>::st(C.rhs, i, acc);
    }
  }
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
    int x, y, z, i;
    for (TileIt it(tl.tile, F.nx, F.ny, F.nz); it.next(x, y, z, i);) {
      if (!F.label[i]) continue;
      int cx[2], cy[2], cz[2];
      float wx[2], wy[2], wz[2];
      const int nxx = taps1d(x, C.sx, C.nx, cx, wx);
      const int nyy = taps1d(y, C.sy, C.ny, cy, wy);
      const int nzz = taps1d(z, C.sz, C.nz, cz, wz);
      float s = 0.0f;
      for (int c2 = 0; c2 < nzz; ++c2)
        for (int c1 = 0; c1 < nyy; ++c1)
          for (int c0 = 0; c0 < nxx; ++c0)
            s += wx[c0] * wy[c1] * wz[c2] * St<TZC>::ld(C.z, cx[c0] + C.nx * (cy[c1] + C.ny * cz[c2]));
      St<TZF>::st(F.z, i, St<TZF>::ld(F.z, i) + s * unscale);
    }
  }
}

// The small levels of the V-cycle in one CTA per instance, in shared memory:
// levels first..nlev-1 (each at most kCoarseBlockCells) are loaded, smoothed,
// restricted, solved densely at the coarsest, prolongated and smoothed again
// with the same arithmetic as the grid kernels, then z of level `first` is
// written back for the prolongation into the finer grid level.
template <class T>
__global__ void k_coarse_block(const InstDev* insts, const int* list, int pre, int post) {
  extern __shared__ float smem[];
  const InstDev& I = insts[list[blockIdx.x]];
  if (I.ctrl->done) return;
  const int first = I.first_block, last = I.nlev - 1;
  float* zs[kMaxLevels];
  float* rs[kMaxLevels];
  float* es[kMaxLevels];
  float* ds[kMaxLevels];
  uint8_t* ls[kMaxLevels];
  {
    float* p = smem;
    for (int l = first; l <= last; ++l) {
      const int n = int(I.lv[l].n);
      zs[l] = p; p += n;
      rs[l] = p; p += n;
      es[l] = p; p += n;
      ds[l] = p; p += n;
    }
    uint8_t* q = reinterpret_cast<uint8_t*>(p);
    for (int l = first; l <= last; ++l) {
      ls[l] = q;
      q += (I.lv[l].n + 3) & ~3LL;
    }
  }
  for (int l = first; l <= last; ++l) {
    const LevelDev& L = I.lv[l];
    for (int i = threadIdx.x; i < int(L.n); i += blockDim.x) {
      ds[l][i] = St<T>::ld(L.diagT, i);
      ls[l][i] = L.label[i];
      if (l == first) rs[l][i] = St<T>::ld(L.rhs, i);
    }
  }
  __syncthreads();
  auto nbsum = [&](const LevelDev& L, const float* z, int i, int x, int y, int zz) {
    const int sy = L.nx, sz = L.nx * L.ny;
    auto nb = [&](bool in, int j, float w) { return in ? w * z[j] : 0.0f; };
    return d4sum6(nb(x > 0, i - 1, L.wx), nb(x + 1 < L.nx, i + 1, L.wx), nb(y > 0, i - sy, L.wy),
                  nb(y + 1 < L.ny, i + sy, L.wy), nb(zz > 0, i - sz, L.wz), nb(zz + 1 < L.nz, i + sz, L.wz));
  };
  auto pass = [&](int l, int colour, int zero_init) {
    const LevelDev& L = I.lv[l];
    float* z = zs[l];
    for (int i = threadIdx.x; i < int(L.n); i += blockDim.x) {
      int x, y, zz;
      decode(i, L.nx, L.ny, x, y, zz);
      if (((x + y + zz) & 1) != colour) {
        if (zero_init) z[i] = 0.0f;
        continue;
      }
      if (!ls[l][i]) {
        z[i] = 0.0f;
        continue;
      }
      const float s = zero_init ? 0.0f : nbsum(L, z, i, x, y, zz);
      z[i] = (rs[l][i] + s) / ds[l][i];
    }
    __syncthreads();
  };
  // down
  for (int l = first; l < last; ++l) {
    const LevelDev& L = I.lv[l];
    for (int sw = 0; sw < pre; ++sw) {
      pass(l, 0, sw == 0);
      pass(l, 1, 0);
    }
    if (pre == 0) pass(l, 2, 1);
    for (int i = threadIdx.x; i < int(L.n); i += blockDim.x) {
      float r = 0.0f;
      if (ls[l][i]) {
        int x, y, zz;
        decode(i, L.nx, L.ny, x, y, zz);
        r = rs[l][i] - (ds[l][i] * zs[l][i] - nbsum(L, zs[l], i, x, y, zz));
      }
      es[l][i] = r;
    }
    __syncthreads();
    const LevelDev& C = I.lv[l + 1];
    const float scale = L.to_coarse / float((C.sx == 2 ? 2 : 1) * (C.sy == 2 ? 2 : 1) * (C.sz == 2 ? 2 : 1));
    for (int i = threadIdx.x; i < int(C.n); i += blockDim.x) {
      float acc = 0.0f;
      if (ls[l + 1][i]) {
        int X, Y, Z;
        decode(i, C.nx, C.ny, X, Y, Z);
        const int x0 = C.sx == 2 ? max(2 * X - 1, 0) : X, x1 = C.sx == 2 ? min(2 * X + 2, L.nx - 1) : X;
        const int y0 = C.sy == 2 ? max(2 * Y - 1, 0) : Y, y1 = C.sy == 2 ? min(2 * Y + 2, L.ny - 1) : Y;
        const int z0 = C.sz == 2 ? max(2 * Z - 1, 0) : Z, z1 = C.sz == 2 ? min(2 * Z + 2, L.nz - 1) : Z;
        for (int fz = z0; fz <= z1; ++fz) {
          const float wz = C.sz == 2 ? p1d(fz, Z, C.nz) : 1.0f;
          for (int fy = y0; fy <= y1; ++fy) {
            const float wyz = wz * (C.sy == 2 ? p1d(fy, Y, C.ny) : 1.0f);
            const int row = L.nx * (fy + L.ny * fz);
            float s = 0.0f;
            for (int fx = x0; fx <= x1; ++fx) s += (C.sx == 2 ? p1d(fx, X, C.nx) : 1.0f) * es[l][row + fx];
            acc += wyz * s;
          }
        }
        acc *= scale;
      }
      rs[l + 1][i] = acc;
    }
    __syncthreads();
  }
  // coarsest: dense float64 inverse
  {
    const LevelDev& L = I.lv[last];
    const int m = int(L.n);
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
      double s = 0;
      const double* row = I.coarse_inv + (long long)i * m;
      for (int j = 0; j < m; ++j) s += row[j] * (ls[last][j] ? double(rs[last][j]) : 0.0);
      zs[last][i] = ls[last][i] ? float(s) : 0.0f;
    }
    __syncthreads();
  }
  // up
  for (int l = last - 1; l >= first; --l) {
    const LevelDev& F = I.lv[l];
    const LevelDev& C = I.lv[l + 1];
    for (int i = threadIdx.x; i < int(F.n); i += blockDim.x) {
      if (!ls[l][i]) continue;
      int x, y, zz;
      decode(i, F.nx, F.ny, x, y, zz);
      int cx[2], cy[2], cz[2];
      float wx[2], wy[2], wz[2];
      const int nxx = taps1d(x, C.sx, C.nx, cx, wx);
      const int nyy = taps1d(y, C.sy, C.ny, cy, wy);
      const int nzz = taps1d(zz, C.sz, C.nz, cz, wz);
      float s = 0.0f;
      for (int c2 = 0; c2 < nzz; ++c2)
        for (int c1 = 0; c1 < nyy; ++c1)
          for (int c0 = 0; c0 < nxx; ++c0)
            s += wx[c0] * wy[c1] * wz[c2] * zs[l + 1][cx[c0] + C.nx * (cy[c1] + C.ny * cz[c2])];
      zs[l][i] += s;
    }
    __syncthreads();
    for (int sw = 0; sw < post; ++sw) {
      pass(l, 1, 0);
      pass(l, 0, 0);
    }
  }
  const LevelDev& Lf = I.lv[first];
  for (int i = threadIdx.x; i < int(Lf.n); i += blockDim.x) St<T>::st(Lf.z, i, zs[first][i]);
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
    int x, y, zz, i;
    for (TileIt it(tl.tile, L.nx, L.ny, L.nz); it.next(x, y, zz, i);) {
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
    int x, y, zz, i;
    for (TileIt it(tl.tile, L.nx, L.ny, L.nz); it.next(x, y, zz, i);)
      I.d[i] = L.label[i] ? (z[i] - zm) + beta * I.d[i] : 0.0f;
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
    const int sy = L.nx, sz = L.nx * L.ny;
    int x, y, z, i;
    for (TileIt it(tl.tile, L.nx, L.ny, L.nz); it.next(x, y, z, i);) {
      float q = 0.0f;
      if (L.label[i]) {
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

// x += alpha d (double-single), r -= alpha q, rr = r . r, max |r|.
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
    const double alpha = c->alpha;
    const float alpha_f = float(alpha);
    double rr = 0, mr = 0;
    int x, y, z, i;
    for (TileIt it(tl.tile, L.nx, L.ny, L.nz); it.next(x, y, z, i);) {
      if (!L.label[i]) continue;
      // double-single accumulation: x_hi + x_lo carries the pressure to ~1e-14
      const double xv = double(I.x[i]) + double(I.xlo[i]) + alpha * double(I.d[i]);
      const float hi = float(xv);
      I.x[i] = hi;
      I.xlo[i] = float(xv - double(hi));
      const float rv = r[i] - alpha_f * I.q[i];
      r[i] = rv;
      rr += double(rv) * rv;
      mr = fmax(mr, fabs(double(rv)));
    }
    const double a0 = block_sum(rr, sh), a1 = block_max(mr, sh);
    if (threadIdx.x == 0) {
      I.partial[tl.tile] = a0;
      I.partial[I.ntiles0 + tl.tile] = a1;
    }
    if (arrive_last(&c->arrive[kStUpdate], I.ntiles0, &flag)) {
      const double s = gather_slot(I.partial, 0, I.ntiles0, 0, sh);
      const double m = gather_slot(I.partial, 1, I.ntiles0, 1, sh);
      if (threadIdx.x == 0) {
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
    auto X = [&](int j) { return double(I.x[j]) + double(I.xlo[j]); };
    double rr = 0, mr = 0;
    const int sy = L.nx, sz = L.nx * L.ny;
    int x, y, z, i;
    for (TileIt it(tl.tile, L.nx, L.ny, L.nz); it.next(x, y, z, i);) {
      if (!L.label[i]) continue;
      double s = 0;
      if (x > 0) s += X(i - 1);
      if (x + 1 < L.nx) s += X(i + 1);
      if (y > 0) s += X(i - sy);
      if (y + 1 < L.ny) s += X(i + sy);
      if (z > 0) s += X(i - sz);
      if (z + 1 < L.nz) s += X(i + sz);
      const double rv = double(I.b[i]) - (double(L.diag[i]) * X(i) - s);
      r[i] = float(rv);
      rr += rv * rv;
      mr = fmax(mr, fabs(rv));
    }
    const double a0 = block_sum(rr, sh), a1 = block_max(mr, sh);
    if (threadIdx.x == 0) {
      I.partial[tl.tile] = a0;
      I.partial[I.ntiles0 + tl.tile] = a1;
    }
    if (arrive_last(&c->arrive[kStTrue], I.ntiles0, &flag)) {
      const double s = gather_slot(I.partial, 0, I.ntiles0, 0, sh);
      const double m = gather_slot(I.partial, 1, I.ntiles0, 1, sh);
      if (threadIdx.x == 0) {
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
    }
  }
}

// ================================================================= projection
// One face of the projected velocity, evaluated in float64 from the double-single
// pressure and rounded once to the stored float32.
__device__ __forceinline__ float face_update(const InstDev& I, const LevelDev& L, int i, int j, float u) {
  const bool li = L.label[i], lj = L.label[j];
  if (!li && !lj) return 0.0f;
  float th = 1.0f;
  if (li && !lj) th = ghost_theta(L.phi[i], L.phi[j]);
  if (!li && lj) th = ghost_theta(L.phi[j], L.phi[i]);
  const double pi = li ? double(I.x[i]) + double(I.xlo[i]) : 0.0;
  const double pj = lj ? double(I.x[j]) + double(I.xlo[j]) : 0.0;
  return float(double(u) - (pj - pi) / double(th));
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
    const long long uS = I.nx + 1, vS = I.ny + 1;
    int x, y, z, i;
    for (TileIt it(tl.tile, L.nx, L.ny, L.nz); it.next(x, y, z, i);) {
      const long long urow = uS * (y + (long long)I.ny * z);
      const long long vcol = x + (long long)I.nx * vS * z;
      const int sz = I.nx * I.ny;
      const double pi = L.label[i] ? double(I.x[i]) + double(I.xlo[i]) : 0.0;
      {
        const long long f = urow + x + 1;
        I.u[f] = x + 1 < I.nx ? face_update(I, L, i, i + 1, I.u[f]) : 0.0f;
        if (x == 0) I.u[urow] = 0.0f;
      }
      {
        const long long f = vcol + (long long)I.nx * (y + 1);
        float nv = 0.0f;
        if (y + 1 < I.ny) nv = face_update(I, L, i, i + I.nx, I.v[f]);
        else if (I.open_top && L.label[i]) nv = float(double(I.v[f]) + pi / double(ghost_theta(L.phi[i], 0.5f)));
        I.v[f] = nv;
        if (y == 0) I.v[vcol] = 0.0f;
      }
      {
        const long long f = (long long)i + sz;
        I.w[f] = z + 1 < I.nz ? face_update(I, L, i, i + sz, I.w[f]) : 0.0f;
        if (z == 0) I.w[i] = 0.0f;
      }
      I.p_si[i] = float(pi * double(I.pscale));
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
    const long long uS = I.nx + 1, vS = I.ny + 1;
    int x, y, z, i;
    for (TileIt it(tl.tile, L.nx, L.ny, L.nz); it.next(x, y, z, i);) {
      if (!L.label[i]) continue;
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
}

}  // namespace fpp
