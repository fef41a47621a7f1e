// Fused V-cycle and CG kernels for the default schedule (one red-black sweep
// before and after each coarse correction).
//
// Each CTA owns one tile and stages the tile plus the halo its chain of
// stencils needs in shared memory, so that a level's whole down step
// (pre-smooth from zero, residual, restriction) or up step (prolongation,
// post-smooth) is one launch reading its inputs once:
//
//   down, level l, coarse tile C:   I = fine cells of C, F = I + restriction taps,
//     load rhs/diag/label on H = F +- 2, red z on H (pointwise from rhs: the
//     sweep starts at zero), black z on G = F +- 1, residual on F, restrict to C.
//   up, level l, fine tile T:       load z, rhs, diag, label on E = T +- 2 and the
//     coarse z under E, prolongate on E, black on T +- 1, red on T.
//
// The down step leaves its z in the level's scratch array (LevelDev::res) and
// the up step writes the final z to LevelDev::z: a launch never reads, in its
// halo, an array that other CTAs of the same launch write.
//
// The halo cells are recomputed by every CTA that needs them, with the same
// arithmetic in the same order as the owner, so the result does not depend on
// the tiling.  Cells outside the lattice are staged as air with z = 0, which
// reproduces the wall rule of the grid kernels (an out-of-range neighbour
// contributes nothing).  Values are rounded to the level's storage type where
// the grid kernels store them, so both schedules apply the same operator.
#pragma once
#include "kernels.cuh"

namespace fpp {

// ------------------------------------------------------------ index helpers
// floor(n / d) for 0 <= n < 2^16, 1 <= d < 2^16 with m = magic_of(d): with
// m = ceil(2^32 / d) the error m*d - 2^32 < d keeps n*m / 2^32 exact.
__device__ __forceinline__ unsigned magic_of(unsigned d) { return d <= 1 ? 0u : 0xFFFFFFFFu / d + 1u; }
__device__ __forceinline__ unsigned div_m(unsigned n, unsigned d, unsigned m) { return d <= 1 ? n : __umulhi(n, m); }

// A box of cells staged in shared memory: global origin and extents, x fastest.
struct SBox {
  int x0, y0, z0, ex, ey, ez;
  __device__ __forceinline__ int count() const { return ex * ey * ez; }
  __device__ __forceinline__ int at(int gx, int gy, int gz) const {
    return (gx - x0) + ex * ((gy - y0) + ey * (gz - z0));
  }
};

// Calls f(gx, gy, gz, s) for the cells of the sub-box [rx0, rx0 + rex) x ... of
// colour `colour` (0: (x + y + z) even, 1: odd, 2: all), s = index in B.  For a
// single colour rex must be even: every row then holds rex / 2 such cells, and
// consecutive threads take consecutive cells of one colour.
template <class Fn>
__device__ __forceinline__ void for_box(const SBox& B, int rx0, int ry0, int rz0, int rex, int rey, int rez,
                                        int colour, Fn f) {
  const int w = colour == 2 ? rex : (rex >> 1);
  const unsigned n = unsigned(w * rey * rez);
  const unsigned mw = magic_of(unsigned(w)), my = magic_of(unsigned(rey));
  for (unsigned e = threadIdx.x; e < n; e += blockDim.x) {
    const unsigned r = div_m(e, unsigned(w), mw);
    const int lx = int(e - r * unsigned(w));
    const unsigned lz = div_m(r, unsigned(rey), my);
    const int gy = ry0 + int(r - lz * unsigned(rey)), gz = rz0 + int(lz);
    const int gx = colour == 2 ? rx0 + lx : rx0 + 2 * lx + ((rx0 + gy + gz + colour) & 1);
    f(gx, gy, gz, B.at(gx, gy, gz));
  }
}

// Stages every cell of box B: ld(gx, gy, gz, ok) returns the cell's values (its
// global loads), st(s, gx, gy, gz, v) writes them to shared memory.  Each
// thread runs K cells at a time with all their loads issued before the first
// store, so a thread keeps K cells' loads in flight instead of one.
template <int K, class V, class Ld, class St>
__device__ __forceinline__ void stage_box(const SBox& B, Ld ld, St st) {
  const unsigned n = unsigned(B.count());
  const unsigned mw = magic_of(unsigned(B.ex)), my = magic_of(unsigned(B.ey));
  for (unsigned e0 = threadIdx.x; e0 < n; e0 += K * blockDim.x) {
    V v[K];
    int gx[K], gy[K], gz[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const unsigned e = e0 + unsigned(k) * blockDim.x;
      const unsigned r = div_m(e, unsigned(B.ex), mw);
      const unsigned lz = div_m(r, unsigned(B.ey), my);
      gx[k] = B.x0 + int(e - r * unsigned(B.ex));
      gy[k] = B.y0 + int(r - lz * unsigned(B.ey));
      gz[k] = B.z0 + int(lz);
      v[k] = ld(gx[k], gy[k], gz[k], e < n);
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const unsigned e = e0 + unsigned(k) * blockDim.x;
      if (e < n) st(int(e), gx[k], gy[k], gz[k], v[k]);
    }
  }
}

struct Cell3 {
  float a, b;
  uint8_t lb;
};
struct Cell4 {
  float a, b, c;
  uint8_t lb;
};

template <class T>
__device__ __forceinline__ float rnd(float v) { return tof(fromf<T>(v)); }

__device__ __forceinline__ bool inside(int x, int y, int z, int nx, int ny, int nz) {
  return x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz;
}

// Weighted neighbour sum of a staged box in the canonical fold order.
__device__ __forceinline__ float nb_sum(const float* z, int s, int sy, int sz, float wx, float wy, float wz) {
  return d4sum6(wx * z[s - 1], wx * z[s + 1], wy * z[s - sy], wy * z[s + sy], wz * z[s - sz], wz * z[s + sz]);
}

// Fine cells of coarse cells [c0, c0 + cn) along an axis of stride s (interior,
// i0/in) and with the restriction's one-cell halo (f0/fn).
__device__ __forceinline__ void down_axis(int s, int c0, int cn, int& i0, int& in, int& f0, int& fn) {
  if (s == 2) {
    i0 = 2 * c0;
    in = 2 * cn;
    f0 = i0 - 1;
    fn = in + 2;
  } else {
    i0 = f0 = c0;
    in = fn = cn;
  }
}

// Shared-memory bytes of the fused kernels for given tile shapes (host and device).
__host__ __device__ inline int down_smem_bytes(int cx, int cy, int cz, int sx, int sy, int sz) {
  const int fx = sx == 2 ? 2 * cx + 2 : cx, fy = sy == 2 ? 2 * cy + 2 : cy, fz = sz == 2 ? 2 * cz + 2 : cz;
  const int nh = (fx + 4) * (fy + 4) * (fz + 4);
  return ((nh * 13 + fx * fy * fz * 4) + 15) & ~15;
}
__host__ __device__ inline int up_coarse_extent(int t, int s) { return s == 2 ? (t + 4) / 2 + 3 : t + 4; }
__host__ __device__ inline int up_smem_bytes(int tx, int ty, int tz, int sx, int sy, int sz) {
  const int ne = (tx + 4) * (ty + 4) * (tz + 4);
  const int nc = up_coarse_extent(tx, sx) * up_coarse_extent(ty, sy) * up_coarse_extent(tz, sz);
  return ((ne * 13 + nc * 4) + 15) & ~15;
}

// ============================================================== down step
// Pre-smooth (one red-black sweep from z = 0), residual and restriction of
// level `level` into the right-hand side of level + 1, one coarse tile per CTA
// (mgSmoothColour mg.wgsl.ts:325-344, mgResidual :197-205, restriction = P^T/2^k
// of mgTrilinearPressure :217-241).  On level 0 the residual is scaled by sigma.
template <class TZ, class TR, class TD, class TS>
__global__ void __launch_bounds__(kFThreads, 2) k_down(const InstDev* insts, const Tile* tiles, int level) {
  extern __shared__ float sm[];
  const Tile tl = tiles[blockIdx.x];
  const InstDev& I = insts[tl.inst];
  const Ctrl* c = I.ctrl;
  if (c->done) return;
  const LevelDev& F = I.lv[level];
  const LevelDev& C = I.lv[level + 1];
  const float scale = level == 0 ? float(c->sigma) : 1.0f;
  const int CX = F.dcx, CY = F.dcy, CZ = F.dcz;
  const int ntx = (C.nx + CX - 1) / CX, nty = (C.ny + CY - 1) / CY;
  const int tx = tl.tile % ntx, tr = tl.tile / ntx, ty = tr % nty, tz = tr / nty;
  const int cx0 = tx * CX, cy0 = ty * CY, cz0 = tz * CZ;
  int ix0, iex, iy0, iey, iz0, iez, fx0, fex, fy0, fey, fz0, fez;
  down_axis(C.sx, cx0, CX, ix0, iex, fx0, fex);
  down_axis(C.sy, cy0, CY, iy0, iey, fy0, fey);
  down_axis(C.sz, cz0, CZ, iz0, iez, fz0, fez);
  const SBox H{fx0 - 2, fy0 - 2, fz0 - 2, fex + 4, fey + 4, fez + 4};
  const int nH = H.count();
  float* rhs_s = sm;
  float* dg_s = rhs_s + nH;
  float* z_s = dg_s + nH;
  float* res_s = z_s + nH;   // F box
  uint8_t* lab_s = reinterpret_cast<uint8_t*>(res_s + fex * fey * fez);
  const int nx = F.nx, ny = F.ny, nz = F.nz;
  const TR* __restrict__ rhs = static_cast<const TR*>(F.rhs);
  const TD* __restrict__ dg = static_cast<const TD*>(F.diagT);
  const uint8_t* __restrict__ lab = F.label;
  // stage H; red cells start the sweep at rhs / diag, black cells at zero
  stage_box<4, Cell3>(
      H,
      [&](int x, int y, int z, bool ok) {
        Cell3 v{0.0f, 1.0f, 0};
        if (ok && inside(x, y, z, nx, ny, nz)) {
          const int i = x + nx * (y + ny * z);
          v.lb = lab[i];
          v.a = tof(rhs[i]);
          v.b = tof(dg[i]);
        }
        return v;
      },
      [&](int s, int x, int y, int z, const Cell3& v) {
        rhs_s[s] = v.a;
        dg_s[s] = v.b;
        lab_s[s] = v.lb;
        z_s[s] = (v.lb && ((x + y + z) & 1) == 0) ? rnd<TZ>(v.a * __frcp_rn(v.b)) : 0.0f;
      });
  __syncthreads();
  const float wx = F.wx, wy = F.wy, wz = F.wz;
  const int sy = H.ex, sz = H.ex * H.ey;
  // black cells of G = F +- 1 (their neighbours are red)
  for_box(H, fx0 - 1, fy0 - 1, fz0 - 1, fex + 2, fey + 2, fez + 2, 1, [&](int, int, int, int s) {
    if (!lab_s[s]) return;
    z_s[s] = rnd<TZ>((rhs_s[s] + nb_sum(z_s, s, sy, sz, wx, wy, wz)) * __frcp_rn(dg_s[s]));
  });
  __syncthreads();
  // residual on F; the interior's pre-smoothed z goes to the level's scratch
  // array (the up step reads it there and writes the final z to F.z, so its
  // halo reads never see a neighbour tile's output)
  TZ* __restrict__ zo = static_cast<TZ*>(F.res);
  for_box(H, fx0, fy0, fz0, fex, fey, fez, 2, [&](int x, int y, int z, int s) {
    float r = 0.0f;
    if (lab_s[s]) r = scale * (rhs_s[s] - (dg_s[s] * z_s[s] - nb_sum(z_s, s, sy, sz, wx, wy, wz)));
    res_s[(x - fx0) + fex * ((y - fy0) + fey * (z - fz0))] = r;
    if (x >= ix0 && y >= iy0 && z >= iz0 && x < ix0 + iex && y < iy0 + iey && z < iz0 + iez &&
        inside(x, y, z, nx, ny, nz))
      zo[x + nx * (y + ny * z)] = fromf<TZ>(z_s[s]);
  });
  __syncthreads();
  // separable restriction: x pass (F z, F y, coarse x) then y pass (F z, coarse y, coarse x)
  float* xs = z_s;                       // z_s is free from here on
  float* ys = z_s + fez * fey * CX;
  {
    const int n = fez * fey * CX;
    const unsigned m1 = magic_of(CX), m2 = magic_of(fey);
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      const unsigned r = div_m(e, CX, m1), lz = div_m(r, fey, m2);
      const int cx = e - int(r) * CX, ly = int(r) - int(lz) * fey;
      xs[e] = rline(C.sx, cx0 + cx, C.nx, nx, fx0, &res_s[(int(lz) * fey + ly) * fex], 1);
    }
  }
  __syncthreads();
  {
    const int n = fez * CY * CX;
    const unsigned m1 = magic_of(CX), m2 = magic_of(CY);
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      const unsigned r = div_m(e, CX, m1), lz = div_m(r, CY, m2);
      const int cx = e - int(r) * CX, cy = int(r) - int(lz) * CY;
      ys[e] = rline(C.sy, cy0 + cy, C.ny, ny, fy0, &xs[int(lz) * fey * CX + cx], CX);
    }
  }
  __syncthreads();
  // z pass and store
  {
    const float out_scale = F.to_coarse / float((C.sx == 2 ? 2 : 1) * (C.sy == 2 ? 2 : 1) * (C.sz == 2 ? 2 : 1));
    TS* __restrict__ out = static_cast<TS*>(C.rhs);
    const int n = CZ * CY * CX;
    const unsigned m1 = magic_of(CX), m2 = magic_of(CY);
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      const unsigned r = div_m(e, CX, m1), cz = div_m(r, CY, m2);
      const int cx = e - int(r) * CX, cy = int(r) - int(cz) * CY;
      const int X = cx0 + cx, Y = cy0 + cy, Z = cz0 + int(cz);
      if (X >= C.nx || Y >= C.ny || Z >= C.nz) continue;
      const int ci = X + C.nx * (Y + C.ny * Z);
      float acc = 0.0f;
      if (C.label[ci]) acc = out_scale * rline(C.sz, Z, C.nz, nz, fz0, &ys[cy * CX + cx], CY * CX);
      out[ci] = fromf<TS>(acc);
    }
  }
}

// ================================================================ up step
// z_l += P z_{l+1} (mgProlongateAdd, mg.wgsl.ts:243-246; from level 1 into
// level 0 the sigma scaling is undone), then one sweep black then red, one fine
// tile per CTA, for levels whose next coarser level does not halve every axis
// (gamma is then folded by k_dot_rz_part over the fixed level-0 tiles).
template <class TZF, class TR, class TD, class TZC>
__global__ void __launch_bounds__(kFThreads, 2) k_up(const InstDev* insts, const Tile* tiles, int level) {
  extern __shared__ float sm[];
  const Tile tl = tiles[blockIdx.x];
  const InstDev& I = insts[tl.inst];
  Ctrl* c = I.ctrl;
  if (c->done) return;
  const LevelDev& F = I.lv[level];
  const LevelDev& C = I.lv[level + 1];
  const float unscale = level == 0 ? float(1.0 / c->sigma) : 1.0f;
  const int TX = F.utx, TY = F.uty, TZ = F.utz;
  const int nx = F.nx, ny = F.ny, nz = F.nz;
  const int ntx = (nx + TX - 1) / TX, nty = (ny + TY - 1) / TY;
  const int tx = tl.tile % ntx, tr = tl.tile / ntx, ty = tr % nty, tz = tr / nty;
  const int x0 = tx * TX, y0 = ty * TY, z0 = tz * TZ;
  const SBox E{x0 - 2, y0 - 2, z0 - 2, TX + 4, TY + 4, TZ + 4};
  // coarse cells under the in-lattice part of E
  auto cspan = [](int e0, int en, int nf, int s, int nc, int& c0, int& cn) {
    const int lo = max(e0, 0), hi = min(e0 + en - 1, nf - 1);
    if (s == 2) {
      c0 = max(lo / 2 - 1, 0);
      cn = min(hi / 2 + 1, nc - 1) - c0 + 1;
    } else {
      c0 = lo;
      cn = hi - lo + 1;
    }
  };
  int qx0, qex, qy0, qey, qz0, qez;
  cspan(E.x0, E.ex, nx, C.sx, C.nx, qx0, qex);
  cspan(E.y0, E.ey, ny, C.sy, C.ny, qy0, qey);
  cspan(E.z0, E.ez, nz, C.sz, C.nz, qz0, qez);
  const SBox Q{qx0, qy0, qz0, qex, qey, qez};
  const int nE = E.count();
  float* z_s = sm;
  float* rhs_s = z_s + nE;
  float* dg_s = rhs_s + nE;
  float* zc_s = dg_s + nE;
  uint8_t* lab_s = reinterpret_cast<uint8_t*>(zc_s + Q.count());
  const TZF* __restrict__ zf = static_cast<const TZF*>(F.res);   // pre-smoothed z from the down step
  const TR* __restrict__ rhs = static_cast<const TR*>(F.rhs);
  const TD* __restrict__ dg = static_cast<const TD*>(F.diagT);
  const uint8_t* __restrict__ lab = F.label;
  const TZC* __restrict__ zc = static_cast<const TZC*>(C.z);
  stage_box<4, float>(
      Q, [&](int x, int y, int z, bool ok) { return ok ? tof(zc[x + C.nx * (y + C.ny * z)]) : 0.0f; },
      [&](int s, int, int, int, float v) { zc_s[s] = v; });
  stage_box<4, Cell4>(
      E,
      [&](int x, int y, int z, bool ok) {
        Cell4 v{0.0f, 0.0f, 1.0f, 0};
        if (ok && inside(x, y, z, nx, ny, nz)) {
          const int i = x + nx * (y + ny * z);
          v.lb = lab[i];
          v.a = tof(zf[i]);
          v.b = tof(rhs[i]);
          v.c = tof(dg[i]);
        }
        return v;
      },
      [&](int s, int, int, int, const Cell4& v) {
        z_s[s] = v.a;
        rhs_s[s] = v.b;
        dg_s[s] = v.c;
        lab_s[s] = v.lb;
      });
  __syncthreads();
  // prolongation on E (liquid cells)
  for_box(E, E.x0, E.y0, E.z0, E.ex, E.ey, E.ez, 2, [&](int x, int y, int z, int s) {
    if (!lab_s[s]) return;
    int cx[2], cy[2], cz[2];
    float wxx[2], wyy[2], wzz[2];
    taps2(x, C.sx, C.nx, cx, wxx);
    taps2(y, C.sy, C.ny, cy, wyy);
    taps2(z, C.sz, C.nz, cz, wzz);
    float acc = 0.0f;
#pragma unroll
    for (int c2 = 0; c2 < 2; ++c2)
#pragma unroll
      for (int c1 = 0; c1 < 2; ++c1) {
        const int row = Q.at(0, cy[c1], cz[c2]);
#pragma unroll
        for (int c0 = 0; c0 < 2; ++c0) acc += wxx[c0] * wyy[c1] * wzz[c2] * zc_s[row + cx[c0]];
      }
    z_s[s] = rnd<TZF>(z_s[s] + acc * unscale);
  });
  __syncthreads();
  const float wx = F.wx, wy = F.wy, wz = F.wz;
  const int sy = E.ex, sz = E.ex * E.ey;
  for_box(E, x0 - 1, y0 - 1, z0 - 1, TX + 2, TY + 2, TZ + 2, 1, [&](int, int, int, int s) {
    if (!lab_s[s]) return;
    z_s[s] = rnd<TZF>((rhs_s[s] + nb_sum(z_s, s, sy, sz, wx, wy, wz)) * __frcp_rn(dg_s[s]));
  });
  __syncthreads();
  for_box(E, x0, y0, z0, TX, TY, TZ, 0, [&](int, int, int, int s) {
    if (!lab_s[s]) return;
    z_s[s] = rnd<TZF>((rhs_s[s] + nb_sum(z_s, s, sy, sz, wx, wy, wz)) * __frcp_rn(dg_s[s]));
  });
  __syncthreads();
  TZF* __restrict__ zo = static_cast<TZF*>(F.z);
  for_box(E, x0, y0, z0, TX, TY, TZ, 2, [&](int x, int y, int z, int s) {
    if (!inside(x, y, z, nx, ny, nz)) return;
    zo[x + nx * (y + ny * z)] = fromf<TZF>(z_s[s]);
  });
}

}  // namespace fpp
