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

// ====================================================== marching down step
// The same down step for a level that coarsens by two on every axis, as a
// 2.5-D march: a CTA owns a coarse tile of kMX x kMY x kMZ cells and streams
// the fine planes under it once, bottom to top.  Rings of planes in shared
// memory hold what the stencils still need: rhs / diag / label of 3 planes,
// z of 4, and the x-then-y restricted residual of 4.  Step p stages fine plane
// p (loads prefetched into registers during step p - 1) with its red cells
// set pointwise, sweeps the black cells of plane p - 1, forms the residual of
// plane p - 2 (storing its interior z to the level's scratch array) and
// restricts it in x and y; coarse plane Z is finished by the z pass once fine
// plane 2Z + 2 is restricted.  Every cell gets the box kernel's arithmetic in
// the same order, so both give the same bits; only the halo's shape differs:
// (2 kMX + 6)(2 kMY + 6) staged cells per 4 kMX kMY interior ones in a plane,
// and 6 extra planes per 2 kMZ.
constexpr int kMarchLevels = 2;                       // grid levels 0 .. kMarchLevels - 1 may march
constexpr int kMX = 16, kMY = 8, kMZ = 8;             // coarse cells per tile
constexpr int kMThreads = 256;
constexpr int kMHX = 2 * kMX + 6, kMHY = 2 * kMY + 6;   // staged plane (F +- 2)
constexpr int kMHP = kMHX * kMHY;
constexpr int kMFX = 2 * kMX + 2, kMFY = 2 * kMY + 2;   // residual plane (interior + restriction taps)
constexpr int kMPer = (kMHP + kMThreads - 1) / kMThreads;

__host__ __device__ inline int march_down_tiles(int cnx, int cny, int cnz) {
  return ((cnx + kMX - 1) / kMX) * ((cny + kMY - 1) / kMY) * ((cnz + kMZ - 1) / kMZ);
}

template <class TZ, class TR, class TD, class TS>
__global__ void __launch_bounds__(kMThreads, 4) k_down_m(const InstDev* insts, const Tile* tiles, int level) {
  __shared__ float rhs_r[3][kMHP];
  __shared__ float dg_r[3][kMHP];
  __shared__ uint8_t lab_r[3][kMHP];
  __shared__ float z_r[4][kMHP];
  __shared__ float res_p[kMFX * kMFY];
  __shared__ float ys_r[4][kMY * kMX];
  const Tile tl = tiles[blockIdx.x];
  const InstDev& I = insts[tl.inst];
  const Ctrl* c = I.ctrl;
  if (c->done) return;
  const LevelDev& F = I.lv[level];
  const LevelDev& C = I.lv[level + 1];
  const float scale = level == 0 ? float(c->sigma) : 1.0f;
  const int nx = F.nx, ny = F.ny, nz = F.nz, nxy = nx * ny;
  const int ntx = (C.nx + kMX - 1) / kMX, nty = (C.ny + kMY - 1) / kMY;
  const int tx = tl.tile % ntx, tr = tl.tile / ntx, ty = tr % nty, tz = tr / nty;
  const int cx0 = tx * kMX, cy0 = ty * kMY, cz0 = tz * kMZ;
  const int hx0 = 2 * cx0 - 3, hy0 = 2 * cy0 - 3;   // staged plane origin
  const int fx0 = 2 * cx0 - 1, fy0 = 2 * cy0 - 1;   // residual plane origin
  // the march ends at the last coarse plane of the lattice: planes above it are air
  const int pz0 = 2 * cz0 - 3, pz1 = 2 * min(cz0 + kMZ, C.nz) + 2;
  const TR* __restrict__ rhs = static_cast<const TR*>(F.rhs);
  const TD* __restrict__ dg = static_cast<const TD*>(F.diagT);
  const uint8_t* __restrict__ lab = F.label;
  TZ* __restrict__ zo = static_cast<TZ*>(F.res);
  TS* __restrict__ out = static_cast<TS*>(C.rhs);
  const float wx = F.wx, wy = F.wy, wz = F.wz;
  const float out_scale = F.to_coarse / 8.0f;
  const int t = threadIdx.x;
  // The thread's cells keep their (x, y) in every plane: their in-plane offsets,
  // global column offsets, lattice masks and colour parities are set once.
  int aoff[kMPer];      // staged cells: global column offset, -1 outside the lattice or the plane
  unsigned apar = 0;    // bit k: (x + y) of staged cell k is odd
#pragma unroll
  for (int k = 0; k < kMPer; ++k) {
    const int e = t + k * kMThreads;
    const int gx = hx0 + e % kMHX, gy = hy0 + e / kMHX;
    aoff[k] = (e < kMHP && gx >= 0 && gy >= 0 && gx < nx && gy < ny) ? gx + nx * gy : -1;
    apar |= unsigned((gx + gy) & 1) << k;
  }
  constexpr int kW = (kMHX - 2) / 2;                  // black cells per row of G
  constexpr int kBPer = (kW * (kMHY - 2) + kMThreads - 1) / kMThreads;
  int bs[kBPer];        // black cells: in-plane index at even offset; parity term of the row
  unsigned bpar = 0;
#pragma unroll
  for (int k = 0; k < kBPer; ++k) {
    const int e = t + k * kMThreads;
    const int ey = 1 + e / kW;
    bs[k] = e < kW * (kMHY - 2) ? ey * kMHX + 1 + 2 * (e % kW) : -1;
    bpar |= unsigned((hx0 + 1 + hy0 + ey) & 1) << k;
  }
  constexpr int kRPer = (kMFX * kMFY + kMThreads - 1) / kMThreads;
  int rofs[kRPer];      // residual cells: global column offset of interior cells, -1 else
#pragma unroll
  for (int k = 0; k < kRPer; ++k) {
    const int e = t + k * kMThreads;
    const int lx = e % kMFX, ly = e / kMFX, gx = fx0 + lx, gy = fy0 + ly;
    rofs[k] = (e < kMFX * kMFY && lx >= 1 && lx <= 2 * kMX && ly >= 1 && ly <= 2 * kMY && gx < nx && gy < ny)
                  ? gx + nx * gy
                  : -1;
  }
  // restriction: this thread's coarse (x, y) and its 4 x 4 fine taps (weight 0
  // on taps outside the lattice, whose residual is 0: the fold keeps rline's
  // order and bits)
  const int rcx = t % kMX, rcy = t / kMX, RX = cx0 + rcx, RY = cy0 + rcy;
  const bool rown = t < kMX * kMY && RX < C.nx && RY < C.ny;
  float wxr[4], wyr[4];
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    const int fx = 2 * RX + d - 1, fy = 2 * RY + d - 1;
    wxr[d] = (fx >= 0 && fx < nx) ? p1d(fx, RX, C.nx) : 0.0f;
    wyr[d] = (fy >= 0 && fy < ny) ? p1d(fy, RY, C.ny) : 0.0f;
  }
  const int rbase = (2 * rcy) * kMFX + 2 * rcx;   // res_p index of tap (d = -1, d = -1)
  float pr[kMPer], pd[kMPer];
  uint8_t pl[kMPer];
  auto fetch = [&](int p) {
    const bool pin = p >= 0 && p < nz;
#pragma unroll
    for (int k = 0; k < kMPer; ++k) {
      pr[k] = 0.0f;
      pd[k] = 1.0f;
      pl[k] = 0;
      if (pin && aoff[k] >= 0) {
        const int i = aoff[k] + nxy * p;
        pl[k] = lab[i];
        pr[k] = tof(rhs[i]);
        pd[k] = tof(dg[i]);
      }
    }
  };
  auto slot3 = [&](int p) { return (p - pz0) % 3; };
  auto slot4 = [&](int p) { return (p - pz0) & 3; };
  // z pass of coarse plane Z = (r - 2) / 2, whose last fine plane r is restricted
  auto zpass = [&](int r) {
    if (!rown || r < 2 * cz0 + 2 || ((r - 2) & 1)) return;
    const int Z = (r - 2) >> 1;
    if (Z >= cz0 + kMZ || Z >= C.nz) return;
    const int ci = RX + C.nx * (RY + C.ny * Z);
    float acc = 0.0f;
    if (C.label[ci]) {
      float sum = 0.0f;
#pragma unroll
      for (int d = -1; d <= 2; ++d) {
        const int f = 2 * Z + d;
        if (f >= 0 && f < nz) sum += p1d(f, Z, C.nz) * ys_r[slot4(f)][t];
      }
      acc = out_scale * sum;
    }
    out[ci] = fromf<TS>(acc);
  };
  fetch(pz0);
  for (int p = pz0; p <= pz1; ++p) {
    const int k = p - pz0;
    // stage plane p: red cells start the sweep at rhs / diag, black cells at zero
    {
      const int sa = slot3(p), za = slot4(p);
      const unsigned red = (p & 1) ? apar : ~apar;   // bit k: cell k is red in plane p
#pragma unroll
      for (int kk = 0; kk < kMPer; ++kk) {
        const int e = t + kk * kMThreads;
        if (e >= kMHP) continue;
        rhs_r[sa][e] = pr[kk];
        dg_r[sa][e] = pd[kk];
        lab_r[sa][e] = pl[kk];
        z_r[za][e] = (pl[kk] && ((red >> kk) & 1u)) ? rnd<TZ>(pr[kk] * __frcp_rn(pd[kk])) : 0.0f;
      }
    }
    if (p < pz1) fetch(p + 1);
    zpass(p - 3);   // the previous step restricted fine plane p - 3
    __syncthreads();
    // black cells of plane q = p - 1 inside G = F +- 1 (their neighbours are red)
    if (k >= 2) {
      const int q = p - 1, sq = slot3(q), zq = slot4(q), zm = slot4(q - 1), zp = slot4(p);
      const float* zc = z_r[zq];
#pragma unroll
      for (int kk = 0; kk < kBPer; ++kk) {
        if (bs[kk] < 0) continue;
        const int s = bs[kk] + int((((bpar >> kk) ^ unsigned(q)) & 1u) ^ 1u);
        if (!lab_r[sq][s]) continue;
        const float nb = d4sum6(wx * zc[s - 1], wx * zc[s + 1], wy * zc[s - kMHX], wy * zc[s + kMHX],
                                wz * z_r[zm][s], wz * z_r[zp][s]);
        z_r[zq][s] = rnd<TZ>((rhs_r[sq][s] + nb) * __frcp_rn(dg_r[sq][s]));
      }
    }
    __syncthreads();
    // residual of plane r = p - 2 on F; its interior z goes to the scratch array
    const int r = p - 2;
    if (k >= 4) {
      const int sr = slot3(r), zr = slot4(r), zm = slot4(r - 1), zp = slot4(r + 1);
      const bool zin = r >= 2 * cz0 && r < 2 * (cz0 + kMZ) && r < nz;
      const float* zc = z_r[zr];
#pragma unroll
      for (int kk = 0; kk < kRPer; ++kk) {
        const int e = t + kk * kMThreads;
        if (e >= kMFX * kMFY) continue;
        const int s = (e / kMFX + 2) * kMHX + e % kMFX + 2;
        float rv = 0.0f;
        if (lab_r[sr][s])
          rv = scale * (rhs_r[sr][s] - (dg_r[sr][s] * zc[s] -
                                         d4sum6(wx * zc[s - 1], wx * zc[s + 1], wy * zc[s - kMHX], wy * zc[s + kMHX],
                                                wz * z_r[zm][s], wz * z_r[zp][s])));
        res_p[e] = rv;
        if (zin && rofs[kk] >= 0) zo[rofs[kk] + nxy * r] = fromf<TZ>(zc[s]);
      }
    }
    __syncthreads();
    // x then y restriction of the plane into the ring, one coarse (x, y) per thread
    if (k >= 4 && t < kMX * kMY) {
      float sy = 0.0f;
#pragma unroll
      for (int dy = 0; dy < 4; ++dy) {
        const float* row = &res_p[rbase + dy * kMFX];
        float sx = 0.0f;
#pragma unroll
        for (int dx = 0; dx < 4; ++dx) sx += wxr[dx] * row[dx];
        sy += wyr[dy] * sx;
      }
      ys_r[slot4(r)][t] = sy;
    }
    __syncthreads();
  }
  zpass(pz1 - 2);
}

// ================================================================ up step
// z_l += P z_{l+1} (mgProlongateAdd, mg.wgsl.ts:243-246; from level 1 into
// level 0 the sigma scaling is undone), then one sweep black then red, one fine
// tile per CTA.  (gamma is folded by k_dot_rz_part over the fixed level-0
// tiles, or by the level-0 marching up step.)
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

// ======================================================== marching up step
// The up step of a level coarsened by two on every axis as a 2.5-D march (see
// k_down_m): a CTA owns kUX x kUY x kUZ fine cells and streams the
// planes under them once.  Step p stages fine plane p of the halo box E = T +- 2
// with the prolongated coarse correction added (each thread keeps its cells'
// x / y taps for the whole march; coarse planes arrive in a ring of 3),
// sweeps the black cells of plane p - 2 on T +- 1, then the red cells of plane
// p - 4 on T, writing that plane's z (the two-plane lags let one barrier per
// step separate the phases).  Each cell gets k_up's arithmetic in the same
// order.
constexpr int kUX = 32, kUY = 16, kUZ = 16;            // fine cells per tile
constexpr int kUEX = kUX + 4, kUEY = kUY + 4, kUEP = kUEX * kUEY;
constexpr int kUQX = (kUX + 4) / 2 + 3, kUQY = (kUY + 4) / 2 + 3, kUQP = kUQX * kUQY;   // coarse plane box
constexpr int kUPer = (kUEP + kMThreads - 1) / kMThreads;

__host__ __device__ inline int march_up_tiles(int nx, int ny, int nz) {
  return ((nx + kUX - 1) / kUX) * ((ny + kUY - 1) / kUY) * ((nz + kUZ - 1) / kUZ);
}

// Rings of the marching up step (one barrier per step, as in k_down_m).
constexpr int kURing = 5, kUZRing = 6;
__host__ __device__ inline int march_up_smem_bytes() {
  return (2 * kURing * kUEP + kUZRing * kUEP + 3 * kUQP) * 4 + kURing * kUEP;
}

// With DOT (level 0) the step also writes the gamma partials of the fixed
// 32 x 8 x 8 level-0 tiles it covers.  Thread t outputs rows t / 32 and
// 8 + t / 32 of column t % 32 of the tile, in z order: lane and warp of
// k_dot_rz_part's layout, so its per-thread sums and block folds, and hence
// gamma's bits, are that kernel's.
static_assert(kUX == kTX && kUY == 2 * kTY && kUZ % kMaxDepth == 0 && kUX * kUY == 2 * kMThreads,
              "marching up tiles must cover whole dot tiles, two rows per thread");
template <class TZF, class TR, class TD, class TZC, bool DOT = false>
__global__ void __launch_bounds__(kMThreads, 3) k_up_m(const InstDev* insts, const Tile* tiles, int level) {
  extern __shared__ float smu[];
  __shared__ double gsh[DOT ? 6 * 32 : 1];
  float* rhs_r = smu;                              // [kURing][kUEP]
  float* dg_r = rhs_r + kURing * kUEP;             // [kURing][kUEP]
  float* z_r = dg_r + kURing * kUEP;               // [kUZRing][kUEP]
  float* zc_r = z_r + kUZRing * kUEP;              // [3][kUQP]
  uint8_t* lab_r = reinterpret_cast<uint8_t*>(zc_r + 3 * kUQP);   // [kURing][kUEP]
  const Tile tl = tiles[blockIdx.x];
  const InstDev& I = insts[tl.inst];
  const Ctrl* c = I.ctrl;
  if (c->done) return;
  const LevelDev& F = I.lv[level];
  const LevelDev& C = I.lv[level + 1];
  const float unscale = level == 0 ? float(1.0 / c->sigma) : 1.0f;
  const int nx = F.nx, ny = F.ny, nz = F.nz, nxy = nx * ny;
  const int ntx = (nx + kUX - 1) / kUX, nty = (ny + kUY - 1) / kUY;
  const int tx = tl.tile % ntx, tr = tl.tile / ntx, ty = tr % nty, tz = tr / nty;
  const int x0 = tx * kUX, y0 = ty * kUY, z0 = tz * kUZ;
  const int ex0 = x0 - 2, ey0 = y0 - 2;            // staged plane origin
  const int pz0 = z0 - 2, pz1 = min(z0 + kUZ, nz) + 1;   // fine planes streamed (none above the lattice)
  // coarse columns under the in-lattice part of the staged plane (k_up's cspan)
  auto cspan = [](int e0, int en, int nf, int nc, int& c0, int& cn) {
    const int lo = max(e0, 0), hi = min(e0 + en - 1, nf - 1);
    c0 = max(lo / 2 - 1, 0);
    cn = min(hi / 2 + 1, nc - 1) - c0 + 1;
  };
  int qx0, qex, qy0, qey;
  cspan(ex0, kUEX, nx, C.nx, qx0, qex);
  cspan(ey0, kUEY, ny, C.ny, qy0, qey);
  const TZF* __restrict__ zf = static_cast<const TZF*>(F.res);
  const TR* __restrict__ rhs = static_cast<const TR*>(F.rhs);
  const TD* __restrict__ dg = static_cast<const TD*>(F.diagT);
  const uint8_t* __restrict__ lab = F.label;
  const TZC* __restrict__ zc = static_cast<const TZC*>(C.z);
  TZF* __restrict__ zo = static_cast<TZF*>(F.z);
  const float wx = F.wx, wy = F.wy, wz = F.wz;
  const int t = threadIdx.x;
  // The thread's staged cells keep their (x, y) in every plane: column offset
  // (-1 outside the lattice), the coarse-plane offset of tap (c1, c0) = (0, 0)
  // with the steps to taps 1 along x and y (0 where a wall dropped the tap),
  // and the x / y tap weights.
  int aoff[kUPer], qb[kUPer];
  unsigned qstep = 0;   // bits 2k, 2k + 1: x and y step of cell k
  float wxx[kUPer][2], wyy[kUPer][2];
#pragma unroll
  for (int k = 0; k < kUPer; ++k) {
    const int e = t + k * kMThreads;
    const int gx = ex0 + e % kUEX, gy = ey0 + e / kUEX;
    aoff[k] = (e < kUEP && gx >= 0 && gy >= 0 && gx < nx && gy < ny) ? gx + nx * gy : -1;
    int cx[2], cy[2];
    taps2(gx, 2, C.nx, cx, wxx[k]);
    taps2(gy, 2, C.ny, cy, wyy[k]);
    qb[k] = (cx[0] - qx0) + qex * (cy[0] - qy0);
    qstep |= (unsigned(cx[1] - cx[0] == 1) << (2 * k)) | (unsigned(cy[1] - cy[0] == 1) << (2 * k + 1));
  }
  constexpr int kW = (kUEX - 2) / 2;                  // black cells per row of T +- 1
  constexpr int kBPer = (kW * (kUEY - 2) + kMThreads - 1) / kMThreads;
  int bs[kBPer];
  unsigned bpar = 0;
#pragma unroll
  for (int k = 0; k < kBPer; ++k) {
    const int e = t + k * kMThreads;
    const int ey = 1 + e / kW;
    bs[k] = e < kW * (kUEY - 2) ? ey * kUEX + 1 + 2 * (e % kW) : -1;
    bpar |= unsigned((ex0 + 1 + ey0 + ey) & 1) << k;
  }
  constexpr int kTPer = (kUX * kUY + kMThreads - 1) / kMThreads;
  int ts_[kTPer], tofs[kTPer];   // interior cells: in-plane index, column offset (-1 outside the lattice)
  unsigned tpar = 0;
#pragma unroll
  for (int k = 0; k < kTPer; ++k) {
    const int e = t + k * kMThreads;
    const int lx = e % kUX, ly = e / kUX, gx = x0 + lx, gy = y0 + ly;
    ts_[k] = (ly + 2) * kUEX + lx + 2;
    tofs[k] = (e < kUX * kUY && gx < nx && gy < ny) ? gx + nx * gy : -1;
    tpar |= unsigned((gx + gy) & 1) << k;
  }
  // coarse planes: Z goes to slot Z % 3
  auto load_coarse = [&](int Z) {
    float* d = zc_r + (Z % 3) * kUQP;
    for (int e = t; e < qex * qey; e += kMThreads) {
      const int cxl = e % qex, cyl = e / qex;
      d[cxl + qex * cyl] = tof(zc[(qx0 + cxl) + C.nx * ((qy0 + cyl) + C.ny * Z)]);
    }
  };
  auto coarse_hi = [&](int p) {   // the highest coarse plane fine plane p reads
    int cz[2];
    float w[2];
    taps2(min(max(p, 0), nz - 1), 2, C.nz, cz, w);
    return max(cz[0], cz[1]);
  };
  float pz_[kUPer], pr[kUPer], pd[kUPer];
  uint8_t pl[kUPer];
  auto fetch = [&](int p) {
    const bool pin = p >= 0 && p < nz;
#pragma unroll
    for (int k = 0; k < kUPer; ++k) {
      pz_[k] = 0.0f;
      pr[k] = 0.0f;
      pd[k] = 1.0f;
      pl[k] = 0;
      if (pin && aoff[k] >= 0) {
        const int i = aoff[k] + nxy * p;
        pl[k] = lab[i];
        pz_[k] = tof(zf[i]);
        pr[k] = tof(rhs[i]);
        pd[k] = tof(dg[i]);
      }
    }
  };
  auto sl = [&](int p, int n) { return (p - pz0) % n; };
  int zhi_loaded;
  {
    int cz[2];
    float w[2];
    taps2(min(max(pz0, 0), nz - 1), 2, C.nz, cz, w);
    zhi_loaded = coarse_hi(pz0);
    for (int Z = min(cz[0], cz[1]); Z <= zhi_loaded; ++Z) load_coarse(Z);
  }
  double gacc[2][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};   // per output row: r.z, sum z, sum r
  fetch(pz0);
  __syncthreads();
  for (int p = pz0; p <= pz1 + 2; ++p) {
    // stage plane p with the prolongated correction on liquid cells
    if (p <= pz1) {
      float* rh = rhs_r + sl(p, kURing) * kUEP;
      float* dd = dg_r + sl(p, kURing) * kUEP;
      uint8_t* lb = lab_r + sl(p, kURing) * kUEP;
      float* zz = z_r + sl(p, kUZRing) * kUEP;
      int czs[2];
      float wzz[2];
      taps2(p, 2, C.nz, czs, wzz);
#pragma unroll
      for (int kk = 0; kk < kUPer; ++kk) {
        const int e = t + kk * kMThreads;
        if (e >= kUEP) continue;
        rh[e] = pr[kk];
        dd[e] = pd[kk];
        lb[e] = pl[kk];
        float zv = pz_[kk];
        if (pl[kk]) {
          const int sx = int((qstep >> (2 * kk)) & 1u), sy = int((qstep >> (2 * kk + 1)) & 1u) * qex;
          float acc = 0.0f;
#pragma unroll
          for (int c2 = 0; c2 < 2; ++c2) {
            const float* q = zc_r + (czs[c2] % 3) * kUQP + qb[kk];
#pragma unroll
            for (int c1 = 0; c1 < 2; ++c1)
#pragma unroll
              for (int c0 = 0; c0 < 2; ++c0)
                acc += wxx[kk][c0] * wyy[kk][c1] * wzz[c2] * q[c1 * sy + c0 * sx];
          }
          zv = rnd<TZF>(zv + acc * unscale);
        }
        zz[e] = zv;
      }
      if (p < pz1) {
        fetch(p + 1);
        // the next plane's coarse planes: a new plane evicts one that neither
        // this plane nor the next reads
        const int need = coarse_hi(p + 1);
        for (int Z = zhi_loaded + 1; Z <= need; ++Z) load_coarse(Z);
        zhi_loaded = max(zhi_loaded, need);
      }
    }
    // black cells of plane q = p - 2 on T +- 1
    const int q = p - 2;
    if (q >= pz0 + 1 && q <= pz1 - 1) {
      const float* rh = rhs_r + sl(q, kURing) * kUEP;
      const float* dd = dg_r + sl(q, kURing) * kUEP;
      const uint8_t* lb = lab_r + sl(q, kURing) * kUEP;
      float* zq_ = z_r + sl(q, kUZRing) * kUEP;
      const float* zm = z_r + sl(q - 1, kUZRing) * kUEP;
      const float* zp = z_r + sl(q + 1, kUZRing) * kUEP;
#pragma unroll
      for (int kk = 0; kk < kBPer; ++kk) {
        if (bs[kk] < 0) continue;
        const int s = bs[kk] + int((((bpar >> kk) ^ unsigned(q)) & 1u) ^ 1u);
        if (!lb[s]) continue;
        const float nb = d4sum6(wx * zq_[s - 1], wx * zq_[s + 1], wy * zq_[s - kUEX], wy * zq_[s + kUEX],
                                wz * zm[s], wz * zp[s]);
        zq_[s] = rnd<TZF>((rh[s] + nb) * __frcp_rn(dd[s]));
      }
    }
    // red cells of plane r = p - 4 on T, then the plane's output
    const int r = p - 4;
    if (r >= pz0 + 2 && r <= pz1 - 2) {
      const float* rh = rhs_r + sl(r, kURing) * kUEP;
      const float* dd = dg_r + sl(r, kURing) * kUEP;
      const uint8_t* lb = lab_r + sl(r, kURing) * kUEP;
      const float* zr_ = z_r + sl(r, kUZRing) * kUEP;
      const float* zm = z_r + sl(r - 1, kUZRing) * kUEP;
      const float* zp = z_r + sl(r + 1, kUZRing) * kUEP;
      const unsigned red = (r & 1) ? tpar : ~tpar;
      const bool rin = r < nz;
#pragma unroll
      for (int kk = 0; kk < kTPer; ++kk) {
        const int s = ts_[kk];
        float zv = zr_[s];
        if (lb[s] && ((red >> kk) & 1u))
          zv = rnd<TZF>((rh[s] + d4sum6(wx * zr_[s - 1], wx * zr_[s + 1], wy * zr_[s - kUEX], wy * zr_[s + kUEX],
                                        wz * zm[s], wz * zp[s])) *
                        __frcp_rn(dd[s]));
        if (rin && tofs[kk] >= 0) zo[tofs[kk] + nxy * r] = fromf<TZF>(zv);
        if (DOT && lb[s]) {   // liquid cells of the lattice (staged labels are 0 outside it)
          const double zd = zv, rd = rh[s];
          gacc[kk][0] += rd * zd;
          gacc[kk][1] += zd;
          gacc[kk][2] += rd;
        }
      }
      // a dot tile ends every 8 planes and at the lattice top
      if (DOT && (((r - z0) & (kMaxDepth - 1)) == kMaxDepth - 1 || r == pz1 - 2)) {
        double v[6] = {gacc[0][0], gacc[0][1], gacc[0][2], gacc[1][0], gacc[1][1], gacc[1][2]};
        block_folds<6, 0>(v, nullptr, gsh);
        if (t == 0) {
          const int nt0 = I.ntiles0, ntx0 = (nx + kTX - 1) / kTX, nty0 = (ny + kTY - 1) / kTY;
          const int ta = tx + ntx0 * (2 * ty + nty0 * (r / kMaxDepth));
          I.partial[ta] = v[0];
          I.partial[nt0 + ta] = v[1];
          I.partial[2 * nt0 + ta] = v[2];
          if (2 * ty + 1 < nty0) {   // the upper dot tile exists
            I.partial[ta + ntx0] = v[3];
            I.partial[nt0 + ta + ntx0] = v[4];
            I.partial[2 * nt0 + ta + ntx0] = v[5];
          }
        }
#pragma unroll
        for (int kk = 0; kk < 2; ++kk) gacc[kk][0] = gacc[kk][1] = gacc[kk][2] = 0.0;
      }
    }
    __syncthreads();
  }
}

// ================================================ marching direction + SpMV
// d' = (z - zmean) + beta d on liquid cells, q = A d' and delta = d' . q
// (applyLiquidOperator, atlas :1171-1192), alpha = gamma / delta, as a 2.5-D
// march over tiles of kQX x kQY x kQZ level-0 cells.  The new direction goes to
// the other buffer (Ctrl::dsel flips in k_dirspmv_finish), so neighbours read
// the old direction race-free.  Step
// p stages d' = (z - zmean) + beta d of fine plane p on T +- 1 into a ring of
// 4 planes (pointwise, from loads prefetched one step earlier), and applies
// the operator to plane p - 2, whose neighbour planes earlier steps staged:
// q = diag d' - (sum of the six neighbours' d'); it writes d' and q of T and
// folds delta = d' . q.  One barrier per step.
constexpr int kQX = 32, kQY = 16, kQZ = 16;
constexpr int kQEX = kQX + 2, kQEY = kQY + 2, kQEP = kQEX * kQEY;
constexpr int kQPer = (kQEP + kMThreads - 1) / kMThreads;
constexpr int kQTPer = (kQX * kQY + kMThreads - 1) / kMThreads;

__host__ __device__ inline int march_spmv_tiles(int nx, int ny, int nz) {
  return ((nx + kQX - 1) / kQX) * ((ny + kQY - 1) / kQY) * ((nz + kQZ - 1) / kQZ);
}

__global__ void __launch_bounds__(kMThreads, 4) k_dirspmv_m(const InstDev* insts, const Tile* tiles) {
  __shared__ float dn_r[4][kQEP];
  __shared__ uint8_t lab_r[4][kQEP];
  __shared__ double sh[32];
  const Tile tl = tiles[blockIdx.x];
  const InstDev& I = insts[tl.inst];
  Ctrl* c = I.ctrl;
  if (c->done) return;
  const LevelDev& L = I.lv[0];
  const int nx = L.nx, ny = L.ny, nz = L.nz, nxy = nx * ny;
  const int ntx = (nx + kQX - 1) / kQX, nty = (ny + kQY - 1) / kQY;
  const int tx = tl.tile % ntx, tr = tl.tile / ntx, ty = tr % nty, tz = tr / nty;
  const int x0 = tx * kQX, y0 = ty * kQY, z0 = tz * kQZ;
  const int ex0 = x0 - 1, ey0 = y0 - 1, pz0 = z0 - 1, pz1 = min(z0 + kQZ, nz);   // none above the lattice
  const int sel = c->dsel;
  const float beta = float(c->beta), zm = float(c->zmean);
  const float* __restrict__ z = static_cast<const float*>(L.z);
  const float* __restrict__ dold = sel ? I.d2 : I.d;
  float* __restrict__ dnew = sel ? I.d : I.d2;
  const uint8_t* __restrict__ lab = L.label;
  const float* __restrict__ dgl = L.diag;
  float* __restrict__ Qo = I.q;
  const int t = threadIdx.x;
  int aoff[kQPer];
#pragma unroll
  for (int k = 0; k < kQPer; ++k) {
    const int e = t + k * kMThreads;
    const int gx = ex0 + e % kQEX, gy = ey0 + e / kQEX;
    aoff[k] = (e < kQEP && gx >= 0 && gy >= 0 && gx < nx && gy < ny) ? gx + nx * gy : -1;
  }
  int ts_[kQTPer], tofs[kQTPer];
#pragma unroll
  for (int k = 0; k < kQTPer; ++k) {
    const int e = t + k * kMThreads;
    const int lx = e % kQX, ly = e / kQX, gx = x0 + lx, gy = y0 + ly;
    ts_[k] = (ly + 1) * kQEX + lx + 1;
    tofs[k] = (e < kQX * kQY && gx < nx && gy < ny) ? gx + nx * gy : -1;
  }
  float pz_[kQPer], pd_[kQPer], pg_[kQTPer];
  uint8_t pl[kQPer];
  auto sl = [&](int p) { return (p - pz0) & 3; };
  // diagonal of plane g's interior liquid cells (g was staged in an earlier
  // step), one step ahead of its operator
  auto fetch_diag = [&](int g) {
    const bool gin = g >= z0 && g < nz;
#pragma unroll
    for (int k = 0; k < kQTPer; ++k)
      pg_[k] = (gin && tofs[k] >= 0 && lab_r[sl(g)][ts_[k]]) ? dgl[tofs[k] + nxy * g] : 0.0f;
  };
  auto fetch = [&](int p) {
    const bool pin = p >= 0 && p < nz;
#pragma unroll
    for (int k = 0; k < kQPer; ++k) {
      pz_[k] = 0.0f;
      pd_[k] = 0.0f;
      pl[k] = 0;
      if (pin && aoff[k] >= 0) {
        const int i = aoff[k] + nxy * p;
        pl[k] = lab[i];
        pz_[k] = z[i];
        pd_[k] = dold[i];
      }
    }
  };
  double dq = 0.0;
  fetch(pz0);
  fetch_diag(pz0 - 2);
  for (int p = pz0; p <= pz1 + 1; ++p) {
    // operator on plane r = p - 2 (planes r - 1 .. r + 1 were staged by earlier
    // steps); its diagonal was fetched in the previous step
    float dgr[kQTPer];
#pragma unroll
    for (int k = 0; k < kQTPer; ++k) dgr[k] = pg_[k];
    if (p <= pz1) {
      float* dn = dn_r[sl(p)];
      uint8_t* lb = lab_r[sl(p)];
#pragma unroll
      for (int k = 0; k < kQPer; ++k) {
        const int e = t + k * kMThreads;
        if (e >= kQEP) continue;
        dn[e] = pl[k] ? (beta == 0.0f ? pz_[k] - zm : (pz_[k] - zm) + beta * pd_[k]) : 0.0f;
        lb[e] = pl[k];
      }
      if (p < pz1) fetch(p + 1);
    }
    fetch_diag(p - 1);
    const int r = p - 2;
    if (r >= z0 && r < z0 + kQZ && r < nz) {
      const float* dn = dn_r[sl(r)];
      const float* dm = dn_r[sl(r - 1)];
      const float* dp = dn_r[sl(r + 1)];
      const uint8_t* lb = lab_r[sl(r)];
#pragma unroll
      for (int k = 0; k < kQTPer; ++k) {
        if (tofs[k] < 0) continue;
        const int s = ts_[k], i = tofs[k] + nxy * r;
        const float dv = dn[s];
        float q = 0.0f;
        if (lb[s]) {
          q = dgr[k] * dv - d4sum6(dn[s - 1], dn[s + 1], dn[s - kQEX], dn[s + kQEX], dm[s], dp[s]);
          dq += double(dv) * q;
        }
        dnew[i] = dv;
        Qo[i] = q;
      }
    }
    __syncthreads();
  }
  const double a0 = block_sum(dq, sh);
  if (t == 0) I.partial[tl.tile] = a0;
}

// delta of each listed instance from its k_dirspmv_m partials in tile order,
// alpha = gamma / delta, and the direction buffers swap (one CTA each).
__global__ void __launch_bounds__(kThreads) k_dirspmv_finish(const InstDev* insts, const int* ilist) {
  __shared__ double sh[32];
  const InstDev& I = insts[ilist[blockIdx.x]];
  Ctrl* c = I.ctrl;
  if (c->done) return;
  const LevelDev& L = I.lv[0];
  const int nt = march_spmv_tiles(L.nx, L.ny, L.nz);
  const int sel = c->dsel;
  const double delta = gather_slot(I.partial, 0, nt, 0, sh);
  if (threadIdx.x == 0) {
    finish_delta(c, delta);
    c->dsel = sel ^ 1;
  }
}

}  // namespace fpp
