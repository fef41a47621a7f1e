// Column-block V-cycle and direction+SpMV kernels for grid levels that coarsen
// by two on every axis.
//
// A thread owns one 2 x 2 block of fine cells in x / y (one coarse column) and
// marches it through the z planes of its tile.  In a plane the block holds two
// red and two black cells, and because block origins have even coordinate sums
// the red pair is cells {0, 3} on even planes and {1, 2} on odd planes for every
// thread: the colour pattern is uniform over the CTA, so the red and black
// phases run without divergence.  The block's own z neighbours (the planes
// above and below) stay in registers; only the four in-plane neighbours across
// the block's edges come from shared memory, where each plane is staged once.
// One barrier per plane separates the phases of a step, which work on
// different planes:
//
//   down (k_cdown), step p:  stage plane p (red cells z = rhs / diag from zero),
//     black sweep of plane p-1 and its black cells' residual, residual of the
//     red cells of plane p-2 (and the plane's z to the level's scratch), x pass
//     of the restriction of plane p-3, y and z passes of plane p-4.
//   up (k_cup), step p:  stage plane p (pre-smoothed z plus the prolongated
//     coarse correction), black sweep of plane p-1, red sweep of plane p-2 and
//     its output (level 0: the gamma partials of the fixed dot tiles).
//   direction + SpMV (k_cdirspmv), step p: stage d' of plane p, apply the
//     operator to plane p-1 (q, delta partials).
//
// Halo cells are recomputed by every tile that needs them with the owner's
// arithmetic, so results do not depend on the tiling (tile shape or z chunk),
// and the level-0 reductions fold over the fixed 32 x 8 x 8 dot tiles in a
// fixed order.  Which kernel runs on a level depends only on that level's
// coarsening, never on the batch, so a solve gives the same bits alone and in
// any batch.
//
// Per cell the arithmetic is the smoother, residual and restriction of the
// reference multigrid (mgSmoothColour mg.wgsl.ts:325-344, mgResidual :197-205,
// restriction = transpose of mgTrilinearPressure :217-241 over 2^3, as in the
// fused kernels) and the CG direction and operator of the atlas PCG
// (sparse-atlas-composite-projection.ts:1171-1192).
#pragma once
#include <type_traits>

#include "fused.cuh"

namespace fpp {

// ------------------------------------------------------------------ shapes
// Down step: kCDX x kCDY coarse columns per tile.  Its blocks are shifted by
// one fine cell (block X holds fine cells 2X-1 and 2X), so the restriction of
// coarse column X reads blocks X and X+1 only; the tile runs blocks
// cx0-1 .. cx0+kCDX+1 (fine rings 1-3 around the tile for the red, black and
// residual halos).
constexpr int kCDX = 16, kCDY = 8;
constexpr int kCDBX = kCDX + 3, kCDBY = kCDY + 3;
constexpr int kCDThreads = kCDBX * kCDBY;            // 209
// Up step and direction+SpMV: kCUX x kCUY aligned blocks (fine 2X, 2X+1) per
// tile, 32 x 16 fine cells = two dot tiles, plus a ring of one block.
constexpr int kCUX = 16, kCUY = 8;
constexpr int kCUBX = kCUX + 2, kCUBY = kCUY + 2;
constexpr int kCUThreads = kCUBX * kCUBY;            // 180
static_assert(2 * kCUX == kTX && 2 * kCUY == 2 * kTY && kMaxDepth == 8,
              "an up tile covers 1 x 2 dot tiles in x / y");
// Input planes are staged by asynchronous copies into a ring of kRing planes,
// kAhead planes ahead of the plane being staged; the ring also holds the two
// planes behind it, whose inputs the later phases read again.
constexpr int kRing = 6, kAhead = 3;

__host__ __device__ inline int cdown_tiles(int cnx, int cny, int cnz, int cdz) {
  return ((cnx + kCDX - 1) / kCDX) * ((cny + kCDY - 1) / kCDY) * ((cnz + cdz - 1) / cdz);
}
__host__ __device__ inline int cup_tiles(int nx, int ny, int nz, int cuz) {
  return ((nx + 2 * kCUX - 1) / (2 * kCUX)) * ((ny + 2 * kCUY - 1) / (2 * kCUY)) * ((nz + cuz - 1) / cuz);
}
// Dynamic shared memory of the three kernels (host and device).
__host__ __device__ constexpr int cplane_floats(int bx, int by) { return (2 * bx + 4) * (2 * by + 2); }
__host__ __device__ constexpr int cdown_smem() {
  return 16 * (kRing * 2 + 2) * kCDThreads + 4 * 4 * cplane_floats(kCDBX, kCDBY) + 8 * 2 * kCDThreads;
}
__host__ __device__ constexpr int cup_smem() {
  return 16 * kRing * 3 * kCUThreads + 4 * 4 * cplane_floats(kCUBX, kCUBY) + 4 * 2 * (kCUBX + 2) * (kCUBY + 2) +
         8 * 3 * 2 * 64;
}

// ---------------------------------------------------------- async copies
// cp.async of 4 bytes from global to shared memory (cached in L1); a copy of
// zero source bytes fills the destination with zeros and reads nothing.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem, bool valid) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(gmem), "r"(valid ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// One array's values at a block's four cells of one plane, staged as 16 bytes
// per thread.  Rows 0 and 1 of the block start at element indices i0 and i1
// (cells x and x + 1 of the row); v: bit k set when cell k lies in the
// lattice (k = kx + 2 ky).  Cells outside the lattice read as zero.
template <class T>
struct BlockCopy {   // 4-byte values: one copy per cell, zero-filled outside the lattice
  static_assert(sizeof(T) == 4, "4-byte element");
  // i0, i1 always lie in the lattice's planes (the caller clamps the plane), so
  // even the addresses of zero-filled copies stay inside the handle's memory
  static __device__ __forceinline__ void issue(uint4* dst, const T* src, int i0, int i1, unsigned v) {
    float* d = reinterpret_cast<float*>(dst);
    const T* a = src + i0;
    const T* b = src + i1;
    cp_async4(d + 0, a, v & 1u);
    cp_async4(d + 1, a + 1, v & 2u);
    cp_async4(d + 2, b, v & 4u);
    cp_async4(d + 3, b + 1, v & 8u);
  }
  static __device__ __forceinline__ float4 read(const uint4* s, int, int, unsigned) {
    return *reinterpret_cast<const float4*>(s);
  }
};
// 2-byte values: the aligned 4-byte words that hold a row's two cells (one
// word when the row starts at an even index, two otherwise), each copied only
// when it holds a cell of the lattice; the row's pair is taken out of the
// staged words by a byte permute, and cells outside the lattice are masked.
template <class T>
struct BlockCopy2 {
  static __device__ __forceinline__ void row(unsigned* d, const unsigned* w, int i, bool c0, bool c1) {
    const int a = i >> 1;   // word of cell 0 (floor, also for i = -1)
    const bool odd = i & 1;
    const bool n0 = c0 || (c1 && !odd), n1 = odd && c1;
    cp_async4(d + 0, n0 ? w + a : w, n0);
    cp_async4(d + 1, n1 ? w + a + 1 : w, n1);
  }
  static __device__ __forceinline__ void issue(uint4* dst, const T* src, int i0, int i1, unsigned v) {
    unsigned* d = reinterpret_cast<unsigned*>(dst);
    const unsigned* w = reinterpret_cast<const unsigned*>(src);
    row(d, w, i0, v & 1u, v & 2u);
    row(d + 2, w, i1, v & 4u, v & 8u);
  }
  static __device__ __forceinline__ float2 pair(unsigned lo, unsigned hi, int odd) {
    const unsigned e = __byte_perm(lo, hi, odd ? 0x5432 : 0x3210);
    if constexpr (std::is_same<T, __half>::value) {
      return __half22float2(*reinterpret_cast<const __half2*>(&e));
    } else {
      return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&e));
    }
  }
  static __device__ __forceinline__ float4 read(const uint4* s, int odd0, int odd1, unsigned v) {
    const uint4 w = *s;
    const float2 a = pair(w.x, w.y, odd0), b = pair(w.z, w.w, odd1);
    return make_float4((v & 1u) ? a.x : 0.0f, (v & 2u) ? a.y : 0.0f, (v & 4u) ? b.x : 0.0f, (v & 8u) ? b.y : 0.0f);
  }
};
template <class T>
using Copier = typename std::conditional<sizeof(T) == 4, BlockCopy<T>, BlockCopy2<T>>::type;

__device__ __forceinline__ float at4(const float4& v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }

// The smoothers of the column kernels divide by the diagonal with the
// hardware reciprocal (one MUFU operation, within an ulp or two): these kernels
// alone serve their levels, so every solve applies the same fixed operator.
__device__ __forceinline__ float rcpa(float d) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d));
  return r;
}

// A thread's block in a plane: its four cells' element offsets within a plane
// (row starts), lattice membership, and the plane's validity.
struct BlockRows {
  int r0, r1;        // element offsets of cells 0 and 2 within a plane (x + nx y)
  unsigned vxy;      // bit k: cell k inside the lattice in x / y
  int nxy, lo, hi;   // plane size; planes [lo, hi] are copied (others read as zero)
  __device__ __forceinline__ unsigned valid(int p) const { return (p >= lo && p <= hi) ? vxy : 0u; }
  __device__ __forceinline__ int clamp(int p) const { return min(max(p, lo), hi); }
  __device__ __forceinline__ int odd0(int p) const { return (r0 + nxy * p) & 1; }
  __device__ __forceinline__ int odd1(int p) const { return (r1 + nxy * p) & 1; }
};

// The ring slot of plane p when plane p0 sits in slot s0 (0 <= p - p0 + kRing).
__device__ __forceinline__ int ring(int s0, int d) {
  const int s = s0 + d;
  return s >= kRing ? s - kRing : (s < 0 ? s + kRing : s);
}

// The four in-plane neighbours of cell k of a block, as (xm, xp, ym, yp):
// in-block ones from v[], the two across the block's edges from the staged
// plane s at the block's cell (0, 0) = s[0] (row pitch W).
template <int K, int W>
__device__ __forceinline__ void nb4(const float* s, const float* v, float& xm, float& xp, float& ym, float& yp) {
  if (K == 0) { xm = s[-1]; xp = v[1]; ym = s[-W]; yp = v[2]; }
  if (K == 1) { xm = v[0]; xp = s[2]; ym = s[1 - W]; yp = v[3]; }
  if (K == 2) { xm = s[W - 1]; xp = v[3]; ym = v[0]; yp = s[2 * W]; }
  if (K == 3) { xm = v[2]; xp = s[W + 2]; ym = v[1]; yp = s[2 * W + 1]; }
}

template <int K, int W>
__device__ __forceinline__ float nbsum(const float* s, const float* v, float zm, float zp, float wx, float wy,
                                       float wz) {
  float xm, xp, ym, yp;
  nb4<K, W>(s, v, xm, xp, ym, yp);
  return d4sum6(wx * xm, wx * xp, wy * ym, wy * yp, wz * zm, wz * zp);
}

// The red pair of a plane of parity PAR: cells {0, 3} on even planes, {1, 2} on odd ones.
template <int PAR>
struct RedPair {
  static constexpr int a = PAR ? 1 : 0, b = PAR ? 2 : 3;
};

__device__ __forceinline__ void stage4(float* s, int W, const float* z) {
  *reinterpret_cast<float2*>(s) = make_float2(z[0], z[1]);
  *reinterpret_cast<float2*>(s + W) = make_float2(z[2], z[3]);
}

// ================================================================ down step
// z and residuals of one plane in the down step's pipeline (a liquid cell is
// one with a positive diagonal: the diagonal is zero on air and outside the lattice).
struct CDPlane {
  float z[4], res[4];
};

template <class TZ, class TR, class TD, class TS>
struct CDown {
  static constexpr int BX = kCDBX, BY = kCDBY, W = 2 * BX + 4, H = 2 * BY + 2, PL = W * H, N = kCDThreads;
  uint4* raw;         // [kRing][2][N]: rhs, diag of the block's cells per plane
  float* zs;          // [4][PL] staged z planes (ring), zero pads
  float4* rs4;        // [2][N] residuals of a plane per block
  float2* xs2;        // [2][N] x-pass sums of a plane per block (rows 0, 1)
  const TR* rhs;
  const TD* dg;
  TZ* zo;
  TS* out;
  const uint8_t* clab;
  BlockRows br;
  int nz, cnx, cny, cnz, nxy;
  int t, s00, X, Y;
  unsigned zmask;     // bit k: cell k's z is this tile's output (interior, in the lattice)
  bool res_ok, xpass_ok, emit_ok;
  int z_lo, z_hi;     // fine planes whose z this tile writes: [z_lo, z_hi)
  int cz0, cz1;
  float wx, wy, wz, scale, out_scale;
  float wxr[4], wyr[4];
  float accLo, accHi; // z pass: coarse planes m (lo) and m + 1 (hi)

  __device__ __forceinline__ void issue(int p, int slot) {
    const unsigned v = br.valid(p);
    const int pc = br.clamp(p), i0 = br.r0 + nxy * pc, i1 = br.r1 + nxy * pc;
    Copier<TR>::issue(raw + (slot * 2 + 0) * N + t, rhs, i0, i1, v);
    Copier<TD>::issue(raw + (slot * 2 + 1) * N + t, dg, i0, i1, v);
    cp_async_commit();
  }
  __device__ __forceinline__ void inputs(int p, int slot, float4& r, float4& d) const {
    const int o0 = br.odd0(p), o1 = br.odd1(p);
    r = Copier<TR>::read(raw + (slot * 2 + 0) * N + t, o0, o1, br.vxy);
    d = Copier<TD>::read(raw + (slot * 2 + 1) * N + t, o0, o1, br.vxy);
  }

  // z pass: fine plane f (parity PAR) with its y-pass sum ys
  template <int PAR>
  __device__ __forceinline__ void zpass(int f, float ys) {
    const bool fin = f >= 0 && f < nz;
    if (PAR) {   // f = 2m + 1: third tap of m (d = 1), first tap of m + 1 (d = -1)
      const int m = (f - 1) >> 1;
      if (fin) accLo = fmaf(p1d(f, m, cnz), ys, accLo);
      accHi = fin ? fmaf(p1d(f, m + 1, cnz), ys, 0.0f) : 0.0f;
    } else {     // f = 2m: last tap of m - 1 (d = 2, then emitted), second tap of m (d = 0)
      const int m = f >> 1;
      if (fin) accLo = fmaf(p1d(f, m - 1, cnz), ys, accLo);
      const int Z = m - 1;
      if (emit_ok && Z >= cz0 && Z < cz1) {
        const int ci = X + cnx * (Y + cny * Z);
        out[ci] = fromf<TS>(clab[ci] ? out_scale * accLo : 0.0f);
      }
      if (fin) accHi = fmaf(p1d(f, m, cnz), ys, accHi);
      accLo = accHi;
    }
  }

  // Step p (parity PAR), whose plane sits in ring slot sl.  A: plane p (staged
  // here), B: p - 1, C: p - 2, D: p - 3; xsE: own x-pass sums of plane p - 4.
  template <int PAR>
  __device__ __forceinline__ void step(int p, int sl, CDPlane& A, CDPlane& B, CDPlane& C, CDPlane& D, float2& xsE) {
    constexpr int ra = RedPair<PAR>::a, rb = RedPair<PAR>::b;
    issue(p + kAhead, ring(sl, kAhead));
    // stage plane p: red cells start the sweep at rhs / diag, black cells at zero
    {
      float4 r, d;
      inputs(p, sl, r, d);
#pragma unroll
      for (int k = 0; k < 4; ++k) A.z[k] = 0.0f;
      A.z[ra] = at4(d, ra) > 0.0f ? rnd<TZ>(at4(r, ra) * rcpa(at4(d, ra))) : 0.0f;
      A.z[rb] = at4(d, rb) > 0.0f ? rnd<TZ>(at4(r, rb) * rcpa(at4(d, rb))) : 0.0f;
      stage4(zs + (p & 3) * PL + s00, W, A.z);
    }
    // black sweep of plane p - 1 (cells ra, rb there) and those cells' residual
    {
      float4 r, d;
      inputs(p - 1, ring(sl, -1), r, d);
      float* s = zs + ((p - 1) & 3) * PL + s00;
      const float na = nbsum<ra, W>(s, B.z, C.z[ra], A.z[ra], wx, wy, wz);
      const float nb = nbsum<rb, W>(s, B.z, C.z[rb], A.z[rb], wx, wy, wz);
      const float ga = at4(d, ra), gb = at4(d, rb);
      B.z[ra] = ga > 0.0f ? rnd<TZ>((at4(r, ra) + na) * rcpa(ga)) : 0.0f;
      B.z[rb] = gb > 0.0f ? rnd<TZ>((at4(r, rb) + nb) * rcpa(gb)) : 0.0f;
      B.res[ra] = ga > 0.0f ? scale * (at4(r, ra) - (ga * B.z[ra] - na)) : 0.0f;
      B.res[rb] = gb > 0.0f ? scale * (at4(r, rb) - (gb * B.z[rb] - nb)) : 0.0f;
      s[(ra & 1) + (ra >> 1) * W] = B.z[ra];
      s[(rb & 1) + (rb >> 1) * W] = B.z[rb];
    }
    // red cells' residual of plane p - 2 (their neighbours are black and final)
    {
      const int rp = p - 2;
      float4 r, d;
      inputs(rp, ring(sl, -2), r, d);
      const float* s = zs + (rp & 3) * PL + s00;
      const float na = nbsum<ra, W>(s, C.z, D.z[ra], B.z[ra], wx, wy, wz);
      const float nb = nbsum<rb, W>(s, C.z, D.z[rb], B.z[rb], wx, wy, wz);
      const float ga = at4(d, ra), gb = at4(d, rb);
      C.res[ra] = ga > 0.0f ? scale * (at4(r, ra) - (ga * C.z[ra] - na)) : 0.0f;
      C.res[rb] = gb > 0.0f ? scale * (at4(r, rb) - (gb * C.z[rb] - nb)) : 0.0f;
      if (res_ok) rs4[(rp & 1) * N + t] = make_float4(C.res[0], C.res[1], C.res[2], C.res[3]);
      if (rp >= z_lo && rp < z_hi) {
        TZ* z0p = zo + (br.r0 + nxy * rp);
        TZ* z1p = zo + (br.r1 + nxy * rp);
        if (zmask & 1u) z0p[0] = fromf<TZ>(C.z[0]);
        if (zmask & 2u) z0p[1] = fromf<TZ>(C.z[1]);
        if (zmask & 4u) z1p[0] = fromf<TZ>(C.z[2]);
        if (zmask & 8u) z1p[1] = fromf<TZ>(C.z[3]);
      }
    }
    // x pass of plane p - 3: taps 2X-1, 2X (own block), 2X+1, 2X+2 (block X+1)
    float2 xsD = make_float2(0.0f, 0.0f);
    if (xpass_ok) {
      const float4 R = rs4[((p - 3) & 1) * N + t + 1];
      float s0 = 0.0f, s1 = 0.0f;
      s0 += wxr[0] * D.res[0];
      s0 += wxr[1] * D.res[1];
      s0 += wxr[2] * R.x;
      s0 += wxr[3] * R.y;
      s1 += wxr[0] * D.res[2];
      s1 += wxr[1] * D.res[3];
      s1 += wxr[2] * R.z;
      s1 += wxr[3] * R.w;
      xsD = make_float2(s0, s1);
      xs2[((p - 3) & 1) * N + t] = xsD;
    }
    // y pass of plane p - 4: rows 2Y-1, 2Y (own block), 2Y+1, 2Y+2 (block Y+1); then z pass
    if (emit_ok) {
      const float2 U = xs2[((p - 4) & 1) * N + t + BX];
      float sy = 0.0f;
      sy += wyr[0] * xsE.x;
      sy += wyr[1] * xsE.y;
      sy += wyr[2] * U.x;
      sy += wyr[3] * U.y;
      zpass<PAR>(p - 4, sy);
    }
    xsE = xsD;
    cp_async_wait<kAhead - 1>();   // plane p + 1 has landed (this thread's copies)
    __syncthreads();
  }
};

// Pre-smooth (one red-black sweep from z = 0), residual and restriction of
// level `level` into the right-hand side of level + 1 (coarsened by two on
// every axis), one tile of kCDX x kCDY coarse columns and F.cdz coarse planes
// per CTA.  On level 0 the residual is scaled by sigma and the smoother reads
// the float32 diagonal (TD = float), on coarser levels the stored one.
template <class TZ, class TR, class TD, class TS>
__global__ void __launch_bounds__(kCDThreads, 3) k_cdown(const InstDev* insts, const Tile* tiles, int level) {
  using K = CDown<TZ, TR, TD, TS>;
  extern __shared__ __align__(16) unsigned char csm[];
  const Tile tl = tiles[blockIdx.x];
  const InstDev& I = insts[tl.inst];
  const Ctrl* c = I.ctrl;
  if (c->done) return;
  const LevelDev& F = I.lv[level];
  const LevelDev& C = I.lv[level + 1];
  K k;
  k.raw = reinterpret_cast<uint4*>(csm);
  k.rs4 = reinterpret_cast<float4*>(k.raw + kRing * 2 * K::N);
  k.zs = reinterpret_cast<float*>(k.rs4 + 2 * K::N);
  k.xs2 = reinterpret_cast<float2*>(k.zs + 4 * K::PL);
  k.rhs = static_cast<const TR*>(F.rhs);
  k.dg = static_cast<const TD*>(level == 0 ? static_cast<const void*>(F.diag) : F.diagT);
  k.zo = static_cast<TZ*>(F.res);
  k.out = static_cast<TS*>(C.rhs);
  k.clab = C.label;
  const int nx = F.nx, ny = F.ny;
  k.nz = F.nz;
  k.nxy = nx * ny;
  k.cnx = C.nx;
  k.cny = C.ny;
  k.cnz = C.nz;
  k.wx = F.wx;
  k.wy = F.wy;
  k.wz = F.wz;
  k.scale = level == 0 ? float(c->sigma) : 1.0f;
  k.out_scale = F.to_coarse / 8.0f;
  const int ntx = (C.nx + kCDX - 1) / kCDX, nty = (C.ny + kCDY - 1) / kCDY;
  const int tx = tl.tile % ntx, tr = tl.tile / ntx, ty = tr % nty, tz = tr / nty;
  const int cx0 = tx * kCDX, cy0 = ty * kCDY;
  k.cz0 = tz * F.cdz;
  k.cz1 = min(k.cz0 + F.cdz, C.nz);
  const int t = threadIdx.x, bx = t % K::BX, by = t / K::BX;
  k.t = t;
  k.X = cx0 - 1 + bx;
  k.Y = cy0 - 1 + by;
  k.s00 = (1 + 2 * by) * K::W + 2 + 2 * bx;
  const int gx = 2 * k.X - 1, gy = 2 * k.Y - 1;   // fine cell 0 of the block
  k.zmask = 0;
  k.br.vxy = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int x = gx + (q & 1), y = gy + (q >> 1);
    const bool in = x >= 0 && y >= 0 && x < nx && y < ny;
    if (in) k.br.vxy |= 1u << q;
    if (in && x >= 2 * cx0 && x < 2 * (cx0 + kCDX) && y >= 2 * cy0 && y < 2 * (cy0 + kCDY)) k.zmask |= 1u << q;
  }
  k.br.r0 = gx + nx * gy;
  k.br.r1 = gx + nx * (gy + 1);
  k.br.nxy = k.nxy;
  const int pa = 2 * k.cz0 - 3, pb = 2 * k.cz1 + 2;   // fine planes staged: [pa, pb]
  k.br.lo = max(pa, 0);
  k.br.hi = min(pb, k.nz - 1);
  k.res_ok = bx >= 1 && bx <= kCDX + 1 && by >= 1 && by <= kCDY + 1;
  k.xpass_ok = bx >= 1 && bx <= kCDX && by >= 1 && by <= kCDY + 1;
  k.emit_ok = bx >= 1 && bx <= kCDX && by >= 1 && by <= kCDY && k.X < C.nx && k.Y < C.ny;
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    const int fx = 2 * k.X + d - 1, fy = 2 * k.Y + d - 1;
    k.wxr[d] = (k.X >= 0 && k.X < C.nx && fx >= 0 && fx < nx) ? p1d(fx, k.X, C.nx) : 0.0f;
    k.wyr[d] = (k.Y >= 0 && k.Y < C.ny && fy >= 0 && fy < ny) ? p1d(fy, k.Y, C.ny) : 0.0f;
  }
  k.z_lo = max(2 * k.cz0, 0);
  k.z_hi = min(2 * k.cz1, k.nz);
  k.accLo = k.accHi = 0.0f;
  for (int e = t; e < 4 * K::PL; e += blockDim.x) k.zs[e] = 0.0f;
  for (int e = t; e < kRing * 2 * K::N; e += blockDim.x) k.raw[e] = make_uint4(0u, 0u, 0u, 0u);
  __syncthreads();
  // the first kAhead planes, then the ring runs kAhead planes ahead of the stage
  for (int j = 0; j < kAhead; ++j) k.issue(pa + j, j);
  cp_async_wait<kAhead - 1>();
  __syncthreads();
  // planes in a ring of four register sets: plane p in P[(p - pa) & 3]
  CDPlane P0{}, P1{}, P2{}, P3{};
  float2 xsE = make_float2(0.0f, 0.0f);
  // steps pa .. pb + 2 (pa odd)
  const int steps = (pb + 2 - pa + 1 + 3) & ~3;   // a multiple of 4 (extra steps are no-ops)
  int sl = 0;
  for (int j = 0; j < steps; j += 4) {
    const int p = pa + j;
    k.template step<1>(p, sl, P0, P3, P2, P1, xsE);
    sl = ring(sl, 1);
    k.template step<0>(p + 1, sl, P1, P0, P3, P2, xsE);
    sl = ring(sl, 1);
    k.template step<1>(p + 2, sl, P2, P1, P0, P3, xsE);
    sl = ring(sl, 1);
    k.template step<0>(p + 3, sl, P3, P2, P1, P0, xsE);
    sl = ring(sl, 1);
  }
  cp_async_wait<0>();
}

// ================================================================== up step
struct CUPlane {
  float z[4];
};

template <class TZF, class TR, class TD, class TZC, bool DOT>
struct CUp {
  static constexpr int BX = kCUBX, BY = kCUBY, W = 2 * BX + 4, H = 2 * BY + 2, PL = W * H, N = kCUThreads;
  static constexpr int CW = BX + 2, CH = BY + 2, CP = CW * CH;   // coarse columns under the tile (+1 ring)
  uint4* raw;         // [kRing][3][N]: pre-smoothed z, rhs, diag per plane
  float* zs;          // [4][PL] staged z planes (ring), zero pads
  float* zcs;         // [2][CP] coarse z planes
  double* gsh;        // [3][2][64] dot-tile partials (DOT)
  const TZF* zf;
  const TR* rhs;
  const TD* dg;
  const TZC* zc;
  TZF* zo;
  double* partial;
  BlockRows br;
  int nz, cnx, cny, cnz, nxy, nt0, ntx0, nty0;
  int t, s00, c00, tx, ty, bx, by;
  unsigned omask;     // bit k: cell k is interior and in the lattice (output)
  bool interior;
  int z0, z1;
  int cx_lo, cy_lo;   // coarse origin of the coarse plane box
  float wx, wy, wz, unscale;
  float wxa[2], wxb[2], wya[2], wyb[2];   // prolongation taps: cell kx at columns (X-1+kx, X+kx), rows likewise
  float Ilo[4], Ihi[4];                   // x / y interpolated coarse planes m and m + 1
  float cpre[2];                          // the next coarse plane's values of this thread (read a step early)
  double rz, zsum, rsum;

  __device__ __forceinline__ void issue(int p, int slot) {
    const unsigned v = br.valid(p);
    const int pc = br.clamp(p), i0 = br.r0 + nxy * pc, i1 = br.r1 + nxy * pc;
    Copier<TZF>::issue(raw + (slot * 3 + 0) * N + t, zf, i0, i1, v);
    Copier<TR>::issue(raw + (slot * 3 + 1) * N + t, rhs, i0, i1, v);
    Copier<TD>::issue(raw + (slot * 3 + 2) * N + t, dg, i0, i1, v);
    cp_async_commit();
  }
  __device__ __forceinline__ float4 input(int p, int slot, int a) const {
    return (a == 0 ? Copier<TZF>::read(raw + (slot * 3) * N + t, br.odd0(p), br.odd1(p), br.vxy)
                   : a == 1 ? Copier<TR>::read(raw + (slot * 3 + 1) * N + t, br.odd0(p), br.odd1(p), br.vxy)
                            : Copier<TD>::read(raw + (slot * 3 + 2) * N + t, br.odd0(p), br.odd1(p), br.vxy));
  }

  // this thread's values of coarse plane Z (zero outside the coarse lattice)
  __device__ __forceinline__ void fetch_coarse(int Z) {
    const bool zin = Z >= 0 && Z < cnz;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int e = t + q * N;
      const int X = cx_lo + e % CW, Y = cy_lo + e / CW;
      cpre[q] = (zin && e < CP && X >= 0 && Y >= 0 && X < cnx && Y < cny) ? tof(zc[X + cnx * (Y + cny * Z)]) : 0.0f;
    }
  }
  __device__ __forceinline__ void store_coarse(int Z) {
    float* d = zcs + (Z & 1) * CP;
#pragma unroll
    for (int q = 0; q < 2; ++q)
      if (t + q * N < CP) d[t + q * N] = cpre[q];
  }

  // x then y interpolation of coarse plane Z (staged in slot Z & 1) at the block's four cells
  __device__ __forceinline__ void interp(int Z, float* out4) const {
    const float* q = zcs + (Z & 1) * CP + c00;
    float hx[3][2];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float a = q[j * CW], b = q[j * CW + 1], cc = q[j * CW + 2];
      hx[j][0] = fmaf(wxb[0], b, wxa[0] * a);
      hx[j][1] = fmaf(wxb[1], cc, wxa[1] * b);
    }
#pragma unroll
    for (int ky = 0; ky < 2; ++ky)
#pragma unroll
      for (int kx = 0; kx < 2; ++kx) out4[kx + 2 * ky] = fmaf(wyb[ky], hx[ky + 1][kx], wya[ky] * hx[ky][kx]);
  }

  // gamma partials of the dot tiles that end at fine plane r (fixed fold order)
  __device__ __forceinline__ void fold_dot(int r) {
    if (interior) {
      const int ix = bx - 1, iy = by - 1, dy = iy >> 2, q = ix + 16 * (iy & 3);
      gsh[(0 * 2 + dy) * 64 + q] = rz;
      gsh[(1 * 2 + dy) * 64 + q] = zsum;
      gsh[(2 * 2 + dy) * 64 + q] = rsum;
    }
    rz = zsum = rsum = 0.0;
    __syncthreads();
    const int w = t >> 5, l = t & 31;
    if (w < 2) {
      double v[3];
#pragma unroll
      for (int s = 0; s < 3; ++s) v[s] = gsh[(s * 2 + w) * 64 + l] + gsh[(s * 2 + w) * 64 + l + 32];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int s = 0; s < 3; ++s) v[s] += __shfl_xor_sync(0xffffffffu, v[s], o);
      const int tyd = 2 * ty + w;
      if (l == 0 && tyd < nty0) {
        const int ta = tx + ntx0 * (tyd + nty0 * (r >> 3));
#pragma unroll
        for (int s = 0; s < 3; ++s) partial[s * nt0 + ta] = v[s];
      }
    }
  }

  // Step p (parity PAR), whose plane sits in ring slot sl: A plane p (staged
  // here), B p - 1, C p - 2, D p - 3.
  template <int PAR>
  __device__ __forceinline__ void step(int p, int sl, CUPlane& A, CUPlane& B, CUPlane& C, CUPlane& D) {
    constexpr int ra = RedPair<PAR>::a, rb = RedPair<PAR>::b;
    issue(p + kAhead, ring(sl, kAhead));
    // coarse taps of fine plane p: (m, m + 1) = (p/2 - 1, p/2) for even p,
    // ((p-1)/2, (p+1)/2) for odd p.  An even step stores coarse plane p/2 + 1
    // (fetched the step before) for the odd step after it and fetches the next.
    if (PAR) {
#pragma unroll
      for (int k = 0; k < 4; ++k) Ilo[k] = Ihi[k];
      interp((p + 1) >> 1, Ihi);
    } else {
      store_coarse((p >> 1) + 1);
      fetch_coarse((p >> 1) + 2);
    }
    // stage plane p: z += P z_coarse on liquid cells
    {
      const float4 zp = input(p, sl, 0), d = input(p, sl, 2);
      const int mlo = PAR ? (p - 1) >> 1 : (p >> 1) - 1, mhi = mlo + 1;
      const bool vlo = mlo >= 0 && mlo < cnz, vhi = mhi >= 0 && mhi < cnz;
      const float wl = PAR ? 0.75f : 0.25f, wh = PAR ? 0.25f : 0.75f;
      const float wzl = vlo ? (vhi ? wl : 1.0f) : 0.0f, wzh = vhi ? (vlo ? wh : 1.0f) : 0.0f;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float corr = fmaf(wzh, Ihi[k], wzl * Ilo[k]);
        A.z[k] = at4(d, k) > 0.0f ? rnd<TZF>(at4(zp, k) + corr * unscale) : at4(zp, k);
      }
      stage4(zs + (p & 3) * PL + s00, W, A.z);
    }
    // black sweep of plane p - 1 (its black cells are ra, rb; neighbours red and staged)
    {
      const int sp = ring(sl, -1);
      const float4 r = input(p - 1, sp, 1), d = input(p - 1, sp, 2);
      float* s = zs + ((p - 1) & 3) * PL + s00;
      const float na = nbsum<ra, W>(s, B.z, C.z[ra], A.z[ra], wx, wy, wz);
      const float nb = nbsum<rb, W>(s, B.z, C.z[rb], A.z[rb], wx, wy, wz);
      if (at4(d, ra) > 0.0f) B.z[ra] = rnd<TZF>((at4(r, ra) + na) * rcpa(at4(d, ra)));
      if (at4(d, rb) > 0.0f) B.z[rb] = rnd<TZF>((at4(r, rb) + nb) * rcpa(at4(d, rb)));
      s[(ra & 1) + (ra >> 1) * W] = B.z[ra];
      s[(rb & 1) + (rb >> 1) * W] = B.z[rb];
    }
    // red sweep of plane rp = p - 2 (neighbours black and final), then its output
    {
      const int rp = p - 2, sp = ring(sl, -2);
      const float4 r = input(rp, sp, 1), d = input(rp, sp, 2);
      const float* s = zs + (rp & 3) * PL + s00;
      const float na = nbsum<ra, W>(s, C.z, D.z[ra], B.z[ra], wx, wy, wz);
      const float nb = nbsum<rb, W>(s, C.z, D.z[rb], B.z[rb], wx, wy, wz);
      if (at4(d, ra) > 0.0f) C.z[ra] = rnd<TZF>((at4(r, ra) + na) * rcpa(at4(d, ra)));
      if (at4(d, rb) > 0.0f) C.z[rb] = rnd<TZF>((at4(r, rb) + nb) * rcpa(at4(d, rb)));
      if (rp >= z0 && rp < z1) {
        TZF* z0p = zo + (br.r0 + nxy * rp);
        TZF* z1p = zo + (br.r1 + nxy * rp);
        if (omask & 1u) z0p[0] = fromf<TZF>(C.z[0]);
        if (omask & 2u) z0p[1] = fromf<TZF>(C.z[1]);
        if (omask & 4u) z1p[0] = fromf<TZF>(C.z[2]);
        if (omask & 8u) z1p[1] = fromf<TZF>(C.z[3]);
        if (DOT) {
#pragma unroll
          for (int k = 0; k < 4; ++k)
            if (((omask >> k) & 1u) && at4(d, k) > 0.0f) {
              const double zd = C.z[k], rd = at4(r, k);
              rz += rd * zd;
              zsum += zd;
              rsum += rd;
            }
          if ((rp & 7) == 7 || rp == nz - 1) fold_dot(rp);
        }
      }
    }
    cp_async_wait<kAhead - 1>();
    __syncthreads();
  }
};

// z_l += P z_{l+1} (mgProlongateAdd, mg.wgsl.ts:243-246; from level 1 into
// level 0 the sigma scaling is undone), then one sweep black then red, for a
// level whose next coarser level halves every axis; one tile of 32 x 16 fine
// columns and F.cuz planes per CTA.  With DOT (level 0) it also writes the
// gamma partials (r.z, sum z, sum r over liquid cells) of the 32 x 8 x 8 dot
// tiles it covers: each thread sums its block's cells in plane order, and the
// 64 blocks of a dot tile fold in a fixed tree.
template <class TZF, class TR, class TD, class TZC, bool DOT = false>
__global__ void __launch_bounds__(kCUThreads, 3) k_cup(const InstDev* insts, const Tile* tiles, int level) {
  using K = CUp<TZF, TR, TD, TZC, DOT>;
  extern __shared__ __align__(16) unsigned char csm[];
  const Tile tl = tiles[blockIdx.x];
  const InstDev& I = insts[tl.inst];
  const Ctrl* c = I.ctrl;
  if (c->done) return;
  const LevelDev& F = I.lv[level];
  const LevelDev& C = I.lv[level + 1];
  K k;
  k.raw = reinterpret_cast<uint4*>(csm);
  k.zs = reinterpret_cast<float*>(k.raw + kRing * 3 * K::N);
  k.zcs = k.zs + 4 * K::PL;
  k.gsh = reinterpret_cast<double*>(k.zcs + 2 * K::CP);
  k.zf = static_cast<const TZF*>(F.res);
  k.rhs = static_cast<const TR*>(F.rhs);
  k.dg = static_cast<const TD*>(level == 0 ? static_cast<const void*>(F.diag) : F.diagT);
  k.zc = static_cast<const TZC*>(C.z);
  k.zo = static_cast<TZF*>(F.z);
  k.partial = I.partial;
  const int nx = F.nx, ny = F.ny;
  k.nz = F.nz;
  k.nxy = nx * ny;
  k.cnx = C.nx;
  k.cny = C.ny;
  k.cnz = C.nz;
  k.nt0 = I.ntiles0;
  k.ntx0 = (nx + kTX - 1) / kTX;
  k.nty0 = (ny + kTY - 1) / kTY;
  k.wx = F.wx;
  k.wy = F.wy;
  k.wz = F.wz;
  k.unscale = level == 0 ? float(1.0 / c->sigma) : 1.0f;
  const int ntx = (nx + 2 * kCUX - 1) / (2 * kCUX), nty = (ny + 2 * kCUY - 1) / (2 * kCUY);
  k.tx = tl.tile % ntx;
  const int tr = tl.tile / ntx;
  k.ty = tr % nty;
  const int tz = tr / nty;
  k.z0 = tz * F.cuz;
  k.z1 = min(k.z0 + F.cuz, k.nz);
  const int t = threadIdx.x, bx = t % K::BX, by = t / K::BX;
  k.t = t;
  k.bx = bx;
  k.by = by;
  const int X = k.tx * kCUX - 1 + bx, Y = k.ty * kCUY - 1 + by;   // block = coarse column
  k.s00 = (1 + 2 * by) * K::W + 2 + 2 * bx;
  k.cx_lo = k.tx * kCUX - 2;
  k.cy_lo = k.ty * kCUY - 2;
  k.c00 = by * K::CW + bx;   // coarse (X - 1, Y - 1) in the coarse plane box
  k.interior = bx >= 1 && bx <= kCUX && by >= 1 && by <= kCUY;
  k.omask = 0;
  k.br.vxy = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int x = 2 * X + (q & 1), y = 2 * Y + (q >> 1);
    const bool in = x >= 0 && y >= 0 && x < nx && y < ny;
    if (in) k.br.vxy |= 1u << q;
    if (in && k.interior) k.omask |= 1u << q;
  }
  k.br.r0 = 2 * X + nx * (2 * Y);
  k.br.r1 = 2 * X + nx * (2 * Y + 1);
  k.br.nxy = k.nxy;
  const int pa = k.z0 - 2;   // fine planes staged: [z0 - 2, z1 + 1]
  k.br.lo = max(pa, 0);
  k.br.hi = min(k.z1 + 1, k.nz - 1);
  // prolongation taps with fixed positions (a dropped tap gets weight 0 and the
  // other 1, as in taps2): cell kx = 0 reads coarse columns X-1 (1/4), X (3/4);
  // kx = 1 reads X (3/4), X+1 (1/4)
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int xa = X - 1 + q, xb = X + q, ya = Y - 1 + q, yb = Y + q;
    const float wa = q ? 0.75f : 0.25f, wb = q ? 0.25f : 0.75f;
    const bool vxa = xa >= 0 && xa < C.nx, vxb = xb >= 0 && xb < C.nx;
    const bool vya = ya >= 0 && ya < C.ny, vyb = yb >= 0 && yb < C.ny;
    k.wxa[q] = vxa ? (vxb ? wa : 1.0f) : 0.0f;
    k.wxb[q] = vxb ? (vxa ? wb : 1.0f) : 0.0f;
    k.wya[q] = vya ? (vyb ? wa : 1.0f) : 0.0f;
    k.wyb[q] = vyb ? (vya ? wb : 1.0f) : 0.0f;
  }
  k.rz = k.zsum = k.rsum = 0.0;
  for (int e = t; e < 4 * K::PL; e += blockDim.x) k.zs[e] = 0.0f;
  for (int e = t; e < kRing * 3 * K::N; e += blockDim.x) k.raw[e] = make_uint4(0u, 0u, 0u, 0u);
  __syncthreads();
  for (int j = 0; j < kAhead; ++j) k.issue(pa + j, j);
  // the first step (even) interpolates coarse planes m0 = pa/2 - 1 and m0 + 1
  // and stores m0 + 2 for the odd step after it
  const int m0 = (pa >> 1) - 1;
  k.fetch_coarse(m0);
  k.store_coarse(m0);
  k.fetch_coarse(m0 + 1);
  __syncthreads();
  k.interp(m0, k.Ihi);
  k.store_coarse(m0 + 1);
  k.fetch_coarse(m0 + 2);
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; ++q) k.Ilo[q] = k.Ihi[q];
  k.interp(m0 + 1, k.Ihi);
  // (step pa stores coarse plane m0 + 2, which then overwrites plane m0's slot)
  cp_async_wait<kAhead - 1>();
  __syncthreads();
  CUPlane P0{}, P1{}, P2{}, P3{};   // plane p in P[(p - pa) & 3]
  const int steps = (k.z1 + 1 - pa + 1 + 3) & ~3;
  int sl = 0;
  for (int j = 0; j < steps; j += 4) {
    const int p = pa + j;
    k.template step<0>(p, sl, P0, P3, P2, P1);
    sl = ring(sl, 1);
    k.template step<1>(p + 1, sl, P1, P0, P3, P2);
    sl = ring(sl, 1);
    k.template step<0>(p + 2, sl, P2, P1, P0, P3);
    sl = ring(sl, 1);
    k.template step<1>(p + 3, sl, P3, P2, P1, P0);
    sl = ring(sl, 1);
  }
  cp_async_wait<0>();
}

// ================================================== direction + SpMV (level 0)
// One cell per thread: a CTA owns kSX x kSY level-0 columns (two dot tiles) plus
// a ring of one column, and marches them through its z chunk.  Its loads are
// coalesced along x and issued two planes ahead; the thread keeps its column's
// d' of planes p - 2 .. p in registers and reads the four in-plane neighbours
// from a ring of three staged planes (one barrier per plane).
constexpr int kSX = 32, kSY = 16;
constexpr int kSEX = kSX + 2, kSEY = kSY + 2;
constexpr int kSThreads = kSEX * kSEY;   // 612
static_assert(kSX == kTX && kSY == 2 * kTY, "a direction+SpMV tile covers 1 x 2 dot tiles");

__host__ __device__ inline int cspmv_tiles(int nx, int ny, int nz, int cqz) {
  return ((nx + kSX - 1) / kSX) * ((ny + kSY - 1) / kSY) * ((nz + cqz - 1) / cqz);
}

// d' = (z - zmean) + beta d on liquid cells, q = A d' and the delta partials of
// the 32 x 8 x 8 dot tiles (each interior thread sums its column's liquid cells
// in plane order; the 256 columns of a dot tile fold in a fixed order), one
// tile of kSX x kSY level-0 columns and L.cqz planes per CTA.  The new
// direction goes to the other buffer (Ctrl::dsel flips in k_dirspmv_finish),
// so neighbours read the old direction race-free.  A liquid cell is one with a
// positive diagonal.
__global__ void __launch_bounds__(kSThreads, 2) k_cdirspmv(const InstDev* insts, const Tile* tiles) {
  __shared__ float ds[3][kSThreads];
  __shared__ double gsh[2 * 256];
  const Tile tl = tiles[blockIdx.x];
  const InstDev& I = insts[tl.inst];
  Ctrl* c = I.ctrl;
  if (c->done) return;
  const LevelDev& L = I.lv[0];
  const int sel = c->dsel;
  const float* __restrict__ z = static_cast<const float*>(L.z);
  const float* __restrict__ dold = sel ? I.d2 : I.d;
  float* __restrict__ dnew = sel ? I.d : I.d2;
  float* __restrict__ Qo = I.q;
  const float* __restrict__ dgl = L.diag;
  const float beta = float(c->beta), zm = float(c->zmean);
  const int nx = L.nx, ny = L.ny, nz = L.nz, nxy = nx * ny;
  const int ntx = (nx + kSX - 1) / kSX, nty = (ny + kSY - 1) / kSY;
  const int tx = tl.tile % ntx, tr = tl.tile / ntx, ty = tr % nty, tz = tr / nty;
  const int z0 = tz * L.cqz, z1 = min(z0 + L.cqz, nz);
  const int t = threadIdx.x, lx = t % kSEX, ly = t / kSEX;
  const int x = tx * kSX - 1 + lx, y = ty * kSY - 1 + ly;
  const bool in = x >= 0 && y >= 0 && x < nx && y < ny;
  const bool interior = lx >= 1 && lx <= kSX && ly >= 1 && ly <= kSY;
  const bool out = in && interior;
  const int col = in ? x + nx * y : 0;   // a valid column for the addresses of cells outside the lattice
  // planes staged: [z0 - 1, z1]; loads of the planes in the lattice
  const int lo = max(z0 - 1, 0), hi = min(z1, nz - 1);
  float pz[2], pd[2], pg[2];   // prefetch of planes p + 1 (slot (p+1)&1) and p + 2
  auto fetch = [&](int p, int k) {
    const bool v = in && p >= lo && p <= hi;
    const int i = col + nxy * min(max(p, lo), hi);
    pz[k] = v ? z[i] : 0.0f;
    pd[k] = v ? dold[i] : 0.0f;
    pg[k] = v ? dgl[i] : 0.0f;
  };
  const int pa = z0 - 1;
  fetch(pa, 0);
  fetch(pa + 1, 1);
  float dm2 = 0.0f, dm1 = 0.0f, gm1 = 0.0f;   // d' of planes p - 2, p - 1 and the diagonal of p - 1
  double dq = 0.0;
  const int ntx0 = (nx + kTX - 1) / kTX, nty0 = (ny + kTY - 1) / kTY;
  int s0 = 0;   // ring slot of plane p
  // plane p's prefetch sits in pz/pd/pg[(p - pa) & 1]; two steps per iteration keep the index static
  auto step = [&](int p, auto K) {
    constexpr int k = decltype(K)::value;
    const float g = pg[k];
    const float dp = g > 0.0f ? (beta == 0.0f ? pz[k] - zm : (pz[k] - zm) + beta * pd[k]) : 0.0f;
    fetch(p + 2, k);
    ds[s0][t] = dp;
    __syncthreads();
    const int r = p - 1;
    if (r >= z0 && r < z1) {
      const float* sp = ds[s0 == 0 ? 2 : s0 - 1];   // plane r
      float q = 0.0f;
      if (interior && gm1 > 0.0f)
        q = gm1 * dm1 - d4sum6(sp[t - 1], sp[t + 1], sp[t - kSEX], sp[t + kSEX], dm2, dp);
      if (out) {
        const int i = col + nxy * r;
        dnew[i] = dm1;
        Qo[i] = q;
        if (gm1 > 0.0f) dq += double(dm1) * q;
      }
      // a dot tile ends every 8 planes and at the lattice top
      if ((r & 7) == 7 || r == nz - 1) {
        if (interior) gsh[((ly - 1) >> 3) * 256 + (lx - 1) + kSX * ((ly - 1) & 7)] = dq;
        dq = 0.0;
        __syncthreads();
        const int w = t >> 5, l = t & 31;
        if (w < 2) {
          double v = 0.0;
#pragma unroll
          for (int j = 0; j < 8; ++j) v += gsh[w * 256 + l + 32 * j];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          const int tyd = 2 * ty + w;
          if (l == 0 && tyd < nty0) I.partial[tx + ntx0 * (tyd + nty0 * (r >> 3))] = v;
        }
      }
    }
    dm2 = dm1;
    dm1 = dp;
    gm1 = g;
    s0 = s0 == 2 ? 0 : s0 + 1;
  };
  for (int p = pa; p <= z1; p += 2) {
    step(p, std::integral_constant<int, 0>());
    if (p + 1 <= z1) step(p + 1, std::integral_constant<int, 1>());
  }
}

// ================================================ float64 true residual (level 0)
// r = b - A x in float64 from the double-single pressure x + xlo, written over
// the CG residual, with ||r||^2 and max |r| (the acceptance check of
// octree-pipelined-pcg.ts:501-541), on the tiles of k_cdirspmv: one cell per
// thread marching its z chunk, the pressure of the in-plane neighbours staged
// as doubles in a ring of three planes.  Each dot tile's partials fold in a
// fixed order, and the instance's last tile to finish folds the dot tiles in
// order and applies the acceptance rule.  Runs when the instance is a
// candidate or on every true_every-th iteration.
__global__ void __launch_bounds__(kSThreads, 2) k_ctrue(const InstDev* insts, const Tile* tiles) {
  __shared__ double xs[3][kSThreads];
  __shared__ double gsh[2 * 2 * 256];
  __shared__ int flag;
  const Tile tl = tiles[blockIdx.x];
  const InstDev& I = insts[tl.inst];
  Ctrl* c = I.ctrl;
  if (c->done || !(c->candidate || (c->true_every > 0 && c->iter % c->true_every == 0))) return;
  const LevelDev& L = I.lv[0];
  const float* __restrict__ Xh = I.x;
  const float* __restrict__ Xl = I.xlo;
  const float* __restrict__ B = I.b;
  const float* __restrict__ dgl = L.diag;
  float* __restrict__ R = static_cast<float*>(L.rhs);
  const int nx = L.nx, ny = L.ny, nz = L.nz, nxy = nx * ny;
  const int ntx = (nx + kSX - 1) / kSX, nty = (ny + kSY - 1) / kSY;
  const int tx = tl.tile % ntx, tr = tl.tile / ntx, ty = tr % nty, tz = tr / nty;
  const int z0 = tz * L.cqz, z1 = min(z0 + L.cqz, nz);
  const int t = threadIdx.x, lx = t % kSEX, ly = t / kSEX;
  const int x = tx * kSX - 1 + lx, y = ty * kSY - 1 + ly;
  const bool in = x >= 0 && y >= 0 && x < nx && y < ny;
  const bool interior = lx >= 1 && lx <= kSX && ly >= 1 && ly <= kSY;
  const bool out = in && interior;
  const int col = in ? x + nx * y : 0;
  const int lo = max(z0 - 1, 0), hi = min(z1, nz - 1);
  // prefetch of planes p + 1 and p + 2: pressure (hi, lo), and for the
  // operator's own cells b and the diagonal
  float ph[2], pl[2], pb[2], pg[2];
  auto fetch = [&](int p, int k) {
    const bool v = in && p >= lo && p <= hi;
    const int i = col + nxy * min(max(p, lo), hi);
    ph[k] = v ? Xh[i] : 0.0f;
    pl[k] = v ? Xl[i] : 0.0f;
    const bool own = v && interior && p >= z0 && p < z1;
    pb[k] = own ? B[i] : 0.0f;
    pg[k] = own ? dgl[i] : 0.0f;
  };
  const int pa = z0 - 1;
  fetch(pa, 0);
  fetch(pa + 1, 1);
  double xm2 = 0.0, xm1 = 0.0;   // pressure of planes p - 2, p - 1 in this column
  float bm1 = 0.0f, gm1 = 0.0f;  // b and diagonal of plane p - 1
  double rr = 0.0, mr = 0.0;
  const int ntx0 = (nx + kTX - 1) / kTX, nty0 = (ny + kTY - 1) / kTY, nt0 = I.ntiles0;
  double* partial = I.partial;
  int s0 = 0;
  auto step = [&](int p, auto K) {
    constexpr int k = decltype(K)::value;
    const double xp = double(ph[k]) + double(pl[k]);
    const float bp = pb[k], gp = pg[k];
    fetch(p + 2, k);
    xs[s0][t] = xp;
    __syncthreads();
    const int r = p - 1;
    if (r >= z0 && r < z1) {
      const double* sp = xs[s0 == 0 ? 2 : s0 - 1];   // plane r
      if (out && gm1 > 0.0f) {
        const double nbs = ((sp[t - 1] + sp[t + 1]) + (xm2 + xp)) + (sp[t - kSEX] + sp[t + kSEX]);
        const double rv = double(bm1) - (double(gm1) * xm1 - nbs);
        R[col + nxy * r] = float(rv);
        rr += rv * rv;
        mr = fmax(mr, fabs(rv));
      }
      if ((r & 7) == 7 || r == nz - 1) {
        if (interior) {
          const int q = ((ly - 1) >> 3) * 256 + (lx - 1) + kSX * ((ly - 1) & 7);
          gsh[q] = rr;
          gsh[512 + q] = mr;
        }
        rr = 0.0;
        mr = 0.0;
        __syncthreads();
        const int w = t >> 5, l = t & 31;
        if (w < 4) {
          const int dy = w & 1, m = w >> 1;   // warps 0, 1: sums; 2, 3: maxima
          double v = 0.0;
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const double e = gsh[m * 512 + dy * 256 + l + 32 * j];
            v = m ? fmax(v, e) : v + e;
          }
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            const double e = __shfl_xor_sync(0xffffffffu, v, o);
            v = m ? fmax(v, e) : v + e;
          }
          const int tyd = 2 * ty + dy;
          if (l == 0 && tyd < nty0) partial[m * nt0 + tx + ntx0 * (tyd + nty0 * (r >> 3))] = v;
        }
      }
    }
    xm2 = xm1;
    xm1 = xp;
    bm1 = bp;
    gm1 = gp;
    s0 = s0 == 2 ? 0 : s0 + 1;
  };
  for (int p = pa; p <= z1; p += 2) {
    step(p, std::integral_constant<int, 0>());
    if (p + 1 <= z1) step(p + 1, std::integral_constant<int, 1>());
  }
  // the instance's last tile folds the dot tiles in order
  __shared__ double sh[32];
  if (arrive_last(&c->arrive[kStTrue], cspmv_tiles(nx, ny, nz, L.cqz), &flag)) {
    const double sum = gather_slot(partial, 0, nt0, 0, sh);
    const double mx = gather_slot(partial, 1, nt0, 1, sh);
    if (threadIdx.x == 0) finish_true(c, sum, mx);
  }
}

// ==================================================== CG update (level 0)
// x += alpha d (double-single), r -= alpha q, with the ||r||^2 and max |r|
// partials of each dot tile (k_update_finish folds them in dot-tile order), on
// the tiles of k_cdirspmv without their ring: one cell per thread, loads issued
// two planes ahead.  Each warp holds one x row of a dot tile, so a dot tile's
// partial folds its eight warps' shuffle trees in order.
constexpr int kUThreads = kSX * kSY;   // 512
__global__ void __launch_bounds__(kUThreads, 3) k_cupdate(const InstDev* insts, const Tile* tiles) {
  __shared__ double wsh[2][kUThreads / 32];
  const Tile tl = tiles[blockIdx.x];
  const InstDev& I = insts[tl.inst];
  Ctrl* c = I.ctrl;
  if (c->done) return;
  const LevelDev& L = I.lv[0];
  const double alpha = c->alpha;
  const float alpha_f = float(alpha);
  float* __restrict__ X = I.x;
  float* __restrict__ Xlo = I.xlo;
  const float* __restrict__ D = dir_cur(I);
  const float* __restrict__ Q = I.q;
  float* __restrict__ R = static_cast<float*>(L.rhs);
  const uint8_t* __restrict__ lab = L.label;
  const int nx = L.nx, ny = L.ny, nz = L.nz, nxy = nx * ny;
  const int ntx = (nx + kSX - 1) / kSX, nty = (ny + kSY - 1) / kSY;
  const int tx = tl.tile % ntx, tr = tl.tile / ntx, ty = tr % nty, tz = tr / nty;
  const int z0 = tz * L.cqz, z1 = min(z0 + L.cqz, nz);
  const int t = threadIdx.x, lx = t % kSX, ly = t / kSX;
  const int x = tx * kSX + lx, y = ty * kSY + ly;
  const bool in = x < nx && y < ny;
  const int col = in ? x + nx * y : 0;
  float ph[2], pl[2], pd[2], pq[2], pr[2];
  uint8_t pb[2];
  auto fetch = [&](int p, int k) {
    const bool v = in && p < z1;
    const int i = col + nxy * min(p, z1 - 1);
    pb[k] = v ? lab[i] : 0;
    ph[k] = v ? X[i] : 0.0f;
    pl[k] = v ? Xlo[i] : 0.0f;
    pd[k] = v ? D[i] : 0.0f;
    pq[k] = v ? Q[i] : 0.0f;
    pr[k] = v ? R[i] : 0.0f;
  };
  fetch(z0, 0);
  fetch(z0 + 1, 1);
  double rr = 0.0, mr = 0.0;
  const int ntx0 = (nx + kTX - 1) / kTX, nty0 = (ny + kTY - 1) / kTY, nt0 = I.ntiles0;
  auto step = [&](int p, auto K) {
    constexpr int k = decltype(K)::value;
    const bool lq = pb[k] != 0;
    const float h = ph[k], lo = pl[k], dv = pd[k], qv = pq[k], r0 = pr[k];
    fetch(p + 2, k);
    if (lq) {
      const int i = col + nxy * p;
      // double-single accumulation: x_hi + x_lo carries the pressure to ~1e-14
      const double xv = double(h) + double(lo) + alpha * double(dv);
      const float hi = float(xv);
      X[i] = hi;
      Xlo[i] = float(xv - double(hi));
      const float rv = r0 - alpha_f * qv;
      R[i] = rv;
      rr += double(rv) * rv;
      mr = fmax(mr, fabs(double(rv)));
    }
    // a dot tile ends every 8 planes and at the lattice top
    if ((p & 7) == 7 || p == nz - 1) {
      double a = rr, m = mr;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
      }
      const int w = t >> 5;
      if ((t & 31) == 0) {
        wsh[0][w] = a;
        wsh[1][w] = m;
      }
      rr = 0.0;
      mr = 0.0;
      __syncthreads();
      if (t < 2) {   // thread dy folds the eight rows of dot tile dy in order
        double sa = 0.0, sm = 0.0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          sa += wsh[0][8 * t + j];
          sm = fmax(sm, wsh[1][8 * t + j]);
        }
        const int tyd = 2 * ty + t;
        if (tyd < nty0) {
          const int ta = tx + ntx0 * (tyd + nty0 * (p >> 3));
          I.partial[ta] = sa;
          I.partial[nt0 + ta] = sm;
        }
      }
      __syncthreads();
    }
  };
  for (int p = z0; p < z1; p += 2) {
    step(p, std::integral_constant<int, 0>());
    if (p + 1 < z1) step(p + 1, std::integral_constant<int, 1>());
  }
}

// delta of each listed instance from its k_cdirspmv partials in dot-tile
// order, alpha = gamma / delta, and the direction buffers swap (one CTA each).
__global__ void __launch_bounds__(kThreads) k_dirspmv_finish(const InstDev* insts, const int* ilist) {
  __shared__ double sh[32];
  const InstDev& I = insts[ilist[blockIdx.x]];
  Ctrl* c = I.ctrl;
  if (c->done) return;
  const int sel = c->dsel;
  const double delta = gather_slot(I.partial, 0, I.ntiles0, 0, sh);
  if (threadIdx.x == 0) {
    finish_delta(c, delta);
    c->dsel = sel ^ 1;
  }
}

}  // namespace fpp
