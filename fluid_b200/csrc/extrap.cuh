// Velocity extrapolation into the air (CM12 Sec. 3.3, CM11b Secs. 3.3 and
// 3.3.1, Jeong/Ross/Whitaker 2007), the step that runs right before the
// projection's consumer (advection) in the reference
// (lib/methods/uniform/webgpu-uniform-velocity-extrapolation.ts and its
// .wgsl.ts).
//
// The lattice is every cell's +x, +y, +z MAC face (component c of cell p is
// the face between p and p + e_c).  A face is open when it is not a closed wall
// (the domain walls; with embedded solids, faces whose open fraction is at or
// below 1e-5); a source face is an open face with a liquid side (rho' > 0.5).
//  1. The narrow band: the Fast Iterative Method solves the Eikonal distance
//     from the source faces and carries the velocity along it by the upwind
//     extension n . grad u = 0, per component on its own face lattice, up to
//     two cells from the liquid, in at most min(max dims, 16) Jacobi-style
//     passes that stop when the active list is empty (seedActiveFront,
//     updateActiveFront, prepareActiveDispatch, resolveConvergedFront).
//  2. The rest of the air: the known values are restricted down a hierarchy of
//     ceil-halved lattices by renormalised trilinear interpolation of known
//     values only, then prolongated back up filling only unknown values
//     (restrictKnownVelocity, prolongUnknownVelocity).
//  3. The open faces of the lattice take the result (packTransportShell).
// Every floating-point operation is written with round-to-nearest intrinsics,
// in the reference's evaluation order, so the float restatement of the oracle
// reproduces it bit for bit.
#pragma once

#include "solids.cuh"

namespace fpp {

constexpr float kDistInf = 65504.0f;   // DISTANCE_INFINITY
constexpr float kBandCells = 2.0f;     // ACCURATE_BAND_CELLS

struct ExtDev {
  int nx, ny, nz;
  float h;                 // cubic cells
  int open_top, solids;
  const float* vof;
  const float* open;       // cell open fractions (solids) or null
  const float* fv[3];      // face open fractions (solids) or null
  float* vel[3];           // u, v, w (the handle's MAC arrays)
  float4* val[2];          // FIM values (xyz) and known mask (w)
  float4* dist[2];         // FIM distances (xyz) and active mask (w)
  unsigned* count;         // active components written per side; [3] the band's node count
  uint8_t* mark[2];        // band marks (liquid cells, then dilated)
  unsigned* band;          // the band's node indices
};

// The narrow band's passes touch only nodes within a few cells of a source
// face: a node becomes known only at an upwind distance <= 2 h, and one is
// activated only next to a node with a finite distance; a node of a liquid
// cell is a source face (skipped).  The passes therefore run over the air
// cells within kBandReach cells (Chebyshev) of a liquid cell, listed once per
// call; every other node keeps its seeded state, which the seed writes to
// both sides.
constexpr int kBandReach = 6;

__device__ __forceinline__ bool ext_in(const ExtDev& E, int x, int y, int z) {
  return x >= 0 && y >= 0 && z >= 0 && x < E.nx && y < E.ny && z < E.nz;
}
__device__ __forceinline__ long long ext_idx(const ExtDev& E, int x, int y, int z) {
  return x + (long long)E.nx * (y + (long long)E.ny * z);
}
// MAC index of the +face of cell (x, y, z) on axis c.
__device__ __forceinline__ long long ext_face(const ExtDev& E, int c, int x, int y, int z) {
  if (c == 0) return (x + 1) + (long long)(E.nx + 1) * (y + (long long)E.ny * z);
  if (c == 1) return x + (long long)E.nx * ((y + 1) + (long long)(E.ny + 1) * z);
  return x + (long long)E.nx * (y + (long long)E.ny * (z + 1));
}
// openBaseFace: inside the lattice and not a closed wall or closed solid face.
__device__ __forceinline__ bool ext_open(const ExtDev& E, int x, int y, int z, int c) {
  if (!ext_in(E, x, y, z)) return false;
  if (c == 0 && x + 1 >= E.nx) return false;
  if (c == 1 && y + 1 >= E.ny && !E.open_top) return false;
  if (c == 2 && z + 1 >= E.nz) return false;
  if (!E.solids) return true;
  return clamp01(E.fv[c][ext_face(E, c, x, y, z)]) > 1e-5f;
}
// rho' of cell i = (x, y, z) of an nx x ny x nz lattice with embedded solids:
// the fill over the cell's open fraction, and in a solid cell the largest of
// its open neighbours'.
__device__ __forceinline__ float ext_density_solid(const float* vof, const float* open, int nx, int ny, int nz, int x,
                                                int y, int z) {
  const long long i = x + (long long)nx * (y + (long long)ny * z);
  const float v = clamp01(open[i]);
  if (v > kSolidCell) return __fdiv_rn(vof[i], v);
  float best = 0.0f;
  const int dx[6] = {-1, 1, 0, 0, 0, 0}, dy[6] = {0, 0, -1, 1, 0, 0}, dz[6] = {0, 0, 0, 0, -1, 1};
  for (int k = 0; k < 6; ++k) {
    const int X = x + dx[k], Y = y + dy[k], Z = z + dz[k];
    if (X < 0 || Y < 0 || Z < 0 || X >= nx || Y >= ny || Z >= nz) continue;
    const long long j = X + (long long)nx * (Y + (long long)ny * Z);
    const float vj = clamp01(open[j]);
    if (vj > kSolidCell) best = fmaxf(best, __fdiv_rn(vof[j], vj));
  }
  return best;
}
// rho' of cell (x, y, z), 0 outside the lattice.
__device__ __forceinline__ float ext_density(const ExtDev& E, int x, int y, int z) {
  if (!ext_in(E, x, y, z)) return 0.0f;
  if (!E.solids) return E.vof[ext_idx(E, x, y, z)];
  return ext_density_solid(E.vof, E.open, E.nx, E.ny, E.nz, x, y, z);
}
__device__ __forceinline__ bool ext_source(const ExtDev& E, int x, int y, int z, int c) {
  if (!ext_open(E, x, y, z, c)) return false;
  return ext_density(E, x, y, z) > 0.5f ||
         ext_density(E, x + (c == 0), y + (c == 1), z + (c == 2)) > 0.5f;
}
__device__ __forceinline__ float at3(const float4& v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }
__device__ __forceinline__ void set3(float4& v, int c, float s) {
  if (c == 0) v.x = s;
  else if (c == 1) v.y = s;
  else v.z = s;
}
__device__ __forceinline__ bool has_bit(float w, int c) { return (unsigned(w) >> c) & 1u; }

// The FIM state read by one pass (the source side), with the pass's
// constants formed once: 1 / h^2 of godunovDistance, the clamp of
// fimConvergenceEpsilon (2 h and the lattice diagonal) and the band limit.
struct ExtSrc {
  const ExtDev& E;
  const float4* val;
  const float4* dist;
  float inv_h2, eps_lo, eps_hi, band;
  __device__ ExtSrc(const ExtDev& e, int side)
      : E(e), val(side ? e.val[1] : e.val[0]), dist(side ? e.dist[1] : e.dist[0]) {
    inv_h2 = __fdiv_rn(1.0f, __fmul_rn(e.h, e.h));
    eps_lo = __fmul_rn(2.0f, e.h);
    const float ex = __fmul_rn(float(e.nx), e.h), ey = __fmul_rn(float(e.ny), e.h), ez = __fmul_rn(float(e.nz), e.h);
    eps_hi = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey)), __fmul_rn(ez, ez)));
    band = __fmul_rn(kBandCells, e.h);
  }
  // fimConvergenceEpsilon
  __device__ float eps(float ref) const { return __fmul_rn(fminf(fmaxf(fabsf(ref), eps_lo), eps_hi), 1.1920929e-7f); }
  // component c (or the mask, 3) of a node's state, one scalar load
  __device__ float dc(long long i, int c) const { return reinterpret_cast<const float*>(dist + i)[c]; }
  __device__ float vc(long long i, int c) const { return reinterpret_cast<const float*>(val + i)[c]; }
  __device__ float nd(int x, int y, int z, int c) const {   // neighborDistance
    if (!ext_open(E, x, y, z, c)) return kDistInf;
    return dc(ext_idx(E, x, y, z), c);
  }
  __device__ float nv(int x, int y, int z, int c) const {   // neighborValue
    if (!ext_open(E, x, y, z, c)) return 0.0f;
    const long long i = ext_idx(E, x, y, z);
    return has_bit(vc(i, 3), c) ? vc(i, c) : 0.0f;
  }
  // godunovDistance (JRW07 Eq. 2.1 with f = 1), cubic cells
  __device__ float godunov(int x, int y, int z, int c) const {
    float m[3];
    m[0] = fminf(nd(x - 1, y, z, c), nd(x + 1, y, z, c));
    m[1] = fminf(nd(x, y - 1, z, c), nd(x, y + 1, z, c));
    m[2] = fminf(nd(x, y, z - 1, c), nd(x, y, z + 1, c));
    for (int i = 0; i < 2; ++i)
      for (int j = i + 1; j < 3; ++j)
        if (m[j] < m[i]) {
          const float a = m[i];
          m[i] = m[j];
          m[j] = a;
        }
    if (m[0] >= 0.5f * kDistInf) return kDistInf;
    const float h = E.h;
    float root = __fadd_rn(m[0], h);
    for (int count = 2; count <= 3; ++count) {
      if (m[count - 1] >= 0.5f * kDistInf || root <= m[count - 1]) break;
      float a = 0.0f, b = 0.0f, cc = -1.0f;
      for (int k = 0; k < count; ++k) {
        const float inv = inv_h2;
        a = __fadd_rn(a, inv);
        b = __fadd_rn(b, __fmul_rn(m[k], inv));
        cc = __fadd_rn(cc, __fmul_rn(__fmul_rn(m[k], m[k]), inv));
      }
      root = __fdiv_rn(__fadd_rn(b, __fsqrt_rn(fmaxf(__fsub_rn(__fmul_rn(b, b), __fmul_rn(a, cc)), 0.0f))), a);
    }
    return root;
  }
  // upwindExtensionValue
  __device__ float upwind(int x, int y, int z, int c, float solved) const {
    float wt[3], ww[3];
    const float eps = this->eps(solved);
    const float h2 = __fmul_rn(E.h, E.h);
    for (int a = 0; a < 3; ++a) {
      wt[a] = 0.0f;
      ww[a] = 0.0f;
      const int ox = a == 0, oy = a == 1, oz = a == 2;
      const float lo = nd(x - ox, y - oy, z - oz, c), hi = nd(x + ox, y + oy, z + oz, c);
      const float mn = fminf(lo, hi);
      if (mn >= __fsub_rn(solved, eps)) continue;
      float mv = 0.0f, mc = 0.0f;
      if (fabsf(__fsub_rn(lo, mn)) <= eps) {
        mv = __fadd_rn(mv, nv(x - ox, y - oy, z - oz, c));
        mc = __fadd_rn(mc, 1.0f);
      }
      if (fabsf(__fsub_rn(hi, mn)) <= eps) {
        mv = __fadd_rn(mv, nv(x + ox, y + oy, z + oz, c));
        mc = __fadd_rn(mc, 1.0f);
      }
      if (mc <= 0.0f) continue;
      const float w = __fdiv_rn(__fsub_rn(solved, mn), h2);
      wt[a] = __fdiv_rn(__fmul_rn(w, mv), mc);
      ww[a] = w;
    }
    const float sv = __fadd_rn(__fadd_rn(wt[0], wt[2]), wt[1]);
    const float sw = __fadd_rn(__fadd_rn(ww[0], ww[2]), ww[1]);
    return sw > 0.0f ? __fdiv_rn(sv, sw) : 0.0f;
  }
  // activeNodeConverges; upd: the node's updated distance min(old, godunov)
  __device__ bool converges(int x, int y, int z, int c, float& upd) const {
    if (!ext_open(E, x, y, z, c) || ext_source(E, x, y, z, c)) return false;
    const long long i = ext_idx(E, x, y, z);
    if (!has_bit(dc(i, 3), c)) return false;
    const float old = dc(i, c);
    if (old >= 0.5f * kDistInf) return false;
    upd = fminf(old, godunov(x, y, z, c));
    if (upd > band) return false;
    return fabsf(__fsub_rn(upd, old)) <= eps(old);
  }
  // activatedByConvergedUpwindNeighbor.  A converging neighbour's
  // min(neighborDistance, godunovDistance) is its updated distance, which
  // converges() has formed.
  __device__ bool activated(int x, int y, int z, int c) const {
    const float cand = godunov(x, y, z, c);
    if (!ext_open(E, x, y, z, c) || cand > band) return false;
    const float own = dc(ext_idx(E, x, y, z), c);
    const float eps = this->eps(own);
#pragma unroll 1
    for (int a = 0; a < 3; ++a) {
      const int ox = a == 0, oy = a == 1, oz = a == 2;
#pragma unroll 1
      for (int s = -1; s <= 1; s += 2) {
        const int X = x + s * ox, Y = y + s * oy, Z = z + s * oz;
        float un;
        if (!converges(X, Y, Z, c, un)) continue;
        if (own > __fadd_rn(un, eps)) return true;
      }
    }
    return false;
  }
};

__device__ __forceinline__ bool touches_source(const ExtDev& E, int x, int y, int z, int c) {
  for (int a = 0; a < 3; ++a) {
    const int ox = a == 0, oy = a == 1, oz = a == 2;
    if (ext_in(E, x - ox, y - oy, z - oz) && ext_source(E, x - ox, y - oy, z - oz, c)) return true;
    if (ext_in(E, x + ox, y + oy, z + oz) && ext_source(E, x + ox, y + oy, z + oz, c)) return true;
  }
  return false;
}

#define EXT_FOR_CELLS(E, x, y, z, i)                                                                     \
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x,                                  \
                 n_ = (long long)(E).nx * (E).ny * (E).nz;                                             \
       i < n_; i += (long long)gridDim.x * blockDim.x)                                                 \
    if (const int x = int(i % (E).nx), y = int((i / (E).nx) % (E).ny), z = int(i / ((long long)(E).nx * (E).ny)); \
        true)

// seedActiveFront into both sides (SOLIDS as in k_ext_update).
template <bool SOLIDS>
__global__ void k_ext_seed(ExtDev Ein) {
  ExtDev E = Ein;
  E.solids = SOLIDS ? 1 : 0;
  unsigned active_total = 0;
  EXT_FOR_CELLS(E, x, y, z, i) {
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f), d = make_float4(kDistInf, kDistInf, kDistInf, 0.f);
    unsigned known = 0, active = 0;
    for (int c = 0; c < 3; ++c) {
      if (!ext_open(E, x, y, z, c)) continue;
      if (ext_source(E, x, y, z, c)) {
        const float* vc = c == 0 ? E.vel[0] : (c == 1 ? E.vel[1] : E.vel[2]);
        set3(v, c, vc[ext_face(E, c, x, y, z)]);
        set3(d, c, 0.0f);
        known |= 1u << c;
      } else if (touches_source(E, x, y, z, c)) {
        active |= 1u << c;
      }
    }
    v.w = float(known);
    d.w = float(active);
    E.val[0][i] = v;
    E.dist[0][i] = d;
    E.val[1][i] = v;
    E.dist[1][i] = d;
    E.mark[0][i] = ext_density(E, x, y, z) > 0.5f ? 1 : 0;
    active_total += __popc(active);
  }
  if (active_total) atomicAdd(&E.count[0], active_total);
}

// One axis of the band dilation: out = max of in over [-kBandReach, kBandReach] along the axis.
__global__ void k_ext_dilate(ExtDev E, int axis, const uint8_t* in, uint8_t* out) {
  EXT_FOR_CELLS(E, x, y, z, i) {
    const int p[3] = {x, y, z}, d[3] = {E.nx, E.ny, E.nz};
    const long long st = axis == 0 ? 1 : (axis == 1 ? E.nx : (long long)E.nx * E.ny);
    const int lo = max(0, p[axis] - kBandReach), hi = min(d[axis] - 1, p[axis] + kBandReach);
    uint8_t m = 0;
    for (int k = lo; k <= hi && !m; ++k) m = in[i + (k - p[axis]) * st];
    out[i] = m;
  }
}

// The band's node list: air cells near the liquid.  Each warp reserves one
// run of the list for its marked cells, in cell order, so a pass's loads stay
// coalesced (the order of the runs does not matter: a pass computes every node
// from the other side only).
__global__ void k_ext_band_list(ExtDev E, const uint8_t* mark) {
  EXT_FOR_CELLS(E, x, y, z, i) {
    const bool m = mark[i] && !(ext_density(E, x, y, z) > 0.5f);
    const unsigned act = __activemask();
    const unsigned bal = __ballot_sync(act, m);
    const int lane = threadIdx.x & 31, leader = __ffs(act) - 1;
    unsigned base = 0;
    if (lane == leader && bal) base = atomicAdd(&E.count[3], unsigned(__popc(bal)));
    base = __shfl_sync(act, base, leader);
    if (m) E.band[base + __popc(bal & ((1u << lane) - 1u))] = unsigned(i);
  }
}

__global__ void k_ext_reset(unsigned* count, int side) { count[side] = 0u; }

// updateActiveFront from side src to side 1 - src; a pass whose source side
// has no active component copies it (the reference's zero-size dispatch).
// SOLIDS: the lattice has embedded solids (E.solids); the instance without
// them carries none of their face and density tests.
template <bool SOLIDS>
__global__ void k_ext_update(ExtDev Ein, int src) {
  ExtDev E = Ein;
  E.solids = SOLIDS ? 1 : 0;
  const int dst = 1 - src;
  const bool run = E.count[src] != 0u;
  const ExtSrc S(E, src);
  unsigned active_total = 0;
  const unsigned nband = E.count[3];
  for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < nband; k += gridDim.x * blockDim.x) {
    const long long i = E.band[k];
    const int x = int(i % E.nx), y = int((i / E.nx) % E.ny), z = int(i / ((long long)E.nx * E.ny));
    float4 v = S.val[i], d = S.dist[i];
    if (run) {
      unsigned known = unsigned(v.w), active = unsigned(d.w);
      // A node is activated only next to a converging neighbour, and a
      // converging node is an active one: the components with no active
      // neighbour skip the activation test (same result, far fewer loads).
      unsigned near = 0;
      if (active != 7u) {
        if (x > 0) near |= unsigned(S.dist[i - 1].w);
        if (x + 1 < E.nx) near |= unsigned(S.dist[i + 1].w);
        if (y > 0) near |= unsigned(S.dist[i - E.nx].w);
        if (y + 1 < E.ny) near |= unsigned(S.dist[i + E.nx].w);
        const long long pl = (long long)E.nx * E.ny;
        if (z > 0) near |= unsigned(S.dist[i - pl].w);
        if (z + 1 < E.nz) near |= unsigned(S.dist[i + pl].w);
      }
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        if (!ext_open(E, x, y, z, c) || ext_source(E, x, y, z, c)) continue;
        if ((active >> c) & 1u) {
          const float old = at3(d, c);
          const float eps = S.eps(old);
          const float upd = fminf(old, S.godunov(x, y, z, c));
          const bool band = upd <= S.band;
          if (band) {
            set3(d, c, upd);
            set3(v, c, S.upwind(x, y, z, c, upd));
            known |= 1u << c;
          }
          const bool conv = old < 0.5f * kDistInf && fabsf(__fsub_rn(upd, old)) <= eps;
          active = (!conv && band) ? (active | (1u << c)) : (active & ~(1u << c));
        } else if (((near >> c) & 1u) && S.activated(x, y, z, c)) {
          active |= 1u << c;   // JRW07: a newly added point is updated from the next pass on
        }
      }
      v.w = float(known);
      d.w = float(active);
      active_total += __popc(active);
    }
    (dst ? E.val[1] : E.val[0])[i] = v;
    (dst ? E.dist[1] : E.dist[0])[i] = d;
  }
  if (active_total) atomicAdd(&E.count[dst], active_total);
}

// One level of the known-value hierarchy (values xyz, known mask w).
struct ExtLevel {
  int nx, ny, nz;
  const float4* src;   // restrict: the finer level; prolong: the coarser filled level
  int snx, sny, snz;
  const float4* keep;  // prolong: the target's own known values (restrict: null)
  float4* out;
};

// hierarchyComponentSample: renormalised trilinear interpolation of the
// source's known values at the target's face position (face-centred along c).
__device__ __forceinline__ float2 ext_sample(const ExtLevel& L, int tx, int ty, int tz, int c) {
  const int t[3] = {tx, ty, tz}, sd[3] = {L.snx, L.sny, L.snz}, td[3] = {L.nx, L.ny, L.nz};
  float sp[3];
  for (int a = 0; a < 3; ++a)
    sp[a] = a == c ? __fsub_rn(__fdiv_rn(__fmul_rn(float(t[a] + 1), float(sd[a])), float(td[a])), 1.0f)
                   : __fsub_rn(__fdiv_rn(__fmul_rn(__fadd_rn(float(t[a]), 0.5f), float(sd[a])), float(td[a])), 0.5f);
  int lo[3];
  float fr[3];
  for (int a = 0; a < 3; ++a) {
    const float f = floorf(sp[a]);
    lo[a] = int(f);
    fr[a] = __fsub_rn(sp[a], f);
  }
  float2 cb[8];
  for (int oz = 0; oz <= 1; ++oz)
    for (int oy = 0; oy <= 1; ++oy)
      for (int ox = 0; ox <= 1; ++ox) {
        const int o[3] = {ox, oy, oz};
        int q[3];
        float w[3];
        for (int a = 0; a < 3; ++a) {
          q[a] = min(max(lo[a] + o[a], 0), sd[a] - 1);
          w[a] = o[a] ? fr[a] : __fsub_rn(1.0f, fr[a]);
        }
        const float weight = __fmul_rn(__fmul_rn(w[0], w[1]), w[2]);
        const float4 s = L.src[q[0] + (long long)L.snx * (q[1] + (long long)L.sny * q[2])];
        const int corner = ox + 2 * oy + 4 * oz;
        cb[corner] = make_float2(0.f, 0.f);
        if (weight > 0.0f && has_bit(s.w, c)) cb[corner] = make_float2(__fmul_rn(weight, at3(s, c)), weight);
      }
  auto add = [](float2 a, float2 b) { return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y)); };
  const float2 y0 = add(add(cb[0], cb[5]), add(cb[1], cb[4]));
  const float2 y1 = add(add(cb[2], cb[7]), add(cb[3], cb[6]));
  const float2 s = add(y0, y1);
  return make_float2(s.y > 0.0f ? __fdiv_rn(s.x, s.y) : 0.0f, s.y);
}

// hierarchyCorrespondingCellSample (the y component's restriction fallback).
__device__ __forceinline__ float2 ext_cell_sample(const ExtLevel& L, int tx, int ty, int tz, int c) {
  auto known = [&](int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0 || x >= L.snx || y >= L.sny || z >= L.snz) return make_float2(0.f, 0.f);
    const float4 s = L.src[x + (long long)L.snx * (y + (long long)L.sny * z)];
    return has_bit(s.w, c) ? make_float2(at3(s, c), 1.0f) : make_float2(0.f, 0.f);
  };
  auto add = [](float2 a, float2 b) { return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y)); };
  const int lx = 2 * tx, ly = 2 * ty, lz = 2 * tz;
  float2 acc = make_float2(0.f, 0.f);
  for (int oy = 0; oy <= 1; ++oy) {
    const float2 c00 = known(lx, ly + oy, lz), c11 = known(lx + 1, ly + oy, lz + 1);
    const float2 c10 = known(lx + 1, ly + oy, lz), c01 = known(lx, ly + oy, lz + 1);
    acc = add(acc, add(add(c00, c11), add(c10, c01)));
  }
  return make_float2(acc.y > 0.0f ? __fdiv_rn(acc.x, acc.y) : 0.0f, acc.y);
}

// restrictKnownVelocity
__global__ void k_ext_restrict(ExtLevel L) {
  const long long n = (long long)L.nx * L.ny * L.nz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = int(i % L.nx), y = int((i / L.nx) % L.ny), z = int(i / ((long long)L.nx * L.ny));
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    unsigned known = 0;
    for (int c = 0; c < 3; ++c) {
      float2 r = ext_sample(L, x, y, z, c);
      if (r.y <= 0.0f && c == 1) r = ext_cell_sample(L, x, y, z, c);
      if (r.y > 0.0f) {
        set3(v, c, r.x);
        known |= 1u << c;
      }
    }
    v.w = float(known);
    L.out[i] = v;
  }
}

// prolongUnknownVelocity
__global__ void k_ext_prolong(ExtLevel L) {
  const long long n = (long long)L.nx * L.ny * L.nz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = int(i % L.nx), y = int((i / L.nx) % L.ny), z = int(i / ((long long)L.nx * L.ny));
    float4 v = L.keep[i];
    unsigned known = unsigned(v.w);
    for (int c = 0; c < 3; ++c) {
      if ((known >> c) & 1u) continue;
      const float2 r = ext_sample(L, x, y, z, c);
      if (r.y > 0.0f) {
        set3(v, c, r.x);
        known |= 1u << c;
      }
    }
    v.w = float(known);
    L.out[i] = v;
  }
}

// packTransportShell into the handle's MAC arrays: every open face takes its
// extrapolated value (0 where none is known); closed faces keep theirs.
__global__ void k_ext_pack(ExtDev E, const float4* state, unsigned* filled) {
  unsigned cnt = 0;
  EXT_FOR_CELLS(E, x, y, z, i) {
    const float4 s = state[i];
    for (int c = 0; c < 3; ++c) {
      if (!ext_open(E, x, y, z, c)) continue;
      const bool k = has_bit(s.w, c);
      E.vel[c][ext_face(E, c, x, y, z)] = k ? at3(s, c) : 0.0f;
      cnt += k;
    }
  }
  if (cnt) atomicAdd(filled, cnt);
}

}  // namespace fpp
