// CM12 conservative surface-density transport (Chentanez and Mueller 2012,
// Secs. 3.4-3.5; the step that produces the VOF the projection's labeller
// reads), replacing the dense uniform method's passes
// (lib/methods/uniform/webgpu-uniform-reference.ts:1150-1215 and
// webgpu-uniform-reference.wgsl.ts:640-858, 1187-1255; the paper algebra in
// lib/core/cm12-numerics.ts:47-149).
//
// Per step, one thread per cell in every pass:
//  1. k_tr_trace_beta: backward RK2 trace (at most 16 sub-steps, clamped to
//     the domain, a backward characteristic may leave through a released wall
//     face), the persistent gamma sampled there and conditioned, and each
//     donor's column sum beta scattered as 2^-20 fixed-point integers.
//  2. k_tr_deficit: donors with beta < 1 forward-trace and scatter the missing
//     column weight of density and gamma to their receivers.
//  3. k_tr_gather: rho' = sum of the conditioned row (gamma A_ij / max(1,
//     beta_j)) times the donors' density, plus the deficits; gamma' its row sum.
//  4. k_tr_diffuse: gamma diffusion (LAF11 Sec. 3.2), Jacobi along one axis
//     per launch, x -> y -> z per repetition, each launch reading one snapshot.
//  5. k_tr_sharpen, k_tr_sharpen_scatter, k_tr_sharpen_resolve: the cubic
//     sharpening weight on a Godunov gradient (Sec. 3.5), with the removed
//     mass carried along the density gradient up to D cells (half-cell steps,
//     at most 7) and deposited trilinearly.
// The fixed-point deposits are 32-bit integer atomics (order-independent).
// Every floating-point operation is written with round-to-nearest
// intrinsics in the reference's evaluation order, so the float restatement
// of the oracle reproduces the passes bit for bit.
//
// The velocity sampler reads the MAC arrays as the reference's transport
// shell (packTransportShell): open faces carry their (extrapolated) values,
// domain wall faces read 0; the released-face test reads the raw wall faces.
// Scope: walls and the authored open top; embedded solids, the inflow nozzle
// and dropped balls are not part of this step.
#pragma once

#include <cstdint>

namespace fpp {

constexpr float kTrFixed = 1048576.0f;       // CM12_TRANSPORT_FIXED_SCALE
constexpr float kTrGammaMin = 0.5f;          // CM12_GAMMA_INTERIOR_MIN
constexpr float kTrGammaMax = 2.5f;          // CM12_GAMMA_MAX
constexpr float kTrTau = 0.4f;               // CM12_SHARPENING_TAU
constexpr float kTrIso = 0.5f;               // CM12_LIQUID_ISOVALUE

struct TrDev {
  int nx, ny, nz, open_top;
  float h, dt;
  const float* u;   // [nz][ny][nx + 1]
  const float* v;   // [nz][ny + 1][nx]
  const float* w;   // [nz + 1][ny][nx]
  // The transport shell of each component (k_tr_shell): the face lattice with
  // face indices 0 .. d + 1 along the component's axis and cell indices
  // 0 .. d across it, walls and the outer layer 0, so the sampler's eight
  // corners need no bounds or wall tests (corners outside the lattice carry
  // weight 0 and read 0, as the reference's sampler sees them).
  float* sh[3];
};

__host__ __device__ inline long long tr_shell_sy(int nx, int c) { return c == 0 ? nx + 2 : nx + 1; }
__host__ __device__ inline long long tr_shell_sz(int nx, int ny, int c) {
  return tr_shell_sy(nx, c) * (c == 1 ? ny + 2 : ny + 1);
}
__host__ __device__ inline long long tr_shell_size(int nx, int ny, int nz, int c) {
  return tr_shell_sz(nx, ny, c) * (c == 2 ? nz + 2 : nz + 1);
}

struct TrV3 {
  float x, y, z;
};

__device__ __forceinline__ bool tr_valid(const TrDev& T, int x, int y, int z) {
  return x >= 0 && y >= 0 && z >= 0 && x < T.nx && y < T.ny && z < T.nz;
}
__device__ __forceinline__ long long tr_idx(const TrDev& T, int x, int y, int z) {
  return x + (long long)T.nx * (y + (long long)T.ny * z);
}
__device__ __forceinline__ float tr_face(const TrDev& T, int c, int x, int y, int z) {
  if (c == 0) return T.u[x + (long long)(T.nx + 1) * (y + (long long)T.ny * z)];
  if (c == 1) return T.v[x + (long long)T.nx * (y + (long long)(T.ny + 1) * z)];
  return T.w[x + (long long)T.nx * (y + (long long)T.ny * z)];
}
__device__ __forceinline__ float tr_clamp(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

// d4Sum8: ((t0 + t5) + (t1 + t4)) + ((t2 + t7) + (t3 + t6)).
__device__ __forceinline__ float tr_d4sum8(const float t[8]) {
  const float y0 = __fadd_rn(__fadd_rn(t[0], t[5]), __fadd_rn(t[1], t[4]));
  const float y1 = __fadd_rn(__fadd_rn(t[2], t[7]), __fadd_rn(t[3], t[6]));
  return __fadd_rn(y0, y1);
}

// i32(round(x)): round half to even, saturating (NaN gives 0).
__device__ __forceinline__ int tr_fix(float x) { return __float2int_rn(x); }

__device__ __forceinline__ float tr_corner_w(const TrV3& f, int k) {
  const float wx = (k & 1) ? f.x : __fsub_rn(1.0f, f.x);
  const float wy = (k & 2) ? f.y : __fsub_rn(1.0f, f.y);
  const float wz = (k & 4) ? f.z : __fsub_rn(1.0f, f.z);
  return __fmul_rn(__fmul_rn(wx, wy), wz);
}

// sampleVelocityComponent for the three components at once: trilinear over
// each component's face lattice, the query clamped to [-1, d - 1] along the
// component's axis (face coordinate, offset 1) and to [0, d - 1] across it
// (cell coordinate, offset 0.5).  The two coordinates of each axis are shared
// by the components, the arithmetic per component is the reference's; the
// corners are read from the transport shell.
__device__ TrV3 tr_sample(const TrDev& T, TrV3 p) {
  const int d[3] = {T.nx, T.ny, T.nz};
  const float pp[3] = {p.x, p.y, p.z};
  int bc[3], bf[3];
  float rc[3], rf[3], sc[3], sf[3];   // fractions and 1 - fractions
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float qc = tr_clamp(__fsub_rn(pp[a], 0.5f), 0.0f, float(d[a] - 1));
    const float qf = tr_clamp(__fsub_rn(pp[a], 1.0f), -1.0f, float(d[a] - 1));
    const float fc = floorf(qc), ff = floorf(qf);
    bc[a] = int(fc);
    bf[a] = int(ff);
    rc[a] = __fsub_rn(qc, fc);
    rf[a] = __fsub_rn(qf, ff);
    sc[a] = __fsub_rn(1.0f, rc[a]);
    sf[a] = __fsub_rn(1.0f, rf[a]);
  }
  float out[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const long long sy = tr_shell_sy(T.nx, c), sz = tr_shell_sz(T.nx, T.ny, c);
    const int b0 = c == 0 ? bf[0] + 1 : bc[0], b1 = c == 1 ? bf[1] + 1 : bc[1], b2 = c == 2 ? bf[2] + 1 : bc[2];
    const float r0 = c == 0 ? rf[0] : rc[0], r1 = c == 1 ? rf[1] : rc[1], r2 = c == 2 ? rf[2] : rc[2];
    const float s0 = c == 0 ? sf[0] : sc[0], s1 = c == 1 ? sf[1] : sc[1], s2 = c == 2 ? sf[2] : sc[2];
    const float* q = T.sh[c] + (b0 + sy * b1 + sz * b2);
    float t[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int o0 = k & 1, o1 = (k >> 1) & 1, o2 = (k >> 2) & 1;
      const float w = __fmul_rn(__fmul_rn(o0 ? r0 : s0, o1 ? r1 : s1), o2 ? r2 : s2);
      t[k] = __fmul_rn(w, q[o0 + sy * o1 + sz * o2]);
    }
    out[c] = tr_d4sum8(t);
  }
  return TrV3{out[0], out[1], out[2]};
}

__device__ __forceinline__ TrV3 tr_clamp_trace(const TrDev& T, TrV3 p) {
  TrV3 q = p;
  q.x = tr_clamp(q.x, 0.5f, __fsub_rn(float(T.nx), 0.5f));
  q.z = tr_clamp(q.z, 0.5f, __fsub_rn(float(T.nz), 0.5f));
  q.y = fmaxf(q.y, 0.5f);
  if (!T.open_top) q.y = fminf(q.y, __fsub_rn(float(T.ny), 0.5f));
  return q;
}

__device__ __forceinline__ bool tr_exits_released(const TrDev& T, TrV3 p) {
  const int qx = min(max(int(floorf(p.x)), 0), T.nx - 1);
  const int qy = min(max(int(floorf(p.y)), 0), T.ny - 1);
  const int qz = min(max(int(floorf(p.z)), 0), T.nz - 1);
  if (p.x < 0.5f) return tr_face(T, 0, 0, qy, qz) > 1e-6f;
  if (p.x > __fsub_rn(float(T.nx), 0.5f)) return tr_face(T, 0, T.nx, qy, qz) < -1e-6f;
  if (p.y < 0.5f) return tr_face(T, 1, qx, 0, qz) > 1e-6f;
  if (p.y > __fsub_rn(float(T.ny), 0.5f)) return tr_face(T, 1, qx, T.ny, qz) < -1e-6f;
  if (p.z < 0.5f) return tr_face(T, 2, qx, qy, 0) > 1e-6f;
  if (p.z > __fsub_rn(float(T.nz), 0.5f)) return tr_face(T, 2, qx, qy, T.nz) < -1e-6f;
  return false;
}

__device__ __forceinline__ float tr_length(TrV3 v) {
  return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y)), __fmul_rn(v.z, v.z)));
}

// integrateTraceOffset: the trace from the cell centre, minus the centre.
__device__ TrV3 tr_trace(const TrDev& T, int x, int y, int z, float dir) {
  const TrV3 pos{__fadd_rn(float(x), 0.5f), __fadd_rn(float(y), 0.5f), __fadd_rn(float(z), 0.5f)};
  const float h = T.h, dt = T.dt;
  const TrV3 v0 = tr_sample(T, pos);   // also the first sub-step's start sample (same point)
  const float steps_f = ceilf(__fdiv_rn(__fmul_rn(tr_length(v0), dt), h));
  int steps = steps_f >= 16.0f ? 16 : int(steps_f);
  if (steps < 1) steps = 1;
  const float sdt = __fdiv_rn(dt, float(steps));
  const float half = __fmul_rn(dir, 0.5f);
  TrV3 p = pos;
  for (int s = 0; s < steps; ++s) {
    const TrV3 a = s == 0 ? v0 : tr_sample(T, p);
    const TrV3 mid = tr_clamp_trace(T, TrV3{__fadd_rn(p.x, __fdiv_rn(__fmul_rn(__fmul_rn(half, a.x), sdt), h)),
                                            __fadd_rn(p.y, __fdiv_rn(__fmul_rn(__fmul_rn(half, a.y), sdt), h)),
                                            __fadd_rn(p.z, __fdiv_rn(__fmul_rn(__fmul_rn(half, a.z), sdt), h))});
    const TrV3 b = tr_sample(T, mid);
    const TrV3 cand{__fadd_rn(p.x, __fdiv_rn(__fmul_rn(__fmul_rn(dir, b.x), sdt), h)),
                    __fadd_rn(p.y, __fdiv_rn(__fmul_rn(__fmul_rn(dir, b.y), sdt), h)),
                    __fadd_rn(p.z, __fdiv_rn(__fmul_rn(__fmul_rn(dir, b.z), sdt), h))};
    if (dir < 0.0f && tr_exits_released(T, cand)) {
      p = cand;
      break;
    }
    p = tr_clamp_trace(T, cand);
  }
  return TrV3{__fsub_rn(p.x, pos.x), __fsub_rn(p.y, pos.y), __fsub_rn(p.z, pos.z)};
}

// The 2 x 2 x 2 stencil at the traced point: base corner, fractions,
// transportStencilWeight per corner (0 outside the lattice) and their
// sequential sum.
struct TrStencil {
  int bx, by, bz;
  float w[8];
  float total;
};

__device__ __forceinline__ TrStencil tr_stencil(const TrDev& T, int x, int y, int z, TrV3 tr) {
  TrStencil S;
  const float fx = floorf(tr.x), fy = floorf(tr.y), fz = floorf(tr.z);
  S.bx = x + int(fx);
  S.by = y + int(fy);
  S.bz = z + int(fz);
  const TrV3 f{__fsub_rn(tr.x, fx), __fsub_rn(tr.y, fy), __fsub_rn(tr.z, fz)};
  S.total = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const bool in = tr_valid(T, S.bx + (k & 1), S.by + ((k >> 1) & 1), S.bz + ((k >> 2) & 1));
    S.w[k] = in ? tr_corner_w(f, k) : 0.0f;
    S.total = __fadd_rn(S.total, S.w[k]);
  }
  return S;
}

__device__ __forceinline__ long long tr_corner(const TrDev& T, const TrStencil& S, int k) {
  return tr_idx(T, S.bx + (k & 1), S.by + ((k >> 1) & 1), S.bz + ((k >> 2) & 1));
}

#define TR_CELLS(T)                                                                                \
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x,                          \
                 n_ = (long long)(T).nx * (T).ny * (T).nz;                                       \
       i < n_; i += (long long)gridDim.x * blockDim.x)

// The transport shells of the three components from the MAC arrays, in one
// launch over their concatenation: face F along the component's axis
// (0 .. d + 1), cells across (0 .. d); F = 0, F = d (a wall unless it is the
// open top) and every index past the lattice hold 0.
__global__ void k_tr_shells(TrDev T, float* __restrict__ s0, float* __restrict__ s1, float* __restrict__ s2) {
  const long long n0 = tr_shell_size(T.nx, T.ny, T.nz, 0), n1 = tr_shell_size(T.nx, T.ny, T.nz, 1);
  const long long total = n0 + n1 + tr_shell_size(T.nx, T.ny, T.nz, 2);
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total; g += (long long)gridDim.x * blockDim.x) {
    const int c = g < n0 ? 0 : (g < n0 + n1 ? 1 : 2);
    const long long i = c == 0 ? g : (c == 1 ? g - n0 : g - n0 - n1);
    float* out = c == 0 ? s0 : (c == 1 ? s1 : s2);
    const long long sy = tr_shell_sy(T.nx, c), sz = tr_shell_sz(T.nx, T.ny, c);
    const int wall_hi = (c == 1 && T.open_top) ? -1 : (c == 0 ? T.nx : (c == 1 ? T.ny : T.nz));
    const int iz = int(i / sz), iy = int((i / sy) % (sz / sy)), ix = int(i % sy);
    const int ic = c == 0 ? ix : (c == 1 ? iy : iz), dc = c == 0 ? T.nx : (c == 1 ? T.ny : T.nz);
    const bool across = (c != 0 && ix >= T.nx) || (c != 1 && iy >= T.ny) || (c != 2 && iz >= T.nz);
    const bool zero = across || ic == 0 || ic == wall_hi || ic > dc;
    out[i] = zero ? 0.0f : tr_face(T, c, ix, iy, iz);
  }
}

// Steps 1-3 of CM12 Sec. 3.4: gamma~ at the departure point (conditioned),
// beta_j += gamma~_i w_ij / sum w.
// The backward offset is kept (trace[3 i ..]) for the gather, which would
// compute the same bits again.
__global__ void k_tr_trace_beta(TrDev T, const float* __restrict__ gam, float* __restrict__ gam_adv, int* beta,
                                float* __restrict__ trace) {
  TR_CELLS(T) {
    const int x = int(i % T.nx), y = int((i / T.nx) % T.ny), z = int(i / ((long long)T.nx * T.ny));
    const TrV3 tr = tr_trace(T, x, y, z, -1.0f);
    trace[3 * i] = tr.x;
    trace[3 * i + 1] = tr.y;
    trace[3 * i + 2] = tr.z;
    const TrStencil S = tr_stencil(T, x, y, z, tr);
    float t[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) t[k] = S.w[k] > 0.0f ? __fmul_rn(S.w[k], gam[tr_corner(T, S, k)]) : 0.0f;
    const float sg = tr_d4sum8(t);
    const float g = S.total >= 0.999999f ? fminf(kTrGammaMax, fmaxf(kTrGammaMin, sg)) : fminf(sg, kTrGammaMax);
    gam_adv[i] = g;
    if (S.total <= 1e-9f) continue;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const float wk = __fdiv_rn(S.w[k], S.total);
      if (wk > 0.0f) atomicAdd(&beta[tr_corner(T, S, k)], tr_fix(__fmul_rn(__fmul_rn(g, wk), kTrFixed)));
    }
  }
}

// Steps 6-7: donors with beta < 1 forward-scatter the missing column weight
// of density and of the pre-advection gamma.
__global__ void k_tr_deficit(TrDev T, const float* __restrict__ rho, const float* __restrict__ gam,
                             const int* __restrict__ beta, int* dep_rho, int* dep_gam) {
  TR_CELLS(T) {
    const float deficit = fmaxf(0.0f, __fsub_rn(1.0f, __fdiv_rn(float(beta[i]), kTrFixed)));
    if (deficit <= 1.0f / kTrFixed) continue;
    const int x = int(i % T.nx), y = int((i / T.nx) % T.ny), z = int(i / ((long long)T.nx * T.ny));
    const TrStencil S = tr_stencil(T, x, y, z, tr_trace(T, x, y, z, 1.0f));
    const float rd = __fmul_rn(rho[i], deficit), gd = __fmul_rn(gam[i], deficit);
    if (S.total <= 1e-9f) {
      atomicAdd(&dep_rho[i], tr_fix(__fmul_rn(rd, kTrFixed)));
      atomicAdd(&dep_gam[i], tr_fix(__fmul_rn(gd, kTrFixed)));
      continue;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const float wk = __fdiv_rn(S.w[k], S.total);
      if (wk <= 0.0f) continue;
      const long long r = tr_corner(T, S, k);
      atomicAdd(&dep_rho[r], tr_fix(__fmul_rn(__fmul_rn(rd, wk), kTrFixed)));
      atomicAdd(&dep_gam[r], tr_fix(__fmul_rn(__fmul_rn(gd, wk), kTrFixed)));
    }
  }
}

// Steps 4-5 and the resolve of 6-7.
__global__ void k_tr_gather(TrDev T, const float* __restrict__ rho, const float* __restrict__ gam_adv,
                            const int* __restrict__ beta, const int* __restrict__ dep_rho,
                            const int* __restrict__ dep_gam, const float* __restrict__ trace,
                            float* __restrict__ rho_out, float* __restrict__ gam_out) {
  TR_CELLS(T) {
    const int x = int(i % T.nx), y = int((i / T.nx) % T.ny), z = int(i / ((long long)T.nx * T.ny));
    const TrStencil S = tr_stencil(T, x, y, z, TrV3{trace[3 * i], trace[3 * i + 1], trace[3 * i + 2]});
    const float g = gam_adv[i];
    float rn = 0.0f, gn = 0.0f;
    if (S.total > 1e-9f) {
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const float wk = __fdiv_rn(S.w[k], S.total);
        if (wk <= 0.0f) continue;
        const long long j = tr_corner(T, S, k);
        const float bj = __fdiv_rn(float(beta[j]), kTrFixed);
        const float sc = __fdiv_rn(__fmul_rn(g, wk), fmaxf(1.0f, bj));
        rn = __fadd_rn(rn, __fmul_rn(sc, rho[j]));
        gn = __fadd_rn(gn, sc);
      }
    }
    rn = __fadd_rn(rn, __fdiv_rn(float(dep_rho[i]), kTrFixed));
    gn = __fadd_rn(gn, __fdiv_rn(float(dep_gam[i]), kTrFixed));
    if (rn < 1e-5f) gn = 1.0f;
    rho_out[i] = fmaxf(rn, 0.0f);
    gam_out[i] = fmaxf(gn, 0.0f);
  }
}

// cm12GammaDiffusionFluxInto for one face (open 1 between two cells).
__device__ __forceinline__ void tr_flux(float orho, float og, float nrho, float ng, float& fr, float& fg) {
  fg = __fmul_rn(0.5f, __fsub_rn(ng, og));   // 0.5 * open with open = 1
  fr = 0.0f;
  if (ng > og) {
    fr = __fdiv_rn(__fmul_rn(nrho, __fsub_rn(ng, og)), __fmul_rn(2.0f, fmaxf(ng, 1e-9f)));
  } else if (og > ng) {
    fr = __fdiv_rn(__fmul_rn(-orho, __fsub_rn(og, ng)), __fmul_rn(2.0f, fmaxf(og, 1e-9f)));
  }
}

// diffuseGammaAxis: both face fluxes from one snapshot.
__global__ void k_tr_diffuse(TrDev T, int axis, const float* __restrict__ rho, const float* __restrict__ gam,
                             float* __restrict__ rho_out, float* __restrict__ gam_out) {
  const int ex = axis == 0, ey = axis == 1, ez = axis == 2;
  TR_CELLS(T) {
    const int x = int(i % T.nx), y = int((i / T.nx) % T.ny), z = int(i / ((long long)T.nx * T.ny));
    const float orho = rho[i], og = gam[i];
    float dr = 0.0f, dg = 0.0f, fr, fg;
    if (tr_valid(T, x - ex, y - ey, z - ez)) {
      const long long j = tr_idx(T, x - ex, y - ey, z - ez);
      tr_flux(orho, og, rho[j], gam[j], fr, fg);
      dr = __fadd_rn(dr, fr);
      dg = __fadd_rn(dg, fg);
    }
    if (tr_valid(T, x + ex, y + ey, z + ez)) {
      const long long j = tr_idx(T, x + ex, y + ey, z + ez);
      tr_flux(orho, og, rho[j], gam[j], fr, fg);
      dr = __fadd_rn(dr, fr);
      dg = __fadd_rn(dg, fg);
    }
    rho_out[i] = __fadd_rn(orho, dr);
    gam_out[i] = __fadd_rn(og, dg);
  }
}

__device__ __forceinline__ float tr_vol(const TrDev& T, const float* rho, int x, int y, int z) {
  return tr_valid(T, x, y, z) ? rho[tr_idx(T, x, y, z)] : 0.0f;
}

// faceOpenFraction without embedded solids: 1 between two cells and on the
// authored open top, 0 on the other walls.
__device__ __forceinline__ float tr_face_open(const TrDev& T, int x, int y, int z, int axis) {
  const bool in = tr_valid(T, x, y, z);
  if (!in || !tr_valid(T, x + (axis == 0), y + (axis == 1), z + (axis == 2)))
    return (axis == 1 && in && y == T.ny - 1 && T.open_top) ? 1.0f : 0.0f;
  return 1.0f;
}

// sharpenDeltaRho + sharpenCompute: rho_s = rho + delta, delta kept.
__global__ void k_tr_sharpen(TrDev T, const float* __restrict__ rho, float strength, float* __restrict__ rho_s,
                             float* __restrict__ delta, unsigned* __restrict__ lost, unsigned* nlost) {
  const float dT = __fmul_rn(__fmul_rn(3.0f, T.dt), strength);
  TR_CELLS(T) {
    const int x = int(i % T.nx), y = int((i / T.nx) % T.ny), z = int(i / ((long long)T.nx * T.ny));
    const float r = rho[i];
    float plus[3], minus[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int ex = a == 0, ey = a == 1, ez = a == 2;
      const float op = fmaxf(tr_face_open(T, x, y, z, a), 0.0f);
      const float om = fmaxf(tr_face_open(T, x - ex, y - ey, z - ez, a), 0.0f);
      const float sp = __fdiv_rn(
          __fmul_rn(-__fsub_rn(__fmul_rn(r, op), __fmul_rn(tr_vol(T, rho, x - ex, y - ey, z - ez), om)), dT), T.h);
      const float sm = __fdiv_rn(
          __fmul_rn(-__fsub_rn(__fmul_rn(tr_vol(T, rho, x + ex, y + ey, z + ez), op), __fmul_rn(r, om)), dT), T.h);
      plus[a] = fmaxf(__fmul_rn(fmaxf(sp, 0.0f), fmaxf(sp, 0.0f)), __fmul_rn(fminf(sm, 0.0f), fminf(sm, 0.0f)));
      minus[a] = fmaxf(__fmul_rn(fminf(sp, 0.0f), fminf(sp, 0.0f)), __fmul_rn(fmaxf(sm, 0.0f), fmaxf(sm, 0.0f)));
    }
    const float gp = __fsqrt_rn(__fadd_rn(__fadd_rn(plus[0], plus[2]), plus[1]));
    const float gm = __fsqrt_rn(__fadd_rn(__fadd_rn(minus[0], minus[2]), minus[1]));
    float md = 0.0f;
    md = fmaxf(md, fabsf(__fsub_rn(r, tr_vol(T, rho, x - 1, y, z))));
    md = fmaxf(md, fabsf(__fsub_rn(r, tr_vol(T, rho, x + 1, y, z))));
    md = fmaxf(md, fabsf(__fsub_rn(r, tr_vol(T, rho, x, y - 1, z))));
    md = fmaxf(md, fabsf(__fsub_rn(r, tr_vol(T, rho, x, y + 1, z))));
    md = fmaxf(md, fabsf(__fsub_rn(r, tr_vol(T, rho, x, y, z - 1))));
    md = fmaxf(md, fabsf(__fsub_rn(r, tr_vol(T, rho, x, y, z + 1))));
    const float d = __fsub_rn(r, kTrIso);
    const float wgt = __fmul_rn(__fmul_rn(__fmul_rn(d, d), d), __fsub_rn(1.0f, fminf(1.0f, __fdiv_rn(md, kTrTau))));
    float dr = wgt >= 0.0f ? __fmul_rn(wgt, gp) : __fmul_rn(wgt, gm);
    if (__fadd_rn(r, dr) < 0.0f || r < 1e-5f) dr = -r;
    else if (r > 0.5f) dr = 0.0f;
    rho_s[i] = __fadd_rn(r, dr);
    delta[i] = dr;
    if (lost) {   // the cells whose mass the scatter carries, one run of the list per warp
      const unsigned act = __activemask();
      const unsigned bal = __ballot_sync(act, dr < 0.0f);
      const int lane = threadIdx.x & 31, leader = __ffs(act) - 1;
      unsigned base = 0;
      if (lane == leader && bal) base = atomicAdd(nlost, unsigned(__popc(bal)));
      base = __shfl_sync(act, base, leader);
      if (dr < 0.0f) lost[base + __popc(bal & ((1u << lane) - 1u))] = unsigned(i);
    }
  }
}

__device__ float tr_sample_volume(const TrDev& T, const float* rho, TrV3 p) {
  const float qx = __fsub_rn(p.x, 0.5f), qy = __fsub_rn(p.y, 0.5f), qz = __fsub_rn(p.z, 0.5f);
  const float fx = floorf(qx), fy = floorf(qy), fz = floorf(qz);
  const int bx = int(fx), by = int(fy), bz = int(fz);
  const TrV3 f{__fsub_rn(qx, fx), __fsub_rn(qy, fy), __fsub_rn(qz, fz)};
  float t[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int X = bx + (k & 1), Y = by + ((k >> 1) & 1), Z = bz + ((k >> 2) & 1);
    t[k] = tr_valid(T, X, Y, Z) ? __fmul_rn(tr_corner_w(f, k), rho[tr_idx(T, X, Y, Z)]) : 0.0f;
  }
  return tr_d4sum8(t);
}

// sharpenScatter: a cell that lost density carries it along the (sharpened)
// density gradient towards the 0.5 contour and deposits it trilinearly.
__global__ void k_tr_sharpen_scatter(TrDev T, const float* __restrict__ delta, const float* __restrict__ rho_s,
                                     float max_dist, const unsigned* __restrict__ lost, const unsigned* nlost, int* dep) {
  const float h2 = __fmul_rn(2.0f, T.h);
  const unsigned m = *nlost;
  for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
    const long long i = lost[k];
    const float dr = delta[i];
    const int x = int(i % T.nx), y = int((i / T.nx) % T.ny), z = int(i / ((long long)T.nx * T.ny));
    TrV3 p{__fadd_rn(float(x), 0.5f), __fadd_rn(float(y), 0.5f), __fadd_rn(float(z), 0.5f)};
    float travelled = 0.0f;
    for (int st = 0; st < 7; ++st) {
      if (tr_sample_volume(T, rho_s, p) >= 0.5f || travelled >= max_dist) break;
      const int cx = int(floorf(p.x)), cy = int(floorf(p.y)), cz = int(floorf(p.z));
      const TrV3 g{__fdiv_rn(__fsub_rn(tr_vol(T, rho_s, cx + 1, cy, cz), tr_vol(T, rho_s, cx - 1, cy, cz)), h2),
                   __fdiv_rn(__fsub_rn(tr_vol(T, rho_s, cx, cy + 1, cz), tr_vol(T, rho_s, cx, cy - 1, cz)), h2),
                   __fdiv_rn(__fsub_rn(tr_vol(T, rho_s, cx, cy, cz + 1), tr_vol(T, rho_s, cx, cy, cz - 1)), h2)};
      const float mag = tr_length(g);
      if (mag < 1e-6f) break;
      const float dist = fminf(0.5f, __fsub_rn(max_dist, travelled));
      p = TrV3{__fadd_rn(p.x, __fmul_rn(__fdiv_rn(g.x, mag), dist)), __fadd_rn(p.y, __fmul_rn(__fdiv_rn(g.y, mag), dist)),
               __fadd_rn(p.z, __fmul_rn(__fdiv_rn(g.z, mag), dist))};
      travelled = __fadd_rn(travelled, dist);
      if (tr_sample_volume(T, rho_s, p) >= 0.5f) break;
    }
    const float ax = __fsub_rn(p.x, 0.5f), ay = __fsub_rn(p.y, 0.5f), az = __fsub_rn(p.z, 0.5f);
    const float fx = floorf(ax), fy = floorf(ay), fz = floorf(az);
    const int cx = int(fx), cy = int(fy), cz = int(fz);
    const TrV3 f{__fsub_rn(ax, fx), __fsub_rn(ay, fy), __fsub_rn(az, fz)};
    float wk[8], total = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      wk[k] = tr_valid(T, cx + (k & 1), cy + ((k >> 1) & 1), cz + ((k >> 2) & 1)) ? tr_corner_w(f, k) : 0.0f;
      total = __fadd_rn(total, wk[k]);
    }
    if (total <= 1e-8f) {
      atomicAdd(&dep[i], tr_fix(__fmul_rn(-dr, kTrFixed)));
      continue;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (wk[k] <= 0.0f) continue;
      atomicAdd(&dep[tr_idx(T, cx + (k & 1), cy + ((k >> 1) & 1), cz + ((k >> 2) & 1))],
                tr_fix(__fmul_rn(__fdiv_rn(__fmul_rn(-dr, wk[k]), total), kTrFixed)));
    }
  }
}

__global__ void k_tr_sharpen_resolve(TrDev T, const float* __restrict__ rho_s, const int* __restrict__ dep,
                                     float* __restrict__ rho_out) {
  TR_CELLS(T) { rho_out[i] = __fadd_rn(rho_s[i], __fdiv_rn(float(dep[i]), kTrFixed)); }
}

// Mass receipt: per-CTA float64 sums and min / max of rho in a fixed tree,
// folded by one CTA in CTA order (the same bits for every launch).
constexpr int kTrMassGrid = 1184;

__global__ void __launch_bounds__(256) k_tr_mass_part(const float* __restrict__ rho, long long n, double* part) {
  __shared__ double ss[256];
  __shared__ float smin[256], smax[256];
  double s = 0.0;
  float mn = 3.402823e38f, mx = -3.402823e38f;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += 256LL * gridDim.x) {
    const float r = rho[i];
    s += double(r);
    mn = fminf(mn, r);
    mx = fmaxf(mx, r);
  }
  ss[threadIdx.x] = s;
  smin[threadIdx.x] = mn;
  smax[threadIdx.x] = mx;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (int(threadIdx.x) < o) {
      ss[threadIdx.x] += ss[threadIdx.x + o];
      smin[threadIdx.x] = fminf(smin[threadIdx.x], smin[threadIdx.x + o]);
      smax[threadIdx.x] = fmaxf(smax[threadIdx.x], smax[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x] = ss[0];
    part[3 * blockIdx.x + 1] = double(smin[0]);
    part[3 * blockIdx.x + 2] = double(smax[0]);
  }
}

// One CTA of 256 threads: thread t folds partials t, t + 256, ... in order,
// then a fixed shared-memory tree.
__global__ void __launch_bounds__(256) k_tr_mass_fold(const double* part, int parts, double* out) {
  __shared__ double ss[256], smin[256], smax[256];
  double s = 0.0, mn = 3.402823e38, mx = -3.402823e38;
  for (int b = threadIdx.x; b < parts; b += 256) {
    s += part[3 * b];
    mn = fmin(mn, part[3 * b + 1]);
    mx = fmax(mx, part[3 * b + 2]);
  }
  ss[threadIdx.x] = s;
  smin[threadIdx.x] = mn;
  smax[threadIdx.x] = mx;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (int(threadIdx.x) < o) {
      ss[threadIdx.x] += ss[threadIdx.x + o];
      smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + o]);
      smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = ss[0];
    out[1] = smin[0];
    out[2] = smax[0];
  }
}

__global__ void k_tr_fill(float* p, long long n, float v) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = v;
}

#undef TR_CELLS

}  // namespace fpp
