// CPU oracle of the CM12 conservative surface-density transport step (test
// infrastructure only: tests/, the smoke check and the bench's CPU baseline
// leg call it, nothing in the product does).  A float32 restatement, in the
// device kernels' operation order, of the reference's dense uniform method:
//
//   lib/methods/uniform/webgpu-uniform-reference.ts:1150-1215  pass sequence
//     (trace gamma and beta, scatter deficits, gather, gamma diffusion x -> y
//     -> z Jacobi repetitions, sharpening with its local mass return)
//   lib/methods/uniform/webgpu-uniform-reference.wgsl.ts
//     :97-112     valid, d4Sum8 (fixed add order of 8 corner terms)
//     :252-271    sampleVolume, sampleVelocityComponent (MAC faces, clamped)
//     :606-626    normalVolume, volumeGradient, betaValue
//     :640-699    clampTraceToDomain, backwardTraceExitsReleasedFace,
//                 integrateTraceOffset (RK2 sub-steps, at most 16),
//                 densityTransportDestination, transportStencilWeight
//     :702-790    sampleGammaStencil, traceGammaAndBeta,
//                 scatterDensityDeficit, gatherConservativeDensity
//     :796-842    gammaDiffusionFaceOpen, diffuseGammaAxis
//     :1187-1255  sharpenDeltaRho, sharpenCompute, sharpenScatter,
//                 sharpenResolve
//   lib/core/cm12-numerics.ts:15-31, 47-149  constants, cm12ConditionedGamma,
//     cm12ConditionedRowCoefficient, cm12VolumeWeightedBetaContribution,
//     cm12VolumeScaledDeficitTransfer, cm12GammaDiffusionFluxInto,
//     cm12SharpeningWeight
//
// The velocity sampler reads the transport shell (packTransportShell,
// webgpu-uniform-velocity-extrapolation.wgsl.ts:498-514): the open faces'
// values, 0 on the domain walls; the released-face test reads the raw wall
// faces.
// Scope: the domain walls and the authored open top; no embedded solids,
// inflow nozzle or dropped balls (their source terms are zero).  The MAC
// arrays are the face layouts u [nz][ny][nx+1], v [nz][ny+1][nx],
// w [nz+1][ny][nx]: face F of an axis sits between cells F - 1 and F, which
// is the reference's padded transport texture along that axis.  The
// fixed-point deposits are 32-bit integers (round half to even, wrapping
// adds), so their sums do not depend on order.  Parity with the reference's
// own GPU path is unpinned: its WebGPU runtime cannot run here.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr float kFixed = 1048576.0f;        // CM12_TRANSPORT_FIXED_SCALE
constexpr float kGammaInteriorMin = 0.5f;   // CM12_GAMMA_INTERIOR_MIN
constexpr float kGammaMax = 2.5f;           // CM12_GAMMA_MAX
constexpr float kTau = 0.4f;                // CM12_SHARPENING_TAU
constexpr float kIso = 0.5f;                // CM12_LIQUID_ISOVALUE

struct V3 {
  float x, y, z;
};

struct Grid {
  int nx, ny, nz;
  float h, dt;
  int open_top;
  const float* u;
  const float* v;
  const float* w;
  bool valid(int x, int y, int z) const { return x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz; }
  long idx(int x, int y, int z) const { return x + (long)nx * (y + (long)ny * z); }
  // MAC face of axis c at face coordinate (fx, fy, fz); the axis coordinate is
  // a face index, the others cell indices.
  float face(int c, int x, int y, int z) const {
    if (c == 0) return u[x + (long)(nx + 1) * (y + (long)ny * z)];
    if (c == 1) return v[x + (long)nx * (y + (long)(ny + 1) * z)];
    return w[x + (long)nx * (y + (long)ny * z)];
  }
};

inline float get(const V3& a, int c) { return c == 0 ? a.x : (c == 1 ? a.y : a.z); }
inline float clampf(float v, float lo, float hi) { return std::fmin(std::fmax(v, lo), hi); }

// d4Sum8: ((t0 + t5) + (t1 + t4)) + ((t2 + t7) + (t3 + t6)).
inline float d4sum8(const float t[8]) {
  const float y0 = (t[0] + t[5]) + (t[1] + t[4]);
  const float y1 = (t[2] + t[7]) + (t[3] + t[6]);
  return y0 + y1;
}

// i32(round(x)): round half to even, saturating.
inline int32_t fix_round(float x) {
  const float r = std::nearbyint(x);
  if (!(r == r)) return 0;
  if (r >= 2147483648.0f) return INT32_MAX;
  if (r < -2147483648.0f) return INT32_MIN;
  return int32_t(r);
}
inline void wrap_add(int32_t& a, int32_t v) { a = int32_t(uint32_t(a) + uint32_t(v)); }

// Trilinear corner weight ((wx wy) wz) of corner k (bit 0 x, 1 y, 2 z).
inline float corner_w(const V3& f, int k) {
  const float wx = (k & 1) ? f.x : 1.0f - f.x;
  const float wy = (k & 2) ? f.y : 1.0f - f.y;
  const float wz = (k & 4) ? f.z : 1.0f - f.z;
  return (wx * wy) * wz;
}

float sample_velocity_c(const Grid& G, V3 p, int c) {
  const float off[3] = {c == 0 ? 1.0f : 0.5f, c == 1 ? 1.0f : 0.5f, c == 2 ? 1.0f : 0.5f};
  const float lo[3] = {c == 0 ? -1.0f : 0.0f, c == 1 ? -1.0f : 0.0f, c == 2 ? -1.0f : 0.0f};
  const int d[3] = {G.nx, G.ny, G.nz};
  float q[3];
  const float pp[3] = {p.x, p.y, p.z};
  int base[3];
  float fr[3];
  for (int a = 0; a < 3; ++a) {
    q[a] = clampf(pp[a] - off[a], lo[a], float(d[a] - 1));
    const float fl = std::floor(q[a]);
    base[a] = int(fl);
    fr[a] = q[a] - fl;
  }
  float t[8];
  for (int k = 0; k < 8; ++k) {
    const int o[3] = {k & 1, (k >> 1) & 1, (k >> 2) & 1};
    const float wx = o[0] ? fr[0] : 1.0f - fr[0];
    const float wy = o[1] ? fr[1] : 1.0f - fr[1];
    const float wz = o[2] ? fr[2] : 1.0f - fr[2];
    int ix[3];
    bool in = true;
    for (int a = 0; a < 3; ++a) {
      ix[a] = base[a] + o[a] + (a == c ? 1 : 0);   // face index on the axis, cell index across
      const int hi = a == c ? d[a] : d[a] - 1;
      if (ix[a] < 0 || ix[a] > hi) in = false;
    }
    // the transport shell holds the open faces only: wall faces read 0
    const bool wall = ix[c] == 0 || (ix[c] == d[c] && !(c == 1 && G.open_top));
    const float val = in && !wall ? G.face(c, ix[0], ix[1], ix[2]) : 0.0f;
    t[k] = ((wx * wy) * wz) * val;
  }
  return d4sum8(t);
}

V3 sample_velocity(const Grid& G, V3 p) {
  return V3{sample_velocity_c(G, p, 0), sample_velocity_c(G, p, 1), sample_velocity_c(G, p, 2)};
}

V3 clamp_trace(const Grid& G, V3 p) {
  V3 q = p;
  q.x = clampf(q.x, 0.5f, float(G.nx) - 0.5f);
  q.z = clampf(q.z, 0.5f, float(G.nz) - 0.5f);
  q.y = std::fmax(q.y, 0.5f);
  if (!G.open_top) q.y = std::fmin(q.y, float(G.ny) - 0.5f);
  return q;
}

// backwardTraceExitsReleasedFace: a departure beyond a wall whose face
// velocity points into the domain.
bool exits_released(const Grid& G, V3 p) {
  const int qx = std::min(std::max(int(std::floor(p.x)), 0), G.nx - 1);
  const int qy = std::min(std::max(int(std::floor(p.y)), 0), G.ny - 1);
  const int qz = std::min(std::max(int(std::floor(p.z)), 0), G.nz - 1);
  if (p.x < 0.5f) return G.face(0, 0, qy, qz) > 1e-6f;
  if (p.x > float(G.nx) - 0.5f) return G.face(0, G.nx, qy, qz) < -1e-6f;
  if (p.y < 0.5f) return G.face(1, qx, 0, qz) > 1e-6f;
  if (p.y > float(G.ny) - 0.5f) return G.face(1, qx, G.ny, qz) < -1e-6f;
  if (p.z < 0.5f) return G.face(2, qx, qy, 0) > 1e-6f;
  if (p.z > float(G.nz) - 0.5f) return G.face(2, qx, qy, G.nz) < -1e-6f;
  return false;
}

inline float length3(V3 v) { return std::sqrt((v.x * v.x + v.y * v.y) + v.z * v.z); }

V3 trace_offset(const Grid& G, int x, int y, int z, float dir) {
  const V3 pos{float(x) + 0.5f, float(y) + 0.5f, float(z) + 0.5f};
  const float h = G.h, dt = G.dt;
  const V3 v0 = sample_velocity(G, pos);
  const float steps_f = std::ceil((length3(v0) * dt) / h);
  int steps = steps_f >= 16.0f ? 16 : int(steps_f);
  if (steps < 1) steps = 1;
  const float sdt = dt / float(steps);
  const float half = dir * 0.5f;
  V3 p = pos;
  for (int s = 0; s < steps; ++s) {
    const V3 a = sample_velocity(G, p);
    const V3 mid = clamp_trace(G, V3{p.x + ((half * a.x) * sdt) / h, p.y + ((half * a.y) * sdt) / h,
                                     p.z + ((half * a.z) * sdt) / h});
    const V3 b = sample_velocity(G, mid);
    const V3 cand{p.x + ((dir * b.x) * sdt) / h, p.y + ((dir * b.y) * sdt) / h, p.z + ((dir * b.z) * sdt) / h};
    if (dir < 0.0f && exits_released(G, cand)) {
      p = cand;
      break;
    }
    p = clamp_trace(G, cand);
  }
  return V3{p.x - pos.x, p.y - pos.y, p.z - pos.z};
}

struct Stencil {
  int bx, by, bz;
  V3 f;
  float w[8];    // transportStencilWeight per corner (0 outside the lattice)
  float total;   // their sequential sum
};

Stencil stencil_at(const Grid& G, int x, int y, int z, V3 tr) {
  Stencil S;
  const float fx = std::floor(tr.x), fy = std::floor(tr.y), fz = std::floor(tr.z);
  S.bx = x + int(fx);
  S.by = y + int(fy);
  S.bz = z + int(fz);
  S.f = V3{tr.x - fx, tr.y - fy, tr.z - fz};
  S.total = 0.0f;
  for (int k = 0; k < 8; ++k) {
    const bool in = G.valid(S.bx + (k & 1), S.by + ((k >> 1) & 1), S.bz + ((k >> 2) & 1));
    S.w[k] = in ? corner_w(S.f, k) : 0.0f;
    S.total += S.w[k];
  }
  return S;
}

inline float conditioned_gamma(float sampled, float total) {
  return total >= 0.999999f ? std::fmin(kGammaMax, std::fmax(kGammaInteriorMin, sampled))
                            : std::fmin(sampled, kGammaMax);
}

// cm12GammaDiffusionFluxInto: (rho, gamma) flux into the first endpoint.
inline void diffusion_flux(float own_rho, float own_g, float n_rho, float n_g, float open, float& fr, float& fg) {
  fg = (0.5f * open) * (n_g - own_g);
  fr = 0.0f;
  if (n_g > own_g) {
    fr = ((open * n_rho) * (n_g - own_g)) / (2.0f * std::fmax(n_g, 1e-9f));
  } else if (own_g > n_g) {
    fr = (((-open) * own_rho) * (own_g - n_g)) / (2.0f * std::fmax(own_g, 1e-9f));
  }
}

struct Transport {
  Grid G;
  long n;
  std::vector<int32_t> dep;   // [0, n) beta / sharpening deposits, [n, 2n) rho deficit, [2n, 3n) gamma deficit

  float beta(int x, int y, int z) const {
    if (!G.valid(x, y, z)) return 1.0f;
    return float(dep[G.idx(x, y, z)]) / kFixed;
  }

  void trace_beta(const float* gam_in, float* gam_adv) {
    for (int z = 0; z < G.nz; ++z)
      for (int y = 0; y < G.ny; ++y)
        for (int x = 0; x < G.nx; ++x) {
          const Stencil S = stencil_at(G, x, y, z, trace_offset(G, x, y, z, -1.0f));
          float t[8];
          for (int k = 0; k < 8; ++k) {
            t[k] = 0.0f;
            if (S.w[k] > 0.0f)
              t[k] = S.w[k] * gam_in[G.idx(S.bx + (k & 1), S.by + ((k >> 1) & 1), S.bz + ((k >> 2) & 1))];
          }
          const float g = conditioned_gamma(d4sum8(t), S.total);
          gam_adv[G.idx(x, y, z)] = g;
          if (S.total <= 1e-9f) continue;
          for (int k = 0; k < 8; ++k) {
            const float wk = S.w[k] / S.total;
            if (wk > 0.0f)
              wrap_add(dep[G.idx(S.bx + (k & 1), S.by + ((k >> 1) & 1), S.bz + ((k >> 2) & 1))],
                       fix_round((g * wk) * kFixed));
          }
        }
  }

  void scatter_deficit(const float* rho, const float* gam) {
    for (int z = 0; z < G.nz; ++z)
      for (int y = 0; y < G.ny; ++y)
        for (int x = 0; x < G.nx; ++x) {
          const float deficit = std::fmax(0.0f, 1.0f - beta(x, y, z));
          if (deficit <= 1.0f / kFixed) continue;
          const long i = G.idx(x, y, z);
          const Stencil S = stencil_at(G, x, y, z, trace_offset(G, x, y, z, 1.0f));
          if (S.total <= 1e-9f) {
            wrap_add(dep[n + i], fix_round((rho[i] * deficit) * kFixed));
            wrap_add(dep[2 * n + i], fix_round((gam[i] * deficit) * kFixed));
            continue;
          }
          for (int k = 0; k < 8; ++k) {
            const float wk = S.w[k] / S.total;
            if (wk <= 0.0f) continue;
            const long r = G.idx(S.bx + (k & 1), S.by + ((k >> 1) & 1), S.bz + ((k >> 2) & 1));
            wrap_add(dep[n + r], fix_round(((rho[i] * deficit) * wk) * kFixed));
            wrap_add(dep[2 * n + r], fix_round(((gam[i] * deficit) * wk) * kFixed));
          }
        }
  }

  void gather(const float* rho, const float* gam_adv, float* rho_out, float* gam_out) {
    for (int z = 0; z < G.nz; ++z)
      for (int y = 0; y < G.ny; ++y)
        for (int x = 0; x < G.nx; ++x) {
          const long i = G.idx(x, y, z);
          const Stencil S = stencil_at(G, x, y, z, trace_offset(G, x, y, z, -1.0f));
          const float g = gam_adv[i];
          float rn = 0.0f, gn = 0.0f;
          for (int k = 0; k < 8; ++k) {
            if (S.total <= 1e-9f) break;
            const float wk = S.w[k] / S.total;
            if (wk <= 0.0f) continue;
            const int X = S.bx + (k & 1), Y = S.by + ((k >> 1) & 1), Z = S.bz + ((k >> 2) & 1);
            const float sc = (g * wk) / std::fmax(1.0f, beta(X, Y, Z));
            rn += sc * rho[G.idx(X, Y, Z)];
            gn += sc;
          }
          rn += float(dep[n + i]) / kFixed;
          gn += float(dep[2 * n + i]) / kFixed;
          if (rn < 1e-5f) gn = 1.0f;
          rho_out[i] = std::fmax(rn, 0.0f);
          gam_out[i] = std::fmax(gn, 0.0f);
        }
  }

  void diffuse(int axis, const float* rho, const float* gam, float* rho_out, float* gam_out) const {
    const int e[3] = {axis == 0, axis == 1, axis == 2};
    for (int z = 0; z < G.nz; ++z)
      for (int y = 0; y < G.ny; ++y)
        for (int x = 0; x < G.nx; ++x) {
          const long i = G.idx(x, y, z);
          const float orho = rho[i], og = gam[i];
          float dr = 0.0f, dg = 0.0f;
          if (G.valid(x - e[0], y - e[1], z - e[2])) {
            const long j = G.idx(x - e[0], y - e[1], z - e[2]);
            float fr, fg;
            diffusion_flux(orho, og, rho[j], gam[j], 1.0f, fr, fg);
            dr += fr;
            dg += fg;
          }
          if (G.valid(x + e[0], y + e[1], z + e[2])) {
            const long j = G.idx(x + e[0], y + e[1], z + e[2]);
            float fr, fg;
            diffusion_flux(orho, og, rho[j], gam[j], 1.0f, fr, fg);
            dr += fr;
            dg += fg;
          }
          rho_out[i] = orho + dr;
          gam_out[i] = og + dg;
        }
  }

  float vol(const float* rho, int x, int y, int z) const { return G.valid(x, y, z) ? rho[G.idx(x, y, z)] : 0.0f; }

  // faceOpenFraction without embedded solids: 1 between two cells, 1 on the
  // authored open top, 0 on every other wall.
  float face_open(int x, int y, int z, int axis) const {
    const int X = x + (axis == 0), Y = y + (axis == 1), Z = z + (axis == 2);
    if (!G.valid(x, y, z) || !G.valid(X, Y, Z)) {
      if (axis == 1 && G.valid(x, y, z) && y == G.ny - 1 && G.open_top) return 1.0f;
      return 0.0f;
    }
    return 1.0f;
  }

  float sharpen_delta(const float* rho, int x, int y, int z, float strength) const {
    const float r = vol(rho, x, y, z);
    const float h = G.h;
    const float dT = (3.0f * G.dt) * strength;
    float s[3][2];
    for (int a = 0; a < 3; ++a) {
      const int ex = a == 0, ey = a == 1, ez = a == 2;
      const float op = std::fmax(face_open(x, y, z, a), 0.0f);
      const float om = std::fmax(face_open(x - ex, y - ey, z - ez, a), 0.0f);
      s[a][0] = ((-(r * op - vol(rho, x - ex, y - ey, z - ez) * om)) * dT) / h;
      s[a][1] = ((-(vol(rho, x + ex, y + ey, z + ez) * op - r * om)) * dT) / h;
    }
    float plus[3], minus[3];
    for (int a = 0; a < 3; ++a) {
      const float sp = s[a][0], sm = s[a][1];
      plus[a] = std::fmax(std::fmax(sp, 0.0f) * std::fmax(sp, 0.0f), std::fmin(sm, 0.0f) * std::fmin(sm, 0.0f));
      minus[a] = std::fmax(std::fmin(sp, 0.0f) * std::fmin(sp, 0.0f), std::fmax(sm, 0.0f) * std::fmax(sm, 0.0f));
    }
    const float gp = std::sqrt((plus[0] + plus[2]) + plus[1]);
    const float gm = std::sqrt((minus[0] + minus[2]) + minus[1]);
    float md = 0.0f;
    const int off[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    for (int k = 0; k < 6; ++k) md = std::fmax(md, std::fabs(r - vol(rho, x + off[k][0], y + off[k][1], z + off[k][2])));
    const float d = r - kIso;
    const float wgt = ((d * d) * d) * (1.0f - std::fmin(1.0f, md / kTau));
    float dr = wgt >= 0.0f ? wgt * gp : wgt * gm;
    if (r + dr < 0.0f || r < 1e-5f) dr = -r;
    else if (r > 0.5f) dr = 0.0f;
    return dr;
  }

  float sample_volume(const float* rho, V3 p) const {
    const V3 q{p.x - 0.5f, p.y - 0.5f, p.z - 0.5f};
    const float fx = std::floor(q.x), fy = std::floor(q.y), fz = std::floor(q.z);
    const int bx = int(fx), by = int(fy), bz = int(fz);
    const V3 f{q.x - fx, q.y - fy, q.z - fz};
    float t[8];
    for (int k = 0; k < 8; ++k) {
      const int X = bx + (k & 1), Y = by + ((k >> 1) & 1), Z = bz + ((k >> 2) & 1);
      t[k] = G.valid(X, Y, Z) ? corner_w(f, k) * rho[G.idx(X, Y, Z)] : 0.0f;
    }
    return d4sum8(t);
  }

  V3 volume_gradient(const float* rho, int x, int y, int z) const {
    const float h2 = 2.0f * G.h;
    return V3{(vol(rho, x + 1, y, z) - vol(rho, x - 1, y, z)) / h2, (vol(rho, x, y + 1, z) - vol(rho, x, y - 1, z)) / h2,
              (vol(rho, x, y, z + 1) - vol(rho, x, y, z - 1)) / h2};
  }

  void sharpen_scatter(const float* delta, const float* rho_s, float max_dist) {
    for (int z = 0; z < G.nz; ++z)
      for (int y = 0; y < G.ny; ++y)
        for (int x = 0; x < G.nx; ++x) {
          const long i = G.idx(x, y, z);
          const float dr = delta[i];
          if (dr >= 0.0f) continue;
          V3 p{float(x) + 0.5f, float(y) + 0.5f, float(z) + 0.5f};
          float travelled = 0.0f;
          for (int st = 0; st < 7; ++st) {
            if (sample_volume(rho_s, p) >= 0.5f || travelled >= max_dist) break;
            const V3 g = volume_gradient(rho_s, int(std::floor(p.x)), int(std::floor(p.y)), int(std::floor(p.z)));
            const float mag = length3(g);
            if (mag < 1e-6f) break;
            const float dist = std::fmin(0.5f, max_dist - travelled);
            p = V3{p.x + (g.x / mag) * dist, p.y + (g.y / mag) * dist, p.z + (g.z / mag) * dist};
            travelled += dist;
            if (sample_volume(rho_s, p) >= 0.5f) break;
          }
          const V3 an{p.x - 0.5f, p.y - 0.5f, p.z - 0.5f};
          const float fx = std::floor(an.x), fy = std::floor(an.y), fz = std::floor(an.z);
          const int cx = int(fx), cy = int(fy), cz = int(fz);
          const V3 f{an.x - fx, an.y - fy, an.z - fz};
          float wk[8], total = 0.0f;
          for (int k = 0; k < 8; ++k) {
            const bool in = G.valid(cx + (k & 1), cy + ((k >> 1) & 1), cz + ((k >> 2) & 1));
            wk[k] = in ? corner_w(f, k) : 0.0f;
            total += wk[k];
          }
          if (total <= 1e-8f) {
            wrap_add(dep[i], fix_round((-dr) * kFixed));
            continue;
          }
          for (int k = 0; k < 8; ++k) {
            if (wk[k] <= 0.0f) continue;
            wrap_add(dep[G.idx(cx + (k & 1), cy + ((k >> 1) & 1), cz + ((k >> 2) & 1))],
                     fix_round((((-dr) * wk[k]) / total) * kFixed));
          }
        }
  }
};

}  // namespace

extern "C" {

// One transport step on (rho, gamma) in place, with the face velocities
// u, v, w (already extrapolated).  diffusion: gamma diffusion repetitions;
// sharpen / mass_return: the sharpening pass and its local mass return;
// strength, max_dist: the sharpening time multiplier and trace distance
// (cells).  stages (may be NULL) receives 4 n floats: rho after the gather,
// gamma after the gather, rho after the diffusion, the sharpening delta.
void orc_transport(int nx, int ny, int nz, double h, double dt, int open_top, const float* u, const float* v,
                   const float* w, float* rho, float* gamma, int diffusion, int sharpen, int mass_return,
                   double strength, double max_dist, float* stages) {
  Transport T;
  T.G = Grid{nx, ny, nz, float(h), float(dt), open_top, u, v, w};
  T.n = (long)nx * ny * nz;
  const long n = T.n;
  T.dep.assign(3 * n, 0);
  std::vector<float> gadv(n), rho_b(n), gam_b(n), tmp_r(n), tmp_g(n), delta(n);
  T.trace_beta(gamma, gadv.data());
  T.scatter_deficit(rho, gamma);
  T.gather(rho, gadv.data(), rho_b.data(), gamma);   // rho' in rho_b, gamma' in gamma
  if (stages) {
    std::memcpy(stages, rho_b.data(), n * 4);
    std::memcpy(stages + n, gamma, n * 4);
  }
  float* cr = rho_b.data();
  float* cg = gamma;
  float* nr = tmp_r.data();
  float* ng = tmp_g.data();
  for (int it = 0; it < diffusion; ++it)
    for (int a = 0; a < 3; ++a) {
      T.diffuse(a, cr, cg, nr, ng);
      std::swap(cr, nr);
      std::swap(cg, ng);
    }
  if (cg != gamma) std::memcpy(gamma, cg, n * 4);
  if (stages) std::memcpy(stages + 2 * n, cr, n * 4);
  if (sharpen) {
    std::fill(T.dep.begin(), T.dep.begin() + n, 0);
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) delta[T.G.idx(x, y, z)] = T.sharpen_delta(cr, x, y, z, float(strength));
    std::vector<float> rs(n);
    for (long i = 0; i < n; ++i) rs[i] = cr[i] + delta[i];
    if (mass_return) {
      T.sharpen_scatter(delta.data(), rs.data(), float(max_dist));
      for (long i = 0; i < n; ++i) rho[i] = rs[i] + float(T.dep[i]) / kFixed;
    } else {
      std::memcpy(rho, rs.data(), n * 4);
    }
    if (stages) std::memcpy(stages + 3 * n, delta.data(), n * 4);
  } else {
    std::memcpy(rho, cr, n * 4);
    if (stages) std::memset(stages + 3 * n, 0, n * 4);
  }
}

}  // extern "C"
