// extrap_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle), never part of the product.
//
// A float32 CPU restatement of the uniform solver's velocity extrapolation
// (paths relative to the peter-suggate/fluid tree):
//  * lib/methods/uniform/webgpu-uniform-velocity-extrapolation.wgsl.ts
//      seedActiveFront :147-169, godunovDistance :186-220, upwindExtensionValue
//      :226-250, activeNodeConverges / activatedByConvergedUpwindNeighbor
//      :255-284, updateActiveFront :286-320, prepareActiveDispatch :331-352,
//      hierarchyComponentSample :386-414, hierarchyCorrespondingCellSample
//      :430-448, restrictKnownVelocity :450-470, prolongUnknownVelocity
//      :472-489, packTransportShell :491-507
//  * lib/methods/uniform/webgpu-uniform-velocity-extrapolation.ts:80-96
//      (pass ceiling min(max dims, 16)), :222-248 (ceil-halved levels)
// on this library's MAC layout (component c of cell p = the +c face of p; the
// domain walls closed except an open top).  Arithmetic is float32 in the
// reference's evaluation order, compiled without contraction, so the device
// kernels reproduce it bit for bit.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

constexpr float kInf = 65504.0f;
constexpr float kBand = 2.0f;

struct Grid {
  int nx, ny, nz;
  float h;
  int openTop;
  const float* vof;
  const float* open;    // may be null (no solids)
  const float* fv[3];   // may be null
  long n() const { return long(nx) * ny * nz; }
  bool in(int x, int y, int z) const { return x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz; }
  long idx(int x, int y, int z) const { return x + long(nx) * (y + long(ny) * z); }
  long face(int c, int x, int y, int z) const {
    if (c == 0) return (x + 1) + long(nx + 1) * (y + long(ny) * z);
    if (c == 1) return x + long(nx) * ((y + 1) + long(ny + 1) * z);
    return x + long(nx) * (y + long(ny) * (z + 1));
  }
};

float clamp01(float v) { return std::min(v > 0.0f ? v : 0.0f, 1.0f); }

bool isOpen(const Grid& g, int x, int y, int z, int c) {
  if (!g.in(x, y, z)) return false;
  if (c == 0 && x + 1 >= g.nx) return false;
  if (c == 1 && y + 1 >= g.ny && !g.openTop) return false;
  if (c == 2 && z + 1 >= g.nz) return false;
  if (!g.fv[0]) return true;
  return clamp01(g.fv[c][g.face(c, x, y, z)]) > 1e-5f;
}

float density(const Grid& g, int x, int y, int z) {
  if (!g.in(x, y, z)) return 0.0f;
  const long i = g.idx(x, y, z);
  if (!g.open) return g.vof[i];
  const float v = clamp01(g.open[i]);
  if (v > 1e-5f) return g.vof[i] / v;
  float best = 0.0f;
  const int dx[6] = {-1, 1, 0, 0, 0, 0}, dy[6] = {0, 0, -1, 1, 0, 0}, dz[6] = {0, 0, 0, 0, -1, 1};
  for (int k = 0; k < 6; ++k) {
    const int X = x + dx[k], Y = y + dy[k], Z = z + dz[k];
    if (!g.in(X, Y, Z)) continue;
    const long j = g.idx(X, Y, Z);
    const float vj = clamp01(g.open[j]);
    if (vj > 1e-5f) best = std::max(best, g.vof[j] / vj);
  }
  return best;
}

bool isSource(const Grid& g, int x, int y, int z, int c) {
  if (!isOpen(g, x, y, z, c)) return false;
  return density(g, x, y, z) > 0.5f || density(g, x + (c == 0), y + (c == 1), z + (c == 2)) > 0.5f;
}

bool bit(float w, int c) { return (unsigned(w) >> c) & 1u; }

float epsOf(const Grid& g, float ref) {
  const float minimum = 2.0f * g.h;
  const float ex = float(g.nx) * g.h, ey = float(g.ny) * g.h, ez = float(g.nz) * g.h;
  const float diagonal = std::sqrt((ex * ex + ey * ey) + ez * ez);
  return std::min(std::max(std::fabs(ref), minimum), diagonal) * 1.1920929e-7f;
}

using State = std::vector<std::array<float, 4>>;   // xyz + mask (w)

struct Src {
  const Grid& g;
  const State& val;
  const State& dist;
  float nd(int x, int y, int z, int c) const { return isOpen(g, x, y, z, c) ? dist[g.idx(x, y, z)][c] : kInf; }
  float nv(int x, int y, int z, int c) const {
    if (!isOpen(g, x, y, z, c)) return 0.0f;
    const auto& s = val[g.idx(x, y, z)];
    return bit(s[3], c) ? s[c] : 0.0f;
  }
  float godunov(int x, int y, int z, int c) const {
    float m[3] = {std::min(nd(x - 1, y, z, c), nd(x + 1, y, z, c)), std::min(nd(x, y - 1, z, c), nd(x, y + 1, z, c)),
                  std::min(nd(x, y, z - 1, c), nd(x, y, z + 1, c))};
    for (int i = 0; i < 2; ++i)
      for (int j = i + 1; j < 3; ++j)
        if (m[j] < m[i]) std::swap(m[i], m[j]);
    if (m[0] >= 0.5f * kInf) return kInf;
    const float h = g.h;
    float root = m[0] + h;
    for (int count = 2; count <= 3; ++count) {
      if (m[count - 1] >= 0.5f * kInf || root <= m[count - 1]) break;
      float a = 0.0f, b = 0.0f, cc = -1.0f;
      for (int k = 0; k < count; ++k) {
        const float inv = 1.0f / (h * h);
        a = a + inv;
        b = b + m[k] * inv;
        cc = cc + (m[k] * m[k]) * inv;
      }
      root = (b + std::sqrt(std::max(b * b - a * cc, 0.0f))) / a;
    }
    return root;
  }
  float upwind(int x, int y, int z, int c, float solved) const {
    float wt[3], ww[3];
    const float eps = epsOf(g, solved);
    const float h2 = g.h * g.h;
    for (int a = 0; a < 3; ++a) {
      wt[a] = 0.0f;
      ww[a] = 0.0f;
      const int ox = a == 0, oy = a == 1, oz = a == 2;
      const float lo = nd(x - ox, y - oy, z - oz, c), hi = nd(x + ox, y + oy, z + oz, c);
      const float mn = std::min(lo, hi);
      if (mn >= solved - eps) continue;
      float mv = 0.0f, mc = 0.0f;
      if (std::fabs(lo - mn) <= eps) { mv = mv + nv(x - ox, y - oy, z - oz, c); mc = mc + 1.0f; }
      if (std::fabs(hi - mn) <= eps) { mv = mv + nv(x + ox, y + oy, z + oz, c); mc = mc + 1.0f; }
      if (mc <= 0.0f) continue;
      const float w = (solved - mn) / h2;
      wt[a] = (w * mv) / mc;
      ww[a] = w;
    }
    const float sv = (wt[0] + wt[2]) + wt[1], sw = (ww[0] + ww[2]) + ww[1];
    return sw > 0.0f ? sv / sw : 0.0f;
  }
  bool converges(int x, int y, int z, int c) const {
    if (!isOpen(g, x, y, z, c) || isSource(g, x, y, z, c)) return false;
    const auto& d = dist[g.idx(x, y, z)];
    if (!bit(d[3], c)) return false;
    const float old = d[c];
    if (old >= 0.5f * kInf) return false;
    const float upd = std::min(old, godunov(x, y, z, c));
    if (upd > kBand * g.h) return false;
    return std::fabs(upd - old) <= epsOf(g, old);
  }
  bool activated(int x, int y, int z, int c) const {
    const float cand = godunov(x, y, z, c);
    if (!isOpen(g, x, y, z, c) || cand > kBand * g.h) return false;
    const float own = dist[g.idx(x, y, z)][c];
    const float eps = epsOf(g, own);
    for (int a = 0; a < 3; ++a) {
      const int ox = a == 0, oy = a == 1, oz = a == 2;
      for (int s = -1; s <= 1; s += 2) {
        const int X = x + s * ox, Y = y + s * oy, Z = z + s * oz;
        if (!converges(X, Y, Z, c)) continue;
        const float un = std::min(nd(X, Y, Z, c), godunov(X, Y, Z, c));
        if (own > un + eps) return true;
      }
    }
    return false;
  }
};

struct Dims { int x, y, z; long n() const { return long(x) * y * z; } };

std::array<float, 2> sample(const State& src, Dims sd, Dims td, int tx, int ty, int tz, int c) {
  const int t[3] = {tx, ty, tz}, s[3] = {sd.x, sd.y, sd.z}, d[3] = {td.x, td.y, td.z};
  float sp[3];
  for (int a = 0; a < 3; ++a)
    sp[a] = a == c ? (float(t[a] + 1) * float(s[a])) / float(d[a]) - 1.0f
                   : ((float(t[a]) + 0.5f) * float(s[a])) / float(d[a]) - 0.5f;
  int lo[3];
  float fr[3];
  for (int a = 0; a < 3; ++a) {
    const float f = std::floor(sp[a]);
    lo[a] = int(f);
    fr[a] = sp[a] - f;
  }
  float cb[8][2];
  for (int oz = 0; oz <= 1; ++oz)
    for (int oy = 0; oy <= 1; ++oy)
      for (int ox = 0; ox <= 1; ++ox) {
        const int o[3] = {ox, oy, oz};
        int q[3];
        float w[3];
        for (int a = 0; a < 3; ++a) {
          q[a] = std::min(std::max(lo[a] + o[a], 0), s[a] - 1);
          w[a] = o[a] ? fr[a] : 1.0f - fr[a];
        }
        const float weight = (w[0] * w[1]) * w[2];
        const auto& st = src[q[0] + long(sd.x) * (q[1] + long(sd.y) * q[2])];
        const int corner = ox + 2 * oy + 4 * oz;
        cb[corner][0] = cb[corner][1] = 0.0f;
        if (weight > 0.0f && bit(st[3], c)) { cb[corner][0] = weight * st[c]; cb[corner][1] = weight; }
      }
  float r[2];
  for (int k = 0; k < 2; ++k) {
    const float y0 = (cb[0][k] + cb[5][k]) + (cb[1][k] + cb[4][k]);
    const float y1 = (cb[2][k] + cb[7][k]) + (cb[3][k] + cb[6][k]);
    r[k] = y0 + y1;
  }
  return {r[1] > 0.0f ? r[0] / r[1] : 0.0f, r[1]};
}

std::array<float, 2> cellSample(const State& src, Dims sd, int tx, int ty, int tz, int c) {
  auto known = [&](int x, int y, int z) -> std::array<float, 2> {
    if (x < 0 || y < 0 || z < 0 || x >= sd.x || y >= sd.y || z >= sd.z) return {0.0f, 0.0f};
    const auto& s = src[x + long(sd.x) * (y + long(sd.y) * z)];
    return bit(s[3], c) ? std::array<float, 2>{s[c], 1.0f} : std::array<float, 2>{0.0f, 0.0f};
  };
  auto add = [](std::array<float, 2> a, std::array<float, 2> b) { return std::array<float, 2>{a[0] + b[0], a[1] + b[1]}; };
  const int lx = 2 * tx, ly = 2 * ty, lz = 2 * tz;
  std::array<float, 2> acc{0.0f, 0.0f};
  for (int oy = 0; oy <= 1; ++oy) {
    const auto c00 = known(lx, ly + oy, lz), c11 = known(lx + 1, ly + oy, lz + 1);
    const auto c10 = known(lx + 1, ly + oy, lz), c01 = known(lx, ly + oy, lz + 1);
    acc = add(acc, add(add(c00, c11), add(c10, c01)));
  }
  return {acc[1] > 0.0f ? acc[0] / acc[1] : 0.0f, acc[1]};
}

}  // namespace

extern "C" {

// Extrapolates u, v, w (MAC layouts, in place) like the device; open / fx / fy /
// fz may be null (no embedded solids).  Returns the number of open faces that
// received a value; passes_run (may be null) gets the FIM passes that changed
// the state.
long orc_extrapolate(int nx, int ny, int nz, double h, int openTop, const float* vof, const float* open,
                     const float* fx, const float* fy, const float* fz, float* u, float* v, float* w,
                     int* passes_run) {
  Grid g{nx, ny, nz, float(h), openTop, vof, open, {fx, fy, fz}};
  float* vel[3] = {u, v, w};
  const long n = g.n();
  State val[2], dist[2];
  for (int s = 0; s < 2; ++s) {
    val[s].assign(n, {0, 0, 0, 0});
    dist[s].assign(n, {kInf, kInf, kInf, 0});
  }
  unsigned count[2] = {0, 0};
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const long i = g.idx(x, y, z);
        unsigned known = 0, active = 0;
        for (int c = 0; c < 3; ++c) {
          if (!isOpen(g, x, y, z, c)) continue;
          if (isSource(g, x, y, z, c)) {
            val[0][i][c] = vel[c][g.face(c, x, y, z)];
            dist[0][i][c] = 0.0f;
            known |= 1u << c;
          } else {
            bool touch = false;
            for (int a = 0; a < 3 && !touch; ++a) {
              const int ox = a == 0, oy = a == 1, oz = a == 2;
              touch = (g.in(x - ox, y - oy, z - oz) && isSource(g, x - ox, y - oy, z - oz, c)) ||
                      (g.in(x + ox, y + oy, z + oz) && isSource(g, x + ox, y + oy, z + oz, c));
            }
            if (touch) active |= 1u << c;
          }
        }
        val[0][i][3] = float(known);
        dist[0][i][3] = float(active);
        count[0] += __builtin_popcount(active);
      }
  const int passes = std::min(std::max(nx, std::max(ny, nz)), 16);
  int ran = 0;
  for (int k = 0; k < passes; ++k) {
    const int src = k & 1, dst = 1 - src;
    count[dst] = 0;
    if (count[src] == 0) {
      val[dst] = val[src];
      dist[dst] = dist[src];
      continue;
    }
    ++ran;
    const Src S{g, val[src], dist[src]};
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
          const long i = g.idx(x, y, z);
          auto vv = val[src][i], dd = dist[src][i];
          unsigned known = unsigned(vv[3]), active = unsigned(dd[3]);
          for (int c = 0; c < 3; ++c) {
            if (!isOpen(g, x, y, z, c) || isSource(g, x, y, z, c)) continue;
            if ((active >> c) & 1u) {
              const float old = dd[c];
              const float eps = epsOf(g, old);
              const float upd = std::min(old, S.godunov(x, y, z, c));
              const bool band = upd <= kBand * g.h;
              if (band) {
                dd[c] = upd;
                vv[c] = S.upwind(x, y, z, c, upd);
                known |= 1u << c;
              }
              const bool conv = old < 0.5f * kInf && std::fabs(upd - old) <= eps;
              active = (!conv && band) ? (active | (1u << c)) : (active & ~(1u << c));
            } else if (S.activated(x, y, z, c)) {
              active |= 1u << c;
            }
          }
          vv[3] = float(known);
          dd[3] = float(active);
          count[dst] += __builtin_popcount(active);
          val[dst][i] = vv;
          dist[dst][i] = dd;
        }
  }
  const int last = passes & 1;
  // the known-value hierarchy
  std::vector<Dims> dims;
  Dims d{nx, ny, nz};
  while (std::min(d.x, std::min(d.y, d.z)) > 1) {
    d = {(d.x + 1) / 2, (d.y + 1) / 2, (d.z + 1) / 2};
    dims.push_back(d);
  }
  const int L = int(dims.size());
  std::vector<State> down(L), up(L);
  const State* finer = &val[last];
  Dims fd{nx, ny, nz};
  for (int l = 0; l < L; ++l) {
    down[l].assign(dims[l].n(), {0, 0, 0, 0});
    for (int z = 0; z < dims[l].z; ++z)
      for (int y = 0; y < dims[l].y; ++y)
        for (int x = 0; x < dims[l].x; ++x) {
          std::array<float, 4> out{0, 0, 0, 0};
          unsigned known = 0;
          for (int c = 0; c < 3; ++c) {
            auto r = sample(*finer, fd, dims[l], x, y, z, c);
            if (r[1] <= 0.0f && c == 1) r = cellSample(*finer, fd, x, y, z, c);
            if (r[1] > 0.0f) { out[c] = r[0]; known |= 1u << c; }
          }
          out[3] = float(known);
          down[l][x + long(dims[l].x) * (y + long(dims[l].y) * z)] = out;
        }
    finer = &down[l];
    fd = dims[l];
  }
  State finest;
  const State* result = &val[last];
  if (L > 0) {
    const State* coarser = &down[L - 1];
    Dims cd = dims[L - 1];
    for (int l = L - 2; l >= -1; --l) {
      const Dims td = l >= 0 ? dims[l] : Dims{nx, ny, nz};
      const State& keep = l >= 0 ? down[l] : val[last];
      State& out = l >= 0 ? up[l] : finest;
      out.assign(td.n(), {0, 0, 0, 0});
      for (int z = 0; z < td.z; ++z)
        for (int y = 0; y < td.y; ++y)
          for (int x = 0; x < td.x; ++x) {
            const long i = x + long(td.x) * (y + long(td.y) * z);
            auto o = keep[i];
            unsigned known = unsigned(o[3]);
            for (int c = 0; c < 3; ++c) {
              if ((known >> c) & 1u) continue;
              const auto r = sample(*coarser, cd, td, x, y, z, c);
              if (r[1] > 0.0f) { o[c] = r[0]; known |= 1u << c; }
            }
            o[3] = float(known);
            out[i] = o;
          }
      coarser = &out;
      cd = td;
    }
    result = &finest;
  }
  long filled = 0;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const auto& s = (*result)[g.idx(x, y, z)];
        for (int c = 0; c < 3; ++c) {
          if (!isOpen(g, x, y, z, c)) continue;
          const bool k = bit(s[3], c);
          vel[c][g.face(c, x, y, z)] = k ? s[c] : 0.0f;
          filled += k;
        }
      }
  if (passes_run) *passes_run = ran;
  return filled;
}

}  // extern "C"
