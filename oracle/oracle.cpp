// oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle), never part of the product.
//
// A CPU float64 restatement of the reference's free-surface pressure projection
// on a dense uniform MAC grid.  Only tests/, __graft_entry__.smoke() and the
// cpu_baseline leg / reference arm of bench.py may load this library; the CUDA
// product path never links, calls or falls back to it.
//
// What it restates (paths are relative to the peter-suggate/fluid tree):
//  * hierarchy planner      lib/methods/uniform/webgpu-uniform-pressure-multigrid.ts:99-169
//                            (planUniformCM11aHierarchy, lockstepLevels, semiCoarsenedLevels)
//  * fine-child map          lib/methods/uniform/webgpu-uniform-pressure-multigrid.wgsl.ts:71-76
//  * phi coarsening (C=2)    webgpu-uniform-pressure-multigrid.wgsl.ts:169-195, mg.ts:470-478
//  * cell labelling          lib/methods/uniform/webgpu-uniform-reference.wgsl.ts:208-242
//  * ghost-fluid theta       lib/core/cm12-numerics.ts:37-45
//  * volume correction       lib/core/cm12-numerics.ts:127-138
//  * A = G^T W G / theta     lib/methods/adaptive-mass/sparse-atlas-composite-projection.ts:978-1192
//  * rhs / nullspace / PCG   sparse-atlas-composite-projection.ts:1194-1262, 1351-1643
//  * direct-curvature PCG    lib/methods/octree-shared/octree-pipelined-pcg.ts:146-158, 232-594
//  * gradient subtract       sparse-atlas-composite-projection.ts:1263-1279, 1542-1566
//                            and webgpu-uniform-reference.wgsl.ts:1052-1099
//
// Units: every quantity is in finest-cell units (h = 1), exactly like the atlas
// oracle.  Dimensional pressure is p_cells * rho * h / dt.
//
// Parity pinning: the PCG recurrence is pinned by the reference's known-answer
// tests (tests/octree-pipelined-pcg.test.ts, ported under tests/golden).  The
// dense-grid assembly is cross-checked against an independent row-form
// restatement of the atlas code (oracle/atlas_rows.py) and scipy's direct solve.
// The reference GPU path itself has no golden values, so parity with it is
// unpinned.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int kMaxLevels = 24;
constexpr long kCoarsestLanes = 256;   // mg.ts UNIFORM_CM11A_COARSEST_LANES
constexpr double kThetaMin = 0.05;      // cm12-numerics.ts CM12_GHOST_FLUID_THETA_MIN
constexpr double kThetaEps = 1e-12;     // atlas denominatorEpsilon default

struct Plan {
  int count = 0;
  int dims[kMaxLevels][3] = {};
  int stride[kMaxLevels][3] = {};   // stride from level l-1 to level l (level 0: 1)
  long coarsest = 0;
  int semi = 0;
  int extended = 0;
  int ok = 0;
};

long haloed(const int* d) { return long(d[0] + 2) * (d[1] + 2) * (d[2] + 2); }

// mg.ts:99-111
bool lockstep(const int* d, std::vector<std::array<int, 3>>& out) {
  int mn = std::min(d[0], std::min(d[1], d[2]));
  if (mn & (mn - 1)) return false;
  int levelCount = 0;
  while ((1 << (levelCount + 1)) <= mn) ++levelCount;   // floor(log2(min))
  int coarsening = 1 << (levelCount - 1);
  for (int a = 0; a < 3; ++a)
    if (d[a] % coarsening) return false;
  out.clear();
  for (int i = 0; i < levelCount; ++i) out.push_back({d[0] >> i, d[1] >> i, d[2] >> i});
  return haloed(out.back().data()) <= kCoarsestLanes;
}

// mg.ts:118-127
void semiLevels(const int* d, std::vector<std::array<int, 3>>& out) {
  out.clear();
  out.push_back({d[0], d[1], d[2]});
  for (;;) {
    auto prev = out.back();
    std::array<int, 3> next;
    for (int a = 0; a < 3; ++a) next[a] = (prev[a] % 2 == 0 && prev[a] > 2) ? prev[a] / 2 : prev[a];
    if (next == prev) return;
    out.push_back(next);
  }
}

Plan plan(int nx, int ny, int nz) {
  Plan p;
  int d[3] = {nx, ny, nz};
  if (nx < 2 || ny < 2 || nz < 2) return p;
  std::vector<std::array<int, 3>> lv;
  bool lock = lockstep(d, lv);
  if (!lock) semiLevels(d, lv);
  p.semi = lock ? 0 : 1;
  if (haloed(lv.back().data()) > kCoarsestLanes) {
    // Extension beyond the reference planner (which rejects these lattices):
    // ceil-halve every axis above two cells until the coarsest fits 256 lanes.
    lv.clear();
    lv.push_back({d[0], d[1], d[2]});
    while (haloed(lv.back().data()) > kCoarsestLanes) {
      auto prev = lv.back();
      std::array<int, 3> next;
      for (int a = 0; a < 3; ++a) next[a] = prev[a] > 2 ? (prev[a] + 1) / 2 : prev[a];
      if (next == prev) return p;
      lv.push_back(next);
      if ((int)lv.size() > kMaxLevels) return p;
    }
    p.extended = 1;
    p.semi = 0;
  }
  if ((int)lv.size() > kMaxLevels) return p;
  p.count = (int)lv.size();
  for (int l = 0; l < p.count; ++l)
    for (int a = 0; a < 3; ++a) {
      p.dims[l][a] = lv[l][a];
      p.stride[l][a] = l == 0 ? 1 : (lv[l][a] < lv[l - 1][a] ? 2 : 1);
    }
  p.coarsest = haloed(lv.back().data());
  p.ok = 1;
  return p;
}

// ---------------------------------------------------------------- numerics
inline double theta(double liquidPhi, double airPhi) {
  double a = std::fabs(liquidPhi);
  return std::min(1.0, std::max(kThetaMin, a / std::max(a + std::fabs(airPhi), kThetaEps)));
}

// Kahan dot of sparse-atlas-composite-projection.ts:1215-1226.
double kahanDot(const double* l, const double* r, long n) {
  double sum = 0, correction = 0;
  for (long i = 0; i < n; ++i) {
    double product = l[i] * r[i];
    double adjusted = product - correction;
    double next = sum + adjusted;
    correction = (next - sum) - adjusted;
    sum = next;
  }
  return sum;
}

// Neumaier dot of octree-pipelined-pcg.ts:146-158.
double neumaierDot(const double* l, const double* r, long n) {
  double sum = 0, comp = 0;
  for (long i = 0; i < n; ++i) {
    double product = l[i] * r[i];
    double next = sum + product;
    comp += std::fabs(sum) >= std::fabs(product) ? (sum - next) + product : (product - next) + sum;
    sum = next;
  }
  return sum + comp;
}

double parallelDot(const double* l, const double* r, long n, int threads) {
  double s = 0;
#ifdef _OPENMP
#pragma omp parallel for reduction(+ : s) num_threads(threads) if (threads > 1)
#endif
  for (long i = 0; i < n; ++i) s += l[i] * r[i];
  return s;
}

struct Level {
  int n[3] = {0, 0, 0};
  int stride[3] = {1, 1, 1};
  long cells = 0;
  double w[3] = {1, 1, 1};     // off-diagonal weights (h0 / h_a)^2
  double extPhi = 0.5;         // open-top exterior phi in finest-cell units
  std::vector<uint8_t> label;  // 1 liquid, 0 air
  std::vector<float> phi;      // level-set sample, finest-cell units
  std::vector<double> diag;
  std::vector<float> ff;       // embedded solids: open fraction of each cell's +x, +y, +z face (3 x cells)
  bool anchored = true;
  long idx(int x, int y, int z) const { return x + long(n[0]) * (y + long(n[1]) * z); }
  // weight of the face between cell i and its +axis neighbour: w_a, scaled by
  // the face's open fraction with embedded solids, 0 for a closed face
  double fw(int a, long i) const {
    if (ff.empty()) return w[a];
    const float f = ff[a * cells + i];
    return f > 1e-6f ? w[a] * double(f) : 0.0;
  }
};

struct Ctx {
  int n[3];
  int openTop;
  double h, rho, dt;
  Plan pl;
  std::vector<Level> lv;
  std::vector<float> vof, u, v, w;
  std::vector<double> b;           // rhs in cell units
  std::vector<double> q;           // volume-correction target divergence (cell units)
  std::vector<double> coarseChol;  // dense Cholesky factor of the coarsest level
  // embedded solids (webgpu-uniform-reference.wgsl.ts:208-233, 530-556, 1005-1024)
  bool solids = false;
  std::vector<float> open;         // cell open fraction
  std::vector<float> fv[3], us[3]; // face open fractions and solid normal velocities (layouts of u, v, w)
  int threads = 1;
  long cells() const { return long(n[0]) * n[1] * n[2]; }
  long uIdx(int x, int y, int z) const { return x + long(n[0] + 1) * (y + long(n[1]) * z); }
  long vIdx(int x, int y, int z) const { return x + long(n[0]) * (y + long(n[1] + 1) * z); }
  long wIdx(int x, int y, int z) const { return x + long(n[0]) * (y + long(n[1]) * z); }
};

float clamp01(float v) { return std::min(v > 0.0f ? v : 0.0f, 1.0f); }   // NaN -> 0

// pressureDensity (ref.wgsl.ts:213-233): rho' = vof / open for an open cell
// (open > 1e-5), otherwise the largest rho' of its open neighbours; float32.
float solidDensity(const Ctx& c, int x, int y, int z) {
  const int nx = c.n[0], ny = c.n[1], nz = c.n[2];
  const long i = x + long(nx) * (y + long(ny) * z);
  const float v = clamp01(c.open[i]);
  if (v > 1e-5f) return c.vof[i] / v;
  float best = 0.0f;
  auto take = [&](bool inside, long j) {
    if (!inside) return;
    const float vj = clamp01(c.open[j]);
    if (vj > 1e-5f) best = std::max(best, c.vof[j] / vj);
  };
  take(x > 0, i - 1);
  take(x + 1 < nx, i + 1);
  take(y > 0, i - nx);
  take(y + 1 < ny, i + nx);
  take(z > 0, i - long(nx) * ny);
  take(z + 1 < nz, i + long(nx) * ny);
  return best;
}

// ref.wgsl.ts:208-242: rho' = vof (no embedded solids) or solidDensity,
// liquid <=> rho' > 0.5, phi = 0.5 - rho' in cell units (the WGSL multiplies by dx).
void labelFine(Ctx& c) {
  Level& L = c.lv[0];
  for (int z = 0; z < c.n[2]; ++z)
    for (int y = 0; y < c.n[1]; ++y)
      for (int x = 0; x < c.n[0]; ++x) {
        const long i = L.idx(x, y, z);
        const float rho = c.solids ? solidDensity(c, x, y, z) : c.vof[i];
        L.label[i] = rho > 0.5f ? 1 : 0;
        L.phi[i] = 0.5f - rho;
        if (c.solids && L.label[i]) {   // a liquid cell needs an open face (mg.wgsl.ts:341)
          auto open = [&](int a, long f) { return clamp01(c.fv[a][f]) > 1e-6f; };
          const int nx = c.n[0], ny = c.n[1], nz = c.n[2];
          const bool any = (x > 0 && open(0, c.uIdx(x, y, z))) || (x + 1 < nx && open(0, c.uIdx(x + 1, y, z))) ||
                           (y > 0 && open(1, c.vIdx(x, y, z))) ||
                           ((y + 1 < ny || c.openTop) && open(1, c.vIdx(x, y + 1, z))) ||
                           (z > 0 && open(2, c.wIdx(x, y, z))) || (z + 1 < nz && open(2, c.wIdx(x, y, z + 1)));
          if (!any) L.label[i] = 0;
        }
      }
}

// divergenceAt (ref.wgsl.ts:1010-1024, CM11a Eqs. 8-10) in cell units with
// face weights W = open fraction (0 for a closed face or a wall): per axis
// (W+ u+ - W- u-) + (W+ - V) us+ - (W- - V) us-, for velocities U, V, W.
template <class TV>
double solidDivergence(const Ctx& c, int x, int y, int z, const TV* U, const TV* Vv, const TV* Wv) {
  const int nx = c.n[0], ny = c.n[1], nz = c.n[2];
  const long i = x + long(nx) * (y + long(ny) * z);
  const double vi = clamp01(c.open[i]);
  auto weight = [](float f) { const float g = clamp01(f); return g > 1e-6f ? double(g) : 0.0; };
  auto axis = [&](int a, bool hm, long fm, bool hp, long fp, const TV* vel) {
    const double wm = hm ? weight(c.fv[a][fm]) : 0.0, wp = hp ? weight(c.fv[a][fp]) : 0.0;
    const double um = hm ? vel[fm] : 0.0, up = hp ? vel[fp] : 0.0;
    const double sm = hm ? c.us[a][fm] : 0.0, sp = hp ? c.us[a][fp] : 0.0;
    return (wp * up - wm * um) + ((wp - vi) * sp - (wm - vi) * sm);
  };
  const double fx = axis(0, x > 0, c.uIdx(x, y, z), x + 1 < nx, c.uIdx(x + 1, y, z), U);
  const double fy = axis(1, y > 0, c.vIdx(x, y, z), y + 1 < ny || c.openTop, c.vIdx(x, y + 1, z), Vv);
  const double fz = axis(2, z > 0, c.wIdx(x, y, z), z + 1 < nz, c.wIdx(x, y, z + 1), Wv);
  return (fx + fz) + fy;
}

// Level-0 face fractions in the level layout: the +x, +y, +z face of each
// cell, a domain-wall face 1 (no coupling; it only enters the coarse means),
// the open top its given fraction.
void solidFacesFine(Ctx& c) {
  Level& L = c.lv[0];
  L.ff.assign(3 * L.cells, 1.0f);
  for (int z = 0; z < c.n[2]; ++z)
    for (int y = 0; y < c.n[1]; ++y)
      for (int x = 0; x < c.n[0]; ++x) {
        const long i = L.idx(x, y, z);
        if (x + 1 < c.n[0]) L.ff[i] = clamp01(c.fv[0][c.uIdx(x + 1, y, z)]);
        if (y + 1 < c.n[1] || c.openTop) L.ff[L.cells + i] = clamp01(c.fv[1][c.vIdx(x, y + 1, z)]);
        if (z + 1 < c.n[2]) L.ff[2 * L.cells + i] = clamp01(c.fv[2][c.wIdx(x, y, z + 1)]);
      }
}

// Coarse face fractions: the mean of the eight children's, per axis
// (mgDownsampleTopology, mg.wgsl.ts:170-183), in float32 in mgD4Sum8 order.
void coarsenFaces(const Level& F, Level& C) {
  C.ff.assign(3 * C.cells, 0.0f);
  for (int z = 0; z < C.n[2]; ++z)
    for (int y = 0; y < C.n[1]; ++y)
      for (int x = 0; x < C.n[0]; ++x) {
        long child[8];
        int cc[3] = {x, y, z};
        for (int corner = 0; corner < 8; ++corner) {
          int o[3] = {corner & 1, (corner >> 1) & 1, (corner >> 2) & 1};
          int f[3];
          for (int a = 0; a < 3; ++a) f[a] = std::min(C.stride[a] * cc[a] + o[a] * (C.stride[a] - 1), F.n[a] - 1);
          child[corner] = F.idx(f[0], f[1], f[2]);
        }
        for (int a = 0; a < 3; ++a) {
          float v[8];
          for (int k = 0; k < 8; ++k) v[k] = F.ff[a * F.cells + child[k]];
          const float y0 = (v[0] + v[5]) + (v[1] + v[4]);
          const float y1 = (v[2] + v[7]) + (v[3] + v[6]);
          C.ff[a * C.cells + C.idx(x, y, z)] = (y0 + y1) / 8.0f;
        }
      }
}

// cm12-numerics.ts:127-138 scaled by h (cell units).
double volumeCorrection(double rho, double h, double dt) {
  double excess = std::max(0.0, rho - 1.0);
  if (excess <= 0) return 0;
  double rate = std::min(0.5 * excess, 1.0) / h;
  return std::min(rate, 1.0 / dt) * h;
}

// atlas assembleLiquidRhs (:1238-1262) on the dense grid: every interior face is
// a row with coefficients -1 (negative cell) / +1 (positive cell) and unit dual
// weight; domain-wall faces carry no row.  b = G^T W u + M q, i.e. -div(u) + q.
void buildRhs(Ctx& c) {
  const Level& L = c.lv[0];
  const int nx = c.n[0], ny = c.n[1], nz = c.n[2];
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        long i = L.idx(x, y, z);
        if (!L.label[i]) { c.b[i] = 0; c.q[i] = 0; continue; }
        double up = x + 1 < nx ? c.u[c.uIdx(x + 1, y, z)] : 0.0;
        double um = x > 0 ? c.u[c.uIdx(x, y, z)] : 0.0;
        double vp = (y + 1 < ny || c.openTop) ? c.v[c.vIdx(x, y + 1, z)] : 0.0;
        double vm = y > 0 ? c.v[c.vIdx(x, y, z)] : 0.0;
        double wp = z + 1 < nz ? c.w[c.wIdx(x, y, z + 1)] : 0.0;
        double wm = z > 0 ? c.w[c.wIdx(x, y, z)] : 0.0;
        double div = (up - um) + (wp - wm) + (vp - vm);
        if (c.solids) {   // weighted flux divergence and the volume correction of rho'
          div = solidDivergence(c, x, y, z, c.u.data(), c.v.data(), c.w.data());
          c.q[i] = volumeCorrection(solidDensity(c, x, y, z), c.h, c.dt);
        } else {
          c.q[i] = volumeCorrection(c.vof[i], c.h, c.dt);
        }
        c.b[i] = -(div - c.q[i]);
      }
}

// mgDownsampleTopology's phi rule (mg.wgsl.ts:169-195) with the D4 fold order
// mgD4Sum8 (mg.wgsl.ts:50-54), evaluated in float32 exactly as the device does.
void coarsenPhi(const Level& F, Level& C, int destIndex) {
  for (int z = 0; z < C.n[2]; ++z)
    for (int y = 0; y < C.n[1]; ++y)
      for (int x = 0; x < C.n[0]; ++x) {
        float phiT[8], posT[8], posF[8], negF[8];
        int cc[3] = {x, y, z};
        for (int corner = 0; corner < 8; ++corner) {
          int o[3] = {corner & 1, (corner >> 1) & 1, (corner >> 2) & 1};
          int f[3];
          for (int a = 0; a < 3; ++a) {
            int s = C.stride[a];
            f[a] = std::min(s * cc[a] + o[a] * (s - 1), F.n[a] - 1);
          }
          float phi = F.phi[F.idx(f[0], f[1], f[2])];
          phiT[corner] = phi;
          posT[corner] = phi >= 0.0f ? phi : 0.0f;
          posF[corner] = phi >= 0.0f ? 1.0f : 0.0f;
          negF[corner] = phi >= 0.0f ? 0.0f : 1.0f;
        }
        auto fold = [](const float* v) {
          float y0 = (v[0] + v[5]) + (v[1] + v[4]);
          float y1 = (v[2] + v[7]) + (v[3] + v[6]);
          return y0 + y1;
        };
        float phiSum = fold(phiT), posSum = fold(posT), posCount = fold(posF), negCount = fold(negF);
        bool mixed = posCount > 0.0f && negCount > 0.0f;
        bool usePositive = mixed && destIndex <= 2;
        float coarse = usePositive ? posSum / std::max(posCount, 1.0f) : phiSum / 8.0f;
        long i = C.idx(x, y, z);
        C.phi[i] = coarse;
        C.label[i] = coarse < 0.0f ? 1 : 0;
      }
}

// mgCoefficientRaw (mg.wgsl.ts:93-115) without embedded solids and with Neumann
// walls: a face to a liquid neighbour has weight w_a, a face to air w_a/theta,
// a wall face nothing; the open top uses exterior phi = h_y/2.  Diagonal only:
// the off-diagonal entry of every liquid-liquid face is -w_a.
void bakeDiag(Level& L, int openTop) {
  bool anyAir = false, anyTopLiquid = false;
  for (int z = 0; z < L.n[2]; ++z)
    for (int y = 0; y < L.n[1]; ++y)
      for (int x = 0; x < L.n[0]; ++x) {
        long i = L.idx(x, y, z);
        if (!L.label[i]) { L.diag[i] = 0; anyAir = true; continue; }
        if (y == L.n[1] - 1) anyTopLiquid = true;
        double pi = L.phi[i];
        double terms[6];
        int c[3] = {x, y, z};
        for (int nb = 0; nb < 6; ++nb) {
          int a = nb / 2, dir = (nb & 1) ? 1 : -1;
          int q[3] = {x, y, z};
          q[a] += dir;
          double t = 0;
          const long stride = a == 0 ? 1 : (a == 1 ? L.n[0] : long(L.n[0]) * L.n[1]);
          const long face = dir > 0 ? i : i - stride;   // the face's lower cell
          if (q[a] < 0 || q[a] >= L.n[a]) {
            if (openTop && a == 1 && dir > 0) t = L.fw(1, i) / theta(pi, L.extPhi);
          } else {
            long j = L.idx(q[0], q[1], q[2]);
            t = L.label[j] ? L.fw(a, face) : L.fw(a, face) / theta(pi, L.phi[j]);
          }
          terms[nb] = t;
          (void)c;
        }
        L.diag[i] = ((terms[0] + terms[1]) + (terms[4] + terms[5])) + (terms[2] + terms[3]);
        if (!L.ff.empty() && L.diag[i] == 0.0) L.label[i] = 0;   // every face closed: no unknown
      }
  L.anchored = anyAir || (openTop && anyTopLiquid);
}

void applyLevel(const Level& L, const double* p, double* out, int threads) {
  const int nx = L.n[0], ny = L.n[1], nz = L.n[2];
  (void)threads;
#ifdef _OPENMP
#pragma omp parallel for collapse(2) num_threads(threads) if (threads > 1)
#endif
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        long i = L.idx(x, y, z);
        if (!L.label[i]) { out[i] = 0; continue; }
        const long sz = long(nx) * ny;
        double s = 0;
        if (x > 0) s += L.fw(0, i - 1) * p[i - 1];
        if (x + 1 < nx) s += L.fw(0, i) * p[i + 1];
        if (y > 0) s += L.fw(1, i - nx) * p[i - nx];
        if (y + 1 < ny) s += L.fw(1, i) * p[i + nx];
        if (z > 0) s += L.fw(2, i - sz) * p[i - sz];
        if (z + 1 < nz) s += L.fw(2, i) * p[i + sz];
        out[i] = L.diag[i] * p[i] - s;   // air neighbours hold zero
      }
}

// Cell-centred trilinear prolongation weights along one axis (mg.wgsl.ts:217-241:
// taps outside the grid dropped, remaining weights renormalised).
int taps1d(int i, int stride, int nc, int* c, double* wgt) {
  if (stride == 1) { c[0] = i; wgt[0] = 1; return 1; }
  int k = i >> 1;
  int a, b;
  double wa, wb;
  if ((i & 1) == 0) { a = k - 1; wa = 0.25; b = k; wb = 0.75; }
  else { a = k; wa = 0.75; b = k + 1; wb = 0.25; }
  int n = 0;
  double tot = 0;
  if (a >= 0 && a < nc) { c[n] = a; wgt[n] = wa; tot += wa; ++n; }
  if (b >= 0 && b < nc) { c[n] = b; wgt[n] = wb; tot += wb; ++n; }
  for (int t = 0; t < n; ++t) wgt[t] /= tot;
  return n;
}

void smooth(const Level& L, const double* rhs, double* z, int colour) {
  const int nx = L.n[0], ny = L.n[1], nz = L.n[2];
  for (int zz = 0; zz < nz; ++zz)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        if (((x + y + zz) & 1) != colour) continue;
        long i = L.idx(x, y, zz);
        if (!L.label[i]) { z[i] = 0; continue; }
        const long sz = long(nx) * ny;
        double s = 0;
        if (x > 0) s += L.fw(0, i - 1) * z[i - 1];
        if (x + 1 < nx) s += L.fw(0, i) * z[i + 1];
        if (y > 0) s += L.fw(1, i - nx) * z[i - nx];
        if (y + 1 < ny) s += L.fw(1, i) * z[i + nx];
        if (zz > 0) s += L.fw(2, i - sz) * z[i - sz];
        if (zz + 1 < nz) s += L.fw(2, i) * z[i + sz];
        z[i] = (rhs[i] + s) / L.diag[i];
      }
}

void restrictRes(const Level& F, const Level& C, const double* r, double* rc) {
  std::fill(rc, rc + C.cells, 0.0);
  int k = 0;
  for (int a = 0; a < 3; ++a) k += C.stride[a] == 2;
  double scale = 1.0 / double(1 << k);
  for (int z = 0; z < F.n[2]; ++z)
    for (int y = 0; y < F.n[1]; ++y)
      for (int x = 0; x < F.n[0]; ++x) {
        long i = F.idx(x, y, z);
        if (!F.label[i] || r[i] == 0) continue;
        int cx[2], cy[2], cz[2];
        double wx[2], wy[2], wz[2];
        int nxx = taps1d(x, C.stride[0], C.n[0], cx, wx);
        int nyy = taps1d(y, C.stride[1], C.n[1], cy, wy);
        int nzz = taps1d(z, C.stride[2], C.n[2], cz, wz);
        for (int c2 = 0; c2 < nzz; ++c2)
          for (int c1 = 0; c1 < nyy; ++c1)
            for (int c0 = 0; c0 < nxx; ++c0)
              rc[C.idx(cx[c0], cy[c1], cz[c2])] += wx[c0] * wy[c1] * wz[c2] * scale * r[i];
      }
  for (long j = 0; j < C.cells; ++j)
    if (!C.label[j]) rc[j] = 0;
}

void prolongAdd(const Level& F, const Level& C, const double* e, double* z) {
  for (int zz = 0; zz < F.n[2]; ++zz)
    for (int y = 0; y < F.n[1]; ++y)
      for (int x = 0; x < F.n[0]; ++x) {
        long i = F.idx(x, y, zz);
        if (!F.label[i]) continue;
        int cx[2], cy[2], cz[2];
        double wx[2], wy[2], wz[2];
        int nxx = taps1d(x, C.stride[0], C.n[0], cx, wx);
        int nyy = taps1d(y, C.stride[1], C.n[1], cy, wy);
        int nzz = taps1d(zz, C.stride[2], C.n[2], cz, wz);
        double s = 0;
        for (int c2 = 0; c2 < nzz; ++c2)
          for (int c1 = 0; c1 < nyy; ++c1)
            for (int c0 = 0; c0 < nxx; ++c0)
              s += wx[c0] * wy[c1] * wz[c2] * e[C.idx(cx[c0], cy[c1], cz[c2])];
        z[i] += s;
      }
}

// Dense Cholesky of the coarsest operator.  Air cells are identity rows; a level
// with no Dirichlet contact gets the rank-one term c/m * 1 1^T so the factor is
// SPD and acts as the pseudo-inverse on mean-zero data.
void factorCoarsest(Ctx& c) {
  const Level& L = c.lv.back();
  const long m = L.cells;
  std::vector<double> A(m * m, 0.0);
  for (int z = 0; z < L.n[2]; ++z)
    for (int y = 0; y < L.n[1]; ++y)
      for (int x = 0; x < L.n[0]; ++x) {
        long i = L.idx(x, y, z);
        if (!L.label[i]) { A[i * m + i] = 1; continue; }
        A[i * m + i] = L.diag[i];
        int q[3];
        for (int nb = 0; nb < 6; ++nb) {
          int a = nb / 2, dir = (nb & 1) ? 1 : -1;
          q[0] = x; q[1] = y; q[2] = z;
          q[a] += dir;
          if (q[a] < 0 || q[a] >= L.n[a]) continue;
          long j = L.idx(q[0], q[1], q[2]);
          if (L.label[j]) A[i * m + j] = -L.fw(a, std::min(i, j));
        }
      }
  if (!L.anchored) {
    double mean = 0;
    for (long i = 0; i < m; ++i) mean += L.diag[i];
    mean /= double(m);
    for (long i = 0; i < m; ++i)
      for (long j = 0; j < m; ++j) A[i * m + j] += mean / double(m);
  }
  for (long j = 0; j < m; ++j) {
    double d = A[j * m + j];
    for (long k = 0; k < j; ++k) d -= A[j * m + k] * A[j * m + k];
    d = std::sqrt(std::max(d, 1e-300));
    A[j * m + j] = d;
    for (long i = j + 1; i < m; ++i) {
      double s = A[i * m + j];
      for (long k = 0; k < j; ++k) s -= A[i * m + k] * A[j * m + k];
      A[i * m + j] = s / d;
    }
  }
  c.coarseChol = A;
}

void solveCoarsest(const Ctx& c, const double* rhs, double* z) {
  const Level& L = c.lv.back();
  const long m = L.cells;
  const double* A = c.coarseChol.data();
  std::vector<double> y(m);
  for (long i = 0; i < m; ++i) {
    double s = L.label[i] ? rhs[i] : 0.0;
    for (long k = 0; k < i; ++k) s -= A[i * m + k] * y[k];
    y[i] = s / A[i * m + i];
  }
  for (long i = m - 1; i >= 0; --i) {
    double s = y[i];
    for (long k = i + 1; k < m; ++k) s -= A[k * m + i] * z[k];
    z[i] = s / A[i * m + i];
  }
  for (long i = 0; i < m; ++i)
    if (!L.label[i]) z[i] = 0;
}

struct VWork {
  std::vector<std::vector<double>> rhs, z, res;
};

// keep: level l starts from the z it holds (the full cycle's prolongated
// guess, webgpu-uniform-pressure-multigrid.ts:560-561) instead of zero.
void vcycle(const Ctx& c, VWork& wk, int l, int pre, int post, bool keep = false) {
  const Level& L = c.lv[l];
  double* z = wk.z[l].data();
  const double* rhs = wk.rhs[l].data();
  if (l == (int)c.lv.size() - 1) { solveCoarsest(c, rhs, z); return; }
  if (!keep) std::fill(z, z + L.cells, 0.0);
  for (int s = 0; s < pre; ++s) { smooth(L, rhs, z, 0); smooth(L, rhs, z, 1); }
  double* res = wk.res[l].data();
  applyLevel(L, z, res, 1);
  for (long i = 0; i < L.cells; ++i) res[i] = L.label[i] ? rhs[i] - res[i] : 0.0;
  const Level& C = c.lv[l + 1];
  restrictRes(L, C, res, wk.rhs[l + 1].data());
  vcycle(c, wk, l + 1, pre, post);
  prolongAdd(L, C, wk.z[l + 1].data(), z);
  for (int s = 0; s < post; ++s) { smooth(L, rhs, z, 1); smooth(L, rhs, z, 0); }
}

void meanZero(const Level& L, double* v) {
  double s = 0;
  long cnt = 0;
  for (long i = 0; i < L.cells; ++i)
    if (L.label[i]) { s += v[i]; ++cnt; }
  if (!cnt) return;
  double m = s / double(cnt);
  for (long i = 0; i < L.cells; ++i)
    if (L.label[i]) v[i] -= m;
}

void precondition(const Ctx& c, VWork& wk, const double* r, double* z, int pre, int post) {
  const Level& L0 = c.lv[0];
  std::copy(r, r + L0.cells, wk.rhs[0].begin());
  vcycle(c, wk, 0, pre, post);
  std::copy(wk.z[0].begin(), wk.z[0].end(), z);
  if (!L0.anchored) meanZero(L0, z);
}

// One full cycle with zero initial guess (fullCycle,
// webgpu-uniform-pressure-multigrid.ts:539-563): r restricted down to level
// fb, one V-cycle from fb (levels fb.. are not nested: they stand for the small
// levels a device solves in one CTA), then for each level l = fb-1 .. 0 the
// prolongated correction is the guess of a V-cycle from l.
void fcycle(const Ctx& c, VWork& wk, const double* r, double* z, int pre, int post, int fb) {
  const Level& L0 = c.lv[0];
  const int last = (int)c.lv.size() - 1;
  fb = std::max(0, std::min(fb, last));
  std::copy(r, r + L0.cells, wk.rhs[0].begin());
  for (int l = 0; l < fb; ++l) restrictRes(c.lv[l], c.lv[l + 1], wk.rhs[l].data(), wk.rhs[l + 1].data());
  vcycle(c, wk, fb, pre, post);
  for (int l = fb - 1; l >= 0; --l) {
    std::fill(wk.z[l].begin(), wk.z[l].end(), 0.0);
    prolongAdd(c.lv[l], c.lv[l + 1], wk.z[l + 1].data(), wk.z[l].data());
    vcycle(c, wk, l, pre, post, true);
  }
  std::copy(wk.z[0].begin(), wk.z[0].end(), z);
  if (!L0.anchored) meanZero(L0, z);
}

// ------------------------------------------------------------ CM11a LCP
// The projected multigrid of the reference's uniform GPU method
// (webgpu-uniform-pressure-multigrid.ts:419-576, .wgsl.ts:155-166, 267-344,
// 404-471) on this oracle's face-weighted levels: p >= p_min with p_min = 0 on
// solid cells that are unknowns (open fraction <= 1e-5), unbounded elsewhere.
constexpr double kNoBound = -3.402823e38;

struct LcpWork {
  std::vector<std::vector<double>> z, rhs, res, pmin;
};

// mgSmoothColour with the projection to the bound (Eq. 18): the colour's liquid
// cells take max(GS update, p_min), the other colour's liquid cells max(z, p_min).
void lcpSmooth(const Level& L, const double* rhs, double* z, const double* pmin, int colour) {
  const int nx = L.n[0], ny = L.n[1], nz = L.n[2];
  const long sz = long(nx) * ny;
  for (int zz = 0; zz < nz; ++zz)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        long i = L.idx(x, y, zz);
        if (((x + y + zz) & 1) != colour) {
          if (L.label[i]) z[i] = std::max(z[i], pmin[i]);
          continue;
        }
        if (!L.label[i]) { z[i] = 0; continue; }
        double s = 0;
        if (x > 0) s += L.fw(0, i - 1) * z[i - 1];
        if (x + 1 < nx) s += L.fw(0, i) * z[i + 1];
        if (y > 0) s += L.fw(1, i - nx) * z[i - nx];
        if (y + 1 < ny) s += L.fw(1, i) * z[i + nx];
        if (zz > 0) s += L.fw(2, i - sz) * z[i - sz];
        if (zz + 1 < nz) s += L.fw(2, i) * z[i + sz];
        z[i] = std::max((rhs[i] + s) / L.diag[i], pmin[i]);
      }
}

// Bound of level C from level F: mode 0 max over the children of (p_min - z),
// 1 max of the children's p_min, 2 unbounded.
void lcpBoundDown(const Level& F, const Level& C, const double* zf, const double* pf, double* pc, int mode) {
  for (int z = 0; z < C.n[2]; ++z)
    for (int y = 0; y < C.n[1]; ++y)
      for (int x = 0; x < C.n[0]; ++x) {
        double b = kNoBound;
        if (mode != 2) {
          int cc[3] = {x, y, z};
          for (int corner = 0; corner < 8; ++corner) {
            int o[3] = {corner & 1, (corner >> 1) & 1, (corner >> 2) & 1};
            int f[3];
            for (int a = 0; a < 3; ++a) f[a] = std::min(C.stride[a] * cc[a] + o[a] * (C.stride[a] - 1), F.n[a] - 1);
            const long k = F.idx(f[0], f[1], f[2]);
            b = std::max(b, mode == 0 && pf[k] != kNoBound ? pf[k] - zf[k] : pf[k]);
          }
        }
        pc[C.idx(x, y, z)] = b;
      }
}

// Projected fixed-point residual of one row (mgMeasureFineResidual / mgSolveCoarsest).
double lcpRowResidual(double r, double z, double pmin, double diag) {
  const double gap = std::max(0.0, z - pmin);
  return (r < 0.0 && -r >= gap * diag) ? gap * diag : std::fabs(r);
}

// mgSolveCoarsest: projected red-black sweeps from z = 0 until the largest
// projected residual is at most tol * max|rhs| or after cap sweeps.
void lcpCoarse(const Level& L, const double* rhs, double* z, const double* pmin, int cap, double tol) {
  std::fill(z, z + L.cells, 0.0);
  double bmax = 0;
  for (long i = 0; i < L.cells; ++i)
    if (L.label[i]) bmax = std::max(bmax, std::fabs(rhs[i]));
  std::vector<double> az(L.cells);
  for (int sweep = 0; sweep < cap; ++sweep) {
    for (int colour = 0; colour < 2; ++colour)
      for (int zz = 0; zz < L.n[2]; ++zz)
        for (int y = 0; y < L.n[1]; ++y)
          for (int x = 0; x < L.n[0]; ++x) {
            const long i = L.idx(x, y, zz);
            if (((x + y + zz) & 1) != colour || !L.label[i] || !(L.diag[i] > 0)) continue;
            const long sy = L.n[0], sz = long(L.n[0]) * L.n[1];
            double s = 0;
            if (x > 0 && L.label[i - 1]) s += L.fw(0, i - 1) * z[i - 1];
            if (x + 1 < L.n[0] && L.label[i + 1]) s += L.fw(0, i) * z[i + 1];
            if (y > 0 && L.label[i - sy]) s += L.fw(1, i - sy) * z[i - sy];
            if (y + 1 < L.n[1] && L.label[i + sy]) s += L.fw(1, i) * z[i + sy];
            if (zz > 0 && L.label[i - sz]) s += L.fw(2, i - sz) * z[i - sz];
            if (zz + 1 < L.n[2] && L.label[i + sz]) s += L.fw(2, i) * z[i + sz];
            z[i] = std::max((rhs[i] + s) / L.diag[i], pmin[i]);
          }
    applyLevel(L, z, az.data(), 1);
    double worst = 0;
    for (long i = 0; i < L.cells; ++i)
      if (L.label[i] && L.diag[i] > 0) worst = std::max(worst, lcpRowResidual(rhs[i] - az[i], z[i], pmin[i], L.diag[i]));
    if (worst <= tol * bmax) break;
  }
}

void lcpResidualRestrict(const Ctx& c, LcpWork& wk, int l) {
  const Level& L = c.lv[l];
  applyLevel(L, wk.z[l].data(), wk.res[l].data(), 1);
  for (long i = 0; i < L.cells; ++i) wk.res[l][i] = L.label[i] ? wk.rhs[l][i] - wk.res[l][i] : 0.0;
  restrictRes(L, c.lv[l + 1], wk.res[l].data(), wk.rhs[l + 1].data());
}

struct LcpOpts {
  int pre, post, constraintLevels, coarseSweeps;
  double coarseTol;
};

void lcpVcycle(const Ctx& c, LcpWork& wk, int l, const LcpOpts& o) {
  const int last = (int)c.lv.size() - 1;
  const Level& L = c.lv[l];
  if (l == last) { lcpCoarse(L, wk.rhs[l].data(), wk.z[l].data(), wk.pmin[l].data(), o.coarseSweeps, o.coarseTol); return; }
  for (int s = 0; s < o.pre; ++s) {
    lcpSmooth(L, wk.rhs[l].data(), wk.z[l].data(), wk.pmin[l].data(), 0);
    lcpSmooth(L, wk.rhs[l].data(), wk.z[l].data(), wk.pmin[l].data(), 1);
  }
  lcpResidualRestrict(c, wk, l);
  std::fill(wk.z[l + 1].begin(), wk.z[l + 1].end(), 0.0);
  lcpBoundDown(L, c.lv[l + 1], wk.z[l].data(), wk.pmin[l].data(), wk.pmin[l + 1].data(), l < o.constraintLevels ? 0 : 2);
  lcpVcycle(c, wk, l + 1, o);
  prolongAdd(L, c.lv[l + 1], wk.z[l + 1].data(), wk.z[l].data());
  for (int s = 0; s < o.post; ++s) {
    lcpSmooth(L, wk.rhs[l].data(), wk.z[l].data(), wk.pmin[l].data(), 1);
    lcpSmooth(L, wk.rhs[l].data(), wk.z[l].data(), wk.pmin[l].data(), 0);
  }
}

double lcpBaseBound(const Ctx& c, long i) {
  return (c.lv[0].label[i] && !(clamp01(c.open[i]) > 1e-5f)) ? 0.0 : kNoBound;
}

void lcpFcycle(const Ctx& c, LcpWork& wk, const LcpOpts& o) {
  const Level& L0 = c.lv[0];
  const int last = (int)c.lv.size() - 1;
  std::vector<double> keep(wk.z[0]), az(L0.cells);
  applyLevel(L0, keep.data(), az.data(), 1);
  for (long i = 0; i < L0.cells; ++i) {
    wk.rhs[0][i] = L0.label[i] ? c.b[i] - az[i] : 0.0;
    const double base = lcpBaseBound(c, i);
    wk.pmin[0][i] = base == kNoBound ? kNoBound : base - keep[i];
  }
  for (int l = 0; l < last; ++l) {
    std::fill(wk.z[l].begin(), wk.z[l].end(), 0.0);
    restrictRes(c.lv[l], c.lv[l + 1], wk.rhs[l].data(), wk.rhs[l + 1].data());
    lcpBoundDown(c.lv[l], c.lv[l + 1], wk.z[l].data(), wk.pmin[l].data(), wk.pmin[l + 1].data(),
                 l < o.constraintLevels ? 1 : 2);
  }
  lcpCoarse(c.lv[last], wk.rhs[last].data(), wk.z[last].data(), wk.pmin[last].data(), o.coarseSweeps, o.coarseTol);
  for (int l = last - 1; l >= 0; --l) {
    std::fill(wk.z[l].begin(), wk.z[l].end(), 0.0);
    prolongAdd(c.lv[l], c.lv[l + 1], wk.z[l + 1].data(), wk.z[l].data());
    lcpVcycle(c, wk, l, o);
  }
  for (long i = 0; i < L0.cells; ++i) {
    wk.z[0][i] = L0.label[i] ? keep[i] + wk.z[0][i] : 0.0;
    wk.rhs[0][i] = L0.label[i] ? c.b[i] : 0.0;
    wk.pmin[0][i] = lcpBaseBound(c, i);
  }
}

void buildAll(Ctx& c) {
  labelFine(c);
  buildRhs(c);
  for (int l = 1; l < (int)c.lv.size(); ++l) coarsenPhi(c.lv[l - 1], c.lv[l], l);
  if (c.solids) {
    solidFacesFine(c);
    for (int l = 1; l < (int)c.lv.size(); ++l) coarsenFaces(c.lv[l - 1], c.lv[l]);
  }
  for (auto& L : c.lv) bakeDiag(L, c.openTop);
  if (c.solids) {   // a liquid cell dropped for its closed faces is no Dirichlet contact
    Level& L = c.lv[0];
    bool air = false, top = false;
    for (long i = 0; i < L.cells; ++i) air |= !(L.phi[i] < 0.0f);
    for (int z = 0; z < L.n[2]; ++z)
      for (int x = 0; x < L.n[0]; ++x) top |= L.label[L.idx(x, L.n[1] - 1, z)] != 0;
    L.anchored = air || (c.openTop && top);
  }
  factorCoarsest(c);
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

// Reference planner (mg.ts:149-169) plus the ceil-halving extension.  dims and
// strides are [count][3]; returns 0 on success, 1 on rejection.
int orc_plan_hierarchy(int nx, int ny, int nz, int* count, int* dims, int* strides,
                       long* coarsest, int* semi, int* extended) {
  Plan p = plan(nx, ny, nz);
  *count = p.count;
  *coarsest = p.coarsest;
  *semi = p.semi;
  *extended = p.extended;
  if (!p.ok) return 1;
  for (int l = 0; l < p.count; ++l)
    for (int a = 0; a < 3; ++a) {
      dims[l * 3 + a] = p.dims[l][a];
      strides[l * 3 + a] = p.stride[l][a];
    }
  return 0;
}

void* orc_create(int nx, int ny, int nz, int openTop, double h, double rho) {
  Plan p = plan(nx, ny, nz);
  if (!p.ok) return nullptr;
  Ctx* c = new Ctx();
  c->n[0] = nx; c->n[1] = ny; c->n[2] = nz;
  c->openTop = openTop;
  c->h = h; c->rho = rho; c->dt = 1.0;
  c->pl = p;
  c->lv.resize(p.count);
  for (int l = 0; l < p.count; ++l) {
    Level& L = c->lv[l];
    for (int a = 0; a < 3; ++a) {
      L.n[a] = p.dims[l][a];
      L.stride[a] = p.stride[l][a];
      double s = double(c->n[a]) / double(L.n[a]);   // h_l / h_0 (mg.ts:588-589)
      L.w[a] = 1.0 / (s * s);
    }
    L.extPhi = 0.5 * double(ny) / double(L.n[1]);
    L.cells = long(L.n[0]) * L.n[1] * L.n[2];
    L.label.assign(L.cells, 0);
    L.phi.assign(L.cells, 0.f);
    L.diag.assign(L.cells, 0.0);
  }
  long N = c->cells();
  c->vof.assign(N, 0.f);
  c->u.assign(long(nx + 1) * ny * nz, 0.f);
  c->v.assign(long(nx) * (ny + 1) * nz, 0.f);
  c->w.assign(long(nx) * ny * (nz + 1), 0.f);
  c->b.assign(N, 0.0);
  c->q.assign(N, 0.0);
  return c;
}

void orc_destroy(void* h) { delete static_cast<Ctx*>(h); }

void orc_set_threads(void* h, int threads) { static_cast<Ctx*>(h)->threads = std::max(1, threads); }

int orc_set_state(void* h, const float* vof, const float* u, const float* v, const float* w, double dt) {
  Ctx& c = *static_cast<Ctx*>(h);
  c.dt = dt;
  std::memcpy(c.vof.data(), vof, sizeof(float) * c.vof.size());
  std::memcpy(c.u.data(), u, sizeof(float) * c.u.size());
  std::memcpy(c.v.data(), v, sizeof(float) * c.v.size());
  std::memcpy(c.w.data(), w, sizeof(float) * c.w.size());
  buildAll(c);
  return 0;
}

int orc_num_levels(void* h) { return (int)static_cast<Ctx*>(h)->lv.size(); }

void orc_level_dims(void* h, int l, int* dims, double* weights, int* anchored) {
  const Level& L = static_cast<Ctx*>(h)->lv[l];
  for (int a = 0; a < 3; ++a) { dims[a] = L.n[a]; weights[a] = L.w[a]; }
  *anchored = L.anchored ? 1 : 0;
}

void orc_get_level(void* h, int l, uint8_t* label, float* phi, double* diag) {
  const Level& L = static_cast<Ctx*>(h)->lv[l];
  if (label) std::memcpy(label, L.label.data(), L.cells);
  if (phi) std::memcpy(phi, L.phi.data(), sizeof(float) * L.cells);
  if (diag) std::memcpy(diag, L.diag.data(), sizeof(double) * L.cells);
}

void orc_get_rhs(void* h, double* b, double* q) {
  Ctx& c = *static_cast<Ctx*>(h);
  if (b) std::memcpy(b, c.b.data(), sizeof(double) * c.b.size());
  if (q) std::memcpy(q, c.q.data(), sizeof(double) * c.q.size());
}

void orc_apply_level(void* h, int l, const double* p, double* out) {
  Ctx& c = *static_cast<Ctx*>(h);
  applyLevel(c.lv[l], p, out, c.threads);
}

void orc_vcycle(void* h, const double* r, double* z, int pre, int post) {
  Ctx& c = *static_cast<Ctx*>(h);
  VWork wk;
  for (auto& L : c.lv) {
    wk.rhs.emplace_back(L.cells, 0.0);
    wk.z.emplace_back(L.cells, 0.0);
    wk.res.emplace_back(L.cells, 0.0);
  }
  precondition(c, wk, r, z, pre, post);
}

// Embedded solids (cell open fractions, face open fractions and optional solid
// normal velocities in the layouts of u, v, w); rebuilds the system of the
// current state.
int orc_set_solids(void* h, const float* open, const float* fx, const float* fy, const float* fz, const float* usx,
                   const float* usy, const float* usz) {
  Ctx& c = *static_cast<Ctx*>(h);
  const long N = c.cells();
  c.solids = true;
  c.open.assign(open, open + N);
  const float* f[3] = {fx, fy, fz};
  const float* s[3] = {usx, usy, usz};
  const long nf[3] = {long(c.u.size()), long(c.v.size()), long(c.w.size())};
  for (int a = 0; a < 3; ++a) {
    c.fv[a].assign(f[a], f[a] + nf[a]);
    if (s[a]) c.us[a].assign(s[a], s[a] + nf[a]);
    else c.us[a].assign(nf[a], 0.0f);
  }
  buildAll(c);
  return 0;
}

// The CM11a LCP solve (embedded solids required); info: 0 cycles, 1 max and
// 2 L2 of the fine projected residual, 3 ||b||_2, 4 bounded rows at their bound.
int orc_solve_lcp(void* h, int fullCycles, int vCycles, int pre, int post, int constraintLevels, int coarseSweeps,
                  double coarseTol, double* p, double* info) {
  Ctx& c = *static_cast<Ctx*>(h);
  if (!c.solids) return 1;
  LcpWork wk;
  for (auto& L : c.lv) {
    wk.z.emplace_back(L.cells, 0.0);
    wk.rhs.emplace_back(L.cells, 0.0);
    wk.res.emplace_back(L.cells, 0.0);
    wk.pmin.emplace_back(L.cells, kNoBound);
  }
  const Level& L0 = c.lv[0];
  for (long i = 0; i < L0.cells; ++i) {
    wk.rhs[0][i] = L0.label[i] ? c.b[i] : 0.0;
    wk.pmin[0][i] = lcpBaseBound(c, i);
  }
  const LcpOpts o{pre, post, constraintLevels, coarseSweeps, coarseTol};
  for (int k = 0; k < fullCycles; ++k) lcpFcycle(c, wk, o);
  for (int k = 0; k < vCycles; ++k) lcpVcycle(c, wk, 0, o);
  std::vector<double> az(L0.cells);
  applyLevel(L0, wk.z[0].data(), az.data(), 1);
  double mx = 0, ss = 0, bb = 0;
  long atBound = 0;
  for (long i = 0; i < L0.cells; ++i) {
    p[i] = L0.label[i] ? wk.z[0][i] : 0.0;
    if (!L0.label[i] || !(L0.diag[i] > 0)) continue;
    const double r = lcpRowResidual(c.b[i] - az[i], wk.z[0][i], wk.pmin[0][i], L0.diag[i]);
    mx = std::max(mx, r);
    ss += r * r;
    bb += c.b[i] * c.b[i];
    atBound += wk.pmin[0][i] != kNoBound && wk.z[0][i] <= wk.pmin[0][i];
  }
  info[0] = fullCycles + vCycles; info[1] = mx; info[2] = std::sqrt(ss); info[3] = std::sqrt(bb);
  info[4] = double(atBound);
  return 0;
}

void orc_level_faces(void* h, int l, float* ff) {
  const Level& L = static_cast<Ctx*>(h)->lv[l];
  std::copy(L.ff.begin(), L.ff.end(), ff);
}

void orc_fcycle(void* h, const double* r, double* z, int pre, int post, int firstBlock) {
  Ctx& c = *static_cast<Ctx*>(h);
  VWork wk;
  for (auto& L : c.lv) {
    wk.rhs.emplace_back(L.cells, 0.0);
    wk.z.emplace_back(L.cells, 0.0);
    wk.res.emplace_back(L.cells, 0.0);
  }
  fcycle(c, wk, r, z, pre, post, firstBlock);
}

// info layout (doubles): 0 iterations, 1 converged, 2 recursive rel residual,
// 3 true rel residual, 4 |b|_2, 5 reductions, 6 failure code (0 none,
// 1 curvature, 2 max-iterations, 3 true-residual-validation), 7 liquid cells.
static void fillInfo(double* info, int it, int conv, double rec, double tru, double bn, int red, int fail,
                     long liquid) {
  info[0] = it; info[1] = conv; info[2] = rec; info[3] = tru; info[4] = bn;
  info[5] = red; info[6] = fail; info[7] = double(liquid);
}

// sparse-atlas-composite-projection.ts:1351-1469: Jacobi-PCG with per-component
// nullspace projection (a dense grid without solids has at most one unanchored
// component, the whole box).
int orc_solve_jacobi(void* h, double relTol, double absTol, int maxIter, double* p, double* info) {
  Ctx& c = *static_cast<Ctx*>(h);
  const Level& L = c.lv[0];
  const long N = L.cells;
  const int T = c.threads;
  auto project = [&](double* v) { if (!L.anchored) meanZero(L, v); };
  auto dot = [&](const double* a, const double* b) { return T > 1 ? parallelDot(a, b, N, T) : kahanDot(a, b, N); };
  std::vector<double> rhs(c.b), r(N), z(N), d(N), q(N);
  project(rhs.data());
  double bnorm = std::sqrt(std::max(0.0, dot(rhs.data(), rhs.data())));
  std::fill(p, p + N, 0.0);
  r = rhs;
  for (long i = 0; i < N; ++i) z[i] = L.diag[i] > 0 ? r[i] / L.diag[i] : 0;
  project(z.data());
  d = z;
  double rz = dot(r.data(), z.data());
  double rnorm = std::sqrt(std::max(0.0, dot(r.data(), r.data())));
  int it = 0, fail = 0;
  double target = std::max(absTol, relTol * bnorm);
  while (it < maxIter && rnorm > target) {
    applyLevel(L, d.data(), q.data(), T);
    project(q.data());
    double curv = dot(d.data(), q.data());
    if (!(curv > 0) || !std::isfinite(curv)) { fail = 1; break; }
    double alpha = rz / curv;
#ifdef _OPENMP
#pragma omp parallel for num_threads(T) if (T > 1)
#endif
    for (long i = 0; i < N; ++i) { p[i] += alpha * d[i]; r[i] -= alpha * q[i]; }
    project(p);
    project(r.data());
    ++it;
    rnorm = std::sqrt(std::max(0.0, dot(r.data(), r.data())));
    if (rnorm <= target) break;
#ifdef _OPENMP
#pragma omp parallel for num_threads(T) if (T > 1)
#endif
    for (long i = 0; i < N; ++i) z[i] = L.diag[i] > 0 ? r[i] / L.diag[i] : 0;
    project(z.data());
    double rzn = dot(r.data(), z.data());
    double beta = rzn / rz;
#ifdef _OPENMP
#pragma omp parallel for num_threads(T) if (T > 1)
#endif
    for (long i = 0; i < N; ++i) d[i] = z[i] + beta * d[i];
    project(d.data());
    rz = rzn;
  }
  std::vector<double> tr(N);
  applyLevel(L, p, tr.data(), T);
  for (long i = 0; i < N; ++i) tr[i] -= rhs[i];
  project(tr.data());
  double tnorm = std::sqrt(std::max(0.0, dot(tr.data(), tr.data())));
  long liquid = 0;
  for (long i = 0; i < N; ++i) liquid += L.label[i];
  if (!fail && tnorm > target) fail = it >= maxIter ? 2 : 3;
  fillInfo(info, it, tnorm <= target, bnorm > 0 ? rnorm / bnorm : 0, bnorm > 0 ? tnorm / bnorm : 0, bnorm,
           0, fail, liquid);
  return fail;
}

}  // extern "C"

namespace {
// The direct-curvature PCG of octree-pipelined-pcg.ts:305-594: Neumaier dots,
// delta = d.Ad reduced directly every step, stop on the recursive residual and
// accept only after an independent b - Ax check.  Failure codes: 1 lost
// positivity/curvature, 2 maximum iterations, 3 true-residual validation.
template <class ApplyA, class ApplyM>
//
// flexible: beta = r_k+1 . (z_k+1 - z_k) / r_k . z_k (Polak-Ribiere), for a
// preconditioner that is not a fixed symmetric operator (the full cycle).
int directCurvaturePCG(long N, ApplyA applyA, ApplyM applyM, const double* b, double* x, bool hasGuess,
                       double relTol, double absTol, int maxIter, double* info, long liquid, bool flexible = false) {
  std::vector<double> r(b, b + N), z(N), Az(N), d(N), Ad(N), tr(N), zOld;
  if (hasGuess) {
    applyA(x, tr.data());
    for (long i = 0; i < N; ++i) r[i] = b[i] - tr[i];
  } else {
    std::fill(x, x + N, 0.0);
  }
  const double bnorm = std::sqrt(std::max(0.0, neumaierDot(b, b, N)));
  const double thr = std::max(absTol, relTol * std::max(bnorm, 1e-300));
  const double bn = bnorm > 0 ? bnorm : 1.0;
  applyM(r.data(), z.data());
  applyA(z.data(), Az.data());
  double gamma = neumaierDot(r.data(), z.data(), N);
  double delta = neumaierDot(z.data(), Az.data(), N);
  double rr = neumaierDot(r.data(), r.data(), N);
  int reductions = 1, it = 0, fail = 0;
  double rec = std::sqrt(std::max(0.0, rr));
  auto trueNorm = [&]() {
    applyA(x, tr.data());
    for (long i = 0; i < N; ++i) tr[i] = b[i] - tr[i];
    return std::sqrt(std::max(0.0, neumaierDot(tr.data(), tr.data(), N)));
  };
  if (rec <= thr) {
    fillInfo(info, 0, 1, rec / bn, rec / bn, bnorm, reductions, 0, liquid);
    return 0;
  }
  if (!(gamma > 0) || !(delta > 0)) {
    fillInfo(info, 0, 0, rec / bn, rec / bn, bnorm, reductions, 1, liquid);
    return 1;
  }
  double alpha = gamma / delta;
  d = z;
  Ad = Az;
  for (;;) {
    for (long i = 0; i < N; ++i) { x[i] += alpha * d[i]; r[i] -= alpha * Ad[i]; }
    ++it;
    if (flexible) zOld = z;
    applyM(r.data(), z.data());
    const double gammaN = neumaierDot(r.data(), z.data(), N);
    const double gammaOld = flexible ? neumaierDot(r.data(), zOld.data(), N) : 0.0;
    rr = neumaierDot(r.data(), r.data(), N);
    ++reductions;
    rec = std::sqrt(std::max(0.0, rr));
    if (rec <= thr) {
      const double tn = trueNorm();
      fail = tn <= thr ? 0 : 3;
      fillInfo(info, it, fail == 0, rec / bn, tn / bn, bnorm, reductions, fail, liquid);
      return fail;
    }
    if (!(gammaN > 0)) { fail = 1; break; }
    if (it >= maxIter) { fail = 2; break; }
    const double beta = (gammaN - gammaOld) / gamma;
    for (long i = 0; i < N; ++i) d[i] = z[i] + beta * d[i];
    applyA(d.data(), Ad.data());
    delta = neumaierDot(d.data(), Ad.data(), N);
    ++reductions;
    if (!(delta > 0)) { fail = 1; break; }
    alpha = gammaN / delta;
    gamma = gammaN;
  }
  const double tn = trueNorm();
  fillInfo(info, it, 0, rec / bn, tn / bn, bnorm, reductions, fail, liquid);
  return fail;
}
}  // namespace

extern "C" {

// The symmetric V-cycle as the fixed SPD preconditioner of directCurvaturePCG.
int orc_solve_mgpcg(void* h, double relTol, double absTol, int maxIter, int pre, int post, double* x,
                    double* info) {
  Ctx& c = *static_cast<Ctx*>(h);
  const Level& L = c.lv[0];
  const long N = L.cells;
  VWork wk;
  for (auto& Lv : c.lv) {
    wk.rhs.emplace_back(Lv.cells, 0.0);
    wk.z.emplace_back(Lv.cells, 0.0);
    wk.res.emplace_back(Lv.cells, 0.0);
  }
  std::vector<double> b(c.b);
  if (!L.anchored) meanZero(L, b.data());
  long liquid = 0;
  for (long i = 0; i < N; ++i) liquid += L.label[i];
  auto A = [&](const double* in, double* out) { applyLevel(L, in, out, 1); };
  auto M = [&](const double* in, double* out) { precondition(c, wk, in, out, pre, post); };
  return directCurvaturePCG(N, A, M, b.data(), x, false, relTol, absTol, maxIter, info, liquid);
}

// The full cycle (first block level firstBlock) under flexible PCG.
int orc_solve_fcg(void* h, double relTol, double absTol, int maxIter, int pre, int post, int firstBlock, double* x,
                  double* info) {
  Ctx& c = *static_cast<Ctx*>(h);
  const Level& L = c.lv[0];
  const long N = L.cells;
  VWork wk;
  for (auto& Lv : c.lv) {
    wk.rhs.emplace_back(Lv.cells, 0.0);
    wk.z.emplace_back(Lv.cells, 0.0);
    wk.res.emplace_back(Lv.cells, 0.0);
  }
  std::vector<double> b(c.b);
  if (!L.anchored) meanZero(L, b.data());
  long liquid = 0;
  for (long i = 0; i < N; ++i) liquid += L.label[i];
  auto A = [&](const double* in, double* out) { applyLevel(L, in, out, 1); };
  auto M = [&](const double* in, double* out) { fcycle(c, wk, in, out, pre, post, firstBlock); };
  return directCurvaturePCG(N, A, M, b.data(), x, false, relTol, absTol, maxIter, info, liquid, true);
}

// Dense-matrix form of the same recurrence for the reference's known-answer
// systems: A is n x n row major, minv the Jacobi inverse diagonal or NULL
// (identity preconditioner), x0 an initial guess or NULL.
int orc_pcg_dense(int n, const double* A, const double* b, const double* minv, const double* x0, int maxIter,
                  double relTol, double absTol, double* x, double* info) {
  auto Am = [&](const double* in, double* out) {
    for (int i = 0; i < n; ++i) {
      double s = 0;
      for (int j = 0; j < n; ++j) s += A[long(i) * n + j] * in[j];
      out[i] = s;
    }
  };
  auto M = [&](const double* in, double* out) {
    for (int i = 0; i < n; ++i) out[i] = minv ? minv[i] * in[i] : in[i];
  };
  if (x0) std::copy(x0, x0 + n, x);
  return directCurvaturePCG(n, Am, M, b, x, x0 != nullptr, relTol, absTol, maxIter, info, n);
}

// Gradient subtract (atlas pressureCorrection + projectedFaceVelocity, and the
// uniform project kernel): u -= (p_j - p_i)/theta on faces with a liquid side,
// zero on faces with no liquid side and on closed walls.  Writes the projected
// velocities (float) and returns divergence receipts in cell units:
// out[0] max|div-q| before, out[1] max|div-q| after, out[2] L2 before, out[3] L2 after.
void orc_grad_subtract(void* h, const double* p, float* uo, float* vo, float* wo, double* out) {
  Ctx& c = *static_cast<Ctx*>(h);
  const Level& L = c.lv[0];
  const int nx = c.n[0], ny = c.n[1], nz = c.n[2];
  std::vector<double> U(c.u.size()), V(c.v.size()), W(c.w.size());
  auto pv = [&](long i) { return L.label[i] ? p[i] : 0.0; };
  auto faceCorr = [&](long i, long j) -> double {   // i negative side, j positive side
    bool li = L.label[i], lj = L.label[j];
    double th = 1.0;
    if (li && !lj) th = theta(L.phi[i], L.phi[j]);
    if (!li && lj) th = theta(L.phi[j], L.phi[i]);
    return (pv(j) - pv(i)) / th;
  };
  // embedded solids: a closed face carries the solids' velocity (ref.wgsl.ts:1085)
  auto closed = [&](int a, long f) { return c.solids && !(clamp01(c.fv[a][f]) > 1e-6f); };
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x <= nx; ++x) {
        long f = c.uIdx(x, y, z);
        if (x == 0 || x == nx) { U[f] = 0; continue; }
        long i = L.idx(x - 1, y, z), j = L.idx(x, y, z);
        if (closed(0, f)) { U[f] = c.us[0][f]; continue; }
        U[f] = (L.label[i] || L.label[j]) ? c.u[f] - faceCorr(i, j) : 0.0;
      }
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y <= ny; ++y)
      for (int x = 0; x < nx; ++x) {
        long f = c.vIdx(x, y, z);
        if (y == 0) { V[f] = 0; continue; }
        if (y == ny) {
          long i = L.idx(x, y - 1, z);
          if (c.openTop && closed(1, f)) V[f] = c.us[1][f];
          else if (c.openTop && L.label[i]) V[f] = c.v[f] - (0.0 - p[i]) / theta(L.phi[i], 0.5);
          else V[f] = 0;
          continue;
        }
        long i = L.idx(x, y - 1, z), j = L.idx(x, y, z);
        if (closed(1, f)) { V[f] = c.us[1][f]; continue; }
        V[f] = (L.label[i] || L.label[j]) ? c.v[f] - faceCorr(i, j) : 0.0;
      }
  for (int z = 0; z <= nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        long f = c.wIdx(x, y, z);
        if (z == 0 || z == nz) { W[f] = 0; continue; }
        long i = L.idx(x, y, z - 1), j = L.idx(x, y, z);
        if (closed(2, f)) { W[f] = c.us[2][f]; continue; }
        W[f] = (L.label[i] || L.label[j]) ? c.w[f] - faceCorr(i, j) : 0.0;
      }
  double m0 = 0, m1 = 0, s0 = 0, s1 = 0;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        long i = L.idx(x, y, z);
        if (!L.label[i]) continue;
        double before = -c.b[i];
        double after = (U[c.uIdx(x + 1, y, z)] - U[c.uIdx(x, y, z)]) + (W[c.wIdx(x, y, z + 1)] - W[c.wIdx(x, y, z)]) +
                       (V[c.vIdx(x, y + 1, z)] - V[c.vIdx(x, y, z)]) - c.q[i];
        if (c.solids)   // the weighted divergence of the projected faces
          after = solidDivergence(c, x, y, z, U.data(), V.data(), W.data()) - c.q[i];
        m0 = std::max(m0, std::fabs(before));
        m1 = std::max(m1, std::fabs(after));
        s0 += before * before;
        s1 += after * after;
      }
  out[0] = m0; out[1] = m1; out[2] = std::sqrt(s0); out[3] = std::sqrt(s1);
  if (uo) for (size_t k = 0; k < U.size(); ++k) uo[k] = float(U[k]);
  if (vo) for (size_t k = 0; k < V.size(); ++k) vo[k] = float(V[k]);
  if (wo) for (size_t k = 0; k < W.size(); ++k) wo[k] = float(W[k]);
}

}  // extern "C"
