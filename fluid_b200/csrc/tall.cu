// Restricted tall-cell pressure projection: MGPCG on the packed tall-cell grid.
//
// Layout (lib/core/tall-cell-grid.ts:171-190, 398-409): an nx x nz grid of
// columns; column (x, z) has a tall cell over world rows [0, base) and a cubic
// band of `band` rows above it.  Every quantity is packed per column in
// P = band + 2 samples, index x + nx * (j + P * z): j = 0 is the tall cell's
// bottom subcell (row 0), j = 1 its top subcell (row base - 1), j >= 2 the band
// row base + j - 2.
//
// Operator.  The paper's two-sample tall cell gives a non-symmetric system
// (docs/papers/tallCells.txt:356-361); this solver keeps CG by building the
// operator from the faces of the equivalent dense MAC grid, the repo's own
// face-row idiom (sparse-atlas-composite-projection.ts:381-620):
// A = sum over faces (1/theta) g g^T with g = T_i - T_j, where T maps the
// samples to a dense cell (a tall subcell interpolates its column's two
// samples linearly, Eq. 5 of the paper; a band cell is its sample; rows above
// the band are air).  A = T^T A_dense T is SPD by construction.  Band rows are
// applied matrix-free (band_entries: the six face neighbours found through the
// column bases, a tall neighbour interpolating its two samples) with a stored
// diagonal; the two tall rows of a column are a 2 x 2 diagonal block plus ELL
// rows of at most kTallW entries.
//
// Hierarchy: each coarser tall grid halves columns, rows and band, and its
// bases cover the finer tall cells (tall_plan.cpp).  Coarse phi is the mean of
// the 8 fine dense children; operators are rediscretised with the same rule
// (normalised levels: unit face weights).  Prolongation interpolates the
// coarse dense field trilinearly (taps dropped and renormalised at walls, the
// rule of mgTrilinearPressure, mg.wgsl.ts:217-241) at every fine sample's own
// position; restriction is its transpose times 1/2 (to_coarse 4 / 8 children),
// accumulated in 32.32 fixed point so the sum is order-independent.  Smoother:
// symmetric 4-colour block Gauss-Seidel (band red, band black, tall columns
// with x + z even, odd; reversed after the coarse correction).  The coarsest
// level (at most kMaxCoarse samples) is inverted densely in float64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "alloc.h"
#include "../../include/fluid_pp.h"
#include "device_util.cuh"
#include "tall_plan.h"
#include "types.h"

namespace fpp {
void set_global_error(const std::string& message);

namespace tall {

constexpr int kTallW = 48;        // off-block slots of a tall row
constexpr int kTB = 256;          // threads per CTA
constexpr int kTGrid = 148 * 8;   // grid cap (grid-stride beyond)
constexpr double kFix = 4294967296.0;   // 2^32: restriction fixed point

// Level vectors (z, rhs, res) are float on level 0 (the CG vectors) and on the
// block levels, and the handle's storage type S (float, half or bfloat16) on
// the grid levels 1 .. first block - 1.  Arithmetic is float: a read view
// converts on load, stores round once.
template <class S>
struct VecView {
  const S* p;
  __device__ __forceinline__ float operator[](long long k) const { return tof(p[k]); }
};
template <class S>
__device__ __forceinline__ VecView<S> view(const float* p) {
  return VecView<S>{reinterpret_cast<const S*>(p)};
}
template <class S>
__device__ __forceinline__ S* stor(float* p) {
  return reinterpret_cast<S*>(p);
}

struct TLevel {
  int nx, nz, fine_ny, band, P;
  int n;        // samples
  int ncol;     // columns
  unsigned long long mnx, mP, mnc;   // magic64 of nx, P and ncol (index decode)
  int* bases;
  float* phi;
  uint8_t* label;
  float* diag;  // A[k][k]; air and inactive samples 1
  float* a01;   // per column A[j0][j1]
  int* tidx;    // kTallW x 2 ncol, row 2 * column + (j == 1)
  float* tval;
  float* z;
  float* rhs;
  float* res;
  unsigned long long* acc;   // restriction accumulators (levels >= 1)
  // Level 0 only: the operator's entries in float64 (the assembly's values
  // before the float rounding).  The true residual applies them, so CG with
  // residual replacement converges to the float64 system's solution; the
  // V-cycle and the CG SpMV use the float entries above.
  double* diag64;
  double* a0164;
  double* tval64;
};

struct TInst {
  TLevel lv[kMaxLevels];
  int nlev;
  float h, rho, dt, pscale;
  float* vof;       // packed, level 0
  float* u;
  float* v;
  float* w;
  float* b;
  float* x;
  float* xlo;
  float* d;
  float* q;
  float* p_si;
  double* partial;  // kSlots x kTGrid
  double* coarse_inv;
  int coarse_m;
  Ctrl* ctrl;
  int* err;         // 1: an ELL row overflowed
};

// ------------------------------------------------------------------ helpers
// floor(n / d) for 32-bit n and d with m = magic64(d) = ceil(2^64 / d) (0 for
// d = 1): m d - 2^64 < d, so n m / 2^64 stays below the next multiple of 2^64 / d.
inline unsigned long long magic64(unsigned d) { return d <= 1 ? 0ull : ~0ull / d + 1ull; }
__device__ __forceinline__ unsigned divq(unsigned n, unsigned long long m) {
  return m == 0 ? n : unsigned(__umul64hi(n, m));
}

__device__ __forceinline__ int sidx(const TLevel& L, int x, int j, int z) { return x + L.nx * (j + L.P * z); }

__device__ __forceinline__ int sample_row(int j, int b) { return j == 0 ? 0 : (j == 1 ? b - 1 : b + j - 2); }

// Dense cell (x, y, z) as samples: tall rows interpolate (1 - t, t), a band
// row is its sample, rows above the band are air (phi 0.5).
struct Rep {
  int n;
  int s0, s1;
  double w0, w1;
  bool liq;
  float phi;
};

__device__ __forceinline__ Rep rep_of(const TLevel& L, int x, int y, int z) {
  Rep r;
  const int b = L.bases[x + L.nx * z];
  if (y < b) {
    const double t = double(y) / double(b - 1);
    r.n = 2;
    r.s0 = sidx(L, x, 0, z);
    r.s1 = sidx(L, x, 1, z);
    r.w0 = 1.0 - t;
    r.w1 = t;
  } else if (y < b + L.band) {
    r.n = 1;
    r.s0 = r.s1 = sidx(L, x, y - b + 2, z);
    r.w0 = 1.0;
    r.w1 = 0.0;
  } else {
    r.n = 0;
    r.s0 = r.s1 = -1;
    r.w0 = r.w1 = 0.0;
    r.liq = false;
    r.phi = 0.5f;
    return r;
  }
  r.liq = L.label[r.s0] != 0;
  r.phi = L.phi[r.s0];
  return r;
}

__device__ __forceinline__ double ghost_theta_d(float liquid_phi, float air_phi) {
  const double a = fabs(double(liquid_phi));
  return fmin(1.0, fmax(0.05, a / fmax(a + fabs(double(air_phi)), 1e-12)));
}

// Value of a packed array at dense cell (x, y, z) (zero above the band).
__device__ __forceinline__ double dense_val(const TLevel& L, const float* a, int x, int y, int z) {
  const int b = L.bases[x + L.nx * z];
  if (y < b) {
    const double t = double(y) / double(b - 1);
    return (1.0 - t) * double(a[sidx(L, x, 0, z)]) + t * double(a[sidx(L, x, 1, z)]);
  }
  if (y < b + L.band) return double(a[sidx(L, x, y - b + 2, z)]);
  return 0.0;
}

// Sample k -> column coordinates (x, z) and packed row j.
__device__ __forceinline__ void decode(const TLevel& L, int k, int& x, int& j, int& z) {
  const unsigned r = divq(unsigned(k), L.mnx), zz = divq(r, L.mP);
  x = k - int(r) * L.nx;
  j = int(r - zz * unsigned(L.P));
  z = int(zz);
}

__device__ __forceinline__ bool sample_active(const TLevel& L, int k, int& x, int& j, int& z, int& b) {
  const unsigned r = divq(unsigned(k), L.mnx), zz = divq(r, L.mP);
  x = k - int(r) * L.nx;
  j = int(r - zz * unsigned(L.P));
  z = int(zz);
  b = L.bases[x + L.nx * z];
  return j < 2 || b + j - 2 < L.fine_ny;
}

// ------------------------------------------------------------------ setup
// Level-0 labels and phi from the packed VOF (liquid iff vof > 0.5, phi = 0.5 - vof).
__global__ void k_tall_label(TInst* I) {
  const TLevel& L = I->lv[0];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < L.n; k += gridDim.x * blockDim.x) {
    int x, j, z, b;
    const bool act = sample_active(L, k, x, j, z, b);
    const float f = I->vof[k];
    if (!isfinite(f)) atomicExch(&I->ctrl->nonfinite, 1);
    L.phi[k] = act ? 0.5f - f : 0.5f;
    bool liq;
    if (j < 2) liq = I->vof[sidx(L, x, 0, z)] > 0.5f;   // the tall segment follows its bottom sample
    else liq = act && f > 0.5f;
    L.label[k] = liq ? 1 : 0;
    if (liq && j != 1) atomicAdd(&I->ctrl->liquid, j == 0 ? 2 : 1);
    if (!liq && act && j != 1) atomicAdd(&I->ctrl->air, 1);
  }
}

// Coarse phi: mean of the fine dense children's phi (fine rows above the band
// are air, 0.5); liquid iff phi < 0, a tall segment following its bottom sample.
__global__ void k_tall_coarsen(TInst* I, int l) {
  const TLevel& F = I->lv[l];
  const TLevel& C = I->lv[l + 1];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < C.n; k += gridDim.x * blockDim.x) {
    int X, j, Z, b;
    if (!sample_active(C, k, X, j, Z, b)) {
      C.phi[k] = 0.5f;
      continue;
    }
    const int Y = sample_row(j, b);
    float s = 0.0f;
    int cnt = 0;
    for (int dz = 0; dz < 2; ++dz)
      for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx) {
          const int x = 2 * X + dx, y = 2 * Y + dy, z = 2 * Z + dz;
          if (x >= F.nx || y >= F.fine_ny || z >= F.nz) continue;
          s += rep_of(F, x, y, z).phi;
          ++cnt;
        }
    C.phi[k] = s / float(cnt > 0 ? cnt : 1);
  }
}

__global__ void k_tall_coarse_labels(TInst* I, int l) {
  const TLevel& C = I->lv[l];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < C.n; k += gridDim.x * blockDim.x) {
    int x, j, z, b;
    const bool act = sample_active(C, k, x, j, z, b);
    bool liq = act && C.phi[k] < 0.0f;
    if (j < 2) liq = C.phi[sidx(C, x, 0, z)] < 0.0f;
    C.label[k] = liq ? 1 : 0;
  }
}

// Off-diagonal entries of band row (x, j >= 2, z) of a column of base b: for
// each liquid face neighbour, -w for every sample of its representation (a
// tall neighbour row interpolates its column's two samples, weights 1 - t and
// t).  Air and wall neighbours have none (their terms sit on the diagonal).
template <class Fn>
__device__ __forceinline__ void band_entries(const TLevel& L, int x, int j, int z, int b, Fn f) {
  const int y = b + j - 2;
  auto lateral = [&](int xn, int zn) {
    if (xn < 0 || zn < 0 || xn >= L.nx || zn >= L.nz) return;
    const int bn = L.bases[xn + L.nx * zn];
    if (y < bn) {
      const int s0 = sidx(L, xn, 0, zn);
      if (!L.label[s0]) return;
      const double t = double(y) / double(bn - 1);
      if (t != 1.0) f(s0, -(1.0 - t));
      if (t != 0.0) f(s0 + L.nx, -t);   // sample 1 of that column
    } else if (y < bn + L.band) {
      const int sn = sidx(L, xn, y - bn + 2, zn);
      if (L.label[sn]) f(sn, -1.0);
    }
  };
  lateral(x - 1, z);
  lateral(x + 1, z);
  lateral(x, z - 1);
  lateral(x, z + 1);
  const int k = sidx(L, x, j, z);
  const int below = j == 2 ? sidx(L, x, 1, z) : k - L.nx;   // the tall cell's top subcell under the band
  if (L.label[below]) f(below, -1.0);
  if (j + 1 < L.P && y + 1 < L.fine_ny && L.label[k + L.nx]) f(k + L.nx, -1.0);
}

// Band rows: the diagonal (face weights, 1/theta on faces to air, none on walls).
__global__ void k_tall_assemble_band(TInst* I, int l) {
  const TLevel& L = I->lv[l];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < L.n; k += gridDim.x * blockDim.x) {
    int x, j, z, b;
    const bool act = sample_active(L, k, x, j, z, b);
    if (j < 2) continue;
    double dg = 0.0;
    if (act && L.label[k]) {
      const int y = b + j - 2;
      const float ph = L.phi[k];
      const int nb[6][3] = {{x - 1, y, z}, {x + 1, y, z}, {x, y - 1, z}, {x, y + 1, z}, {x, y, z - 1}, {x, y, z + 1}};
      for (int f = 0; f < 6; ++f) {
        const int xn = nb[f][0], yn = nb[f][1], zn = nb[f][2];
        if (xn < 0 || yn < 0 || zn < 0 || xn >= L.nx || yn >= L.fine_ny || zn >= L.nz) continue;
        const Rep rn = rep_of(L, xn, yn, zn);
        dg += rn.liq ? 1.0 : 1.0 / ghost_theta_d(ph, rn.phi);
      }
      L.diag[k] = float(dg);
      if (L.diag64) L.diag64[k] = dg;
    } else {
      L.diag[k] = 1.0f;
      if (L.diag64) L.diag64[k] = 1.0;
    }
  }
}

// Integer power sums over rows 0 .. n - 1 (exact in float64 for n < 2^17).
__device__ __forceinline__ double psum1(int n) { return 0.5 * double(n) * double(n - 1); }
__device__ __forceinline__ double psum2(int n) { return double(n - 1) * double(n) * double(2 * n - 1) / 6.0; }

// The two tall rows of a column: 2 x 2 block (internal faces, the face to the
// first band row, lateral faces summed over the tall rows) and the couplings
// to the neighbour columns' samples.  A tall row interpolates (1 - t, t) with
// t = y / B, B = b - 1; on the rows facing a neighbour's tall cell (t' = y /
// B') or air the lateral sums have closed forms in the power sums S0, S1, S2
// of those rows:
//   sum (1 - t)^2 = (B^2 S0 - 2 B S1 + S2) / B^2,  sum (1 - t) t = (B S1 - S2) / B^2,
//   sum t^2 = S2 / B^2,  sum (1 - t)(1 - t') = (B B' S0 - (B + B') S1 + S2) / (B B'),
//   sum (1 - t) t' = (B S1 - S2) / (B B'),  sum t (1 - t') = (B' S1 - S2) / (B B'),
//   sum t t' = S2 / (B B')
// (integer numerators, one rounding).  Rows facing the neighbour's band rows
// are summed one by one and give band entries in row order.
__global__ void k_tall_assemble_tall(TInst* I, int l) {
  const TLevel& L = I->lv[l];
  const int nrow = 2 * L.ncol;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < L.ncol; c += gridDim.x * blockDim.x) {
    const int z = int(divq(unsigned(c), L.mnx)), x = c - z * L.nx;
    const int b = L.bases[c];
    const int s0 = sidx(L, x, 0, z), s1 = sidx(L, x, 1, z);
    int n0 = 0, n1 = 0;
    auto add = [&](int row, int& cnt, int s, double v) {
      if (v == 0.0) return;
      if (cnt >= kTallW) {
        atomicExch(I->err, 1);
        return;
      }
      L.tidx[cnt * nrow + row] = s;
      L.tval[cnt * nrow + row] = float(v);
      if (L.tval64) L.tval64[cnt * nrow + row] = v;
      ++cnt;
    };
    if (L.label[s0]) {
      const float ph = L.phi[s0];
      const double B = double(b - 1), BB = B * B;
      const double kin = 1.0 / B;   // b - 1 internal faces of slope 1 / (b - 1)
      double a00 = kin, a01 = -kin, a11 = kin;
      {
        const int s2 = sidx(L, x, 2, z);
        if (L.label[s2]) {
          a11 += 1.0;
          add(2 * c + 1, n1, s2, -1.0);
        } else {
          a11 += 1.0 / ghost_theta_d(ph, L.phi[s2]);
        }
      }
      // Closed-form (1 - t)^2, (1 - t) t, t^2 sums over rows [y0, y1), times w.
      auto self_sums = [&](int y0, int y1, double w) {
        if (y1 <= y0) return;
        const double S0 = double(y1 - y0), S1 = psum1(y1) - psum1(y0), S2 = psum2(y1) - psum2(y0);
        a00 += w * ((BB * S0 - 2.0 * B * S1 + S2) / BB);
        a01 += w * ((B * S1 - S2) / BB);
        a11 += w * (S2 / BB);
      };
      const int dirs[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
      for (int d = 0; d < 4; ++d) {
        const int xn = x + dirs[d][0], zn = z + dirs[d][1];
        if (xn < 0 || zn < 0 || xn >= L.nx || zn >= L.nz) continue;
        const int bn = L.bases[xn + L.nx * zn];
        const int m0 = sidx(L, xn, 0, zn), m1 = sidx(L, xn, 1, zn);
        // rows [0, min(b, bn)) face the neighbour's tall cell
        const int mt = min(b, bn);
        double c00 = 0.0, c01 = 0.0, c10 = 0.0, c11 = 0.0;
        if (L.label[m0]) {
          self_sums(0, mt, 1.0);
          const double Bn = double(bn - 1), BBn = B * Bn;
          const double S0 = double(mt), S1 = psum1(mt), S2 = psum2(mt);
          c00 = (BBn * S0 - (B + Bn) * S1 + S2) / BBn;
          c01 = (B * S1 - S2) / BBn;
          c10 = (Bn * S1 - S2) / BBn;
          c11 = S2 / BBn;
        } else {
          self_sums(0, mt, 1.0 / ghost_theta_d(ph, L.phi[m0]));
        }
        // rows [bn, min(b, bn + band)) face the neighbour's band rows
        const int ye = min(b, bn + L.band);
        for (int y = bn; y < ye; ++y) {
          const double t = double(y) / B;
          const int sn = sidx(L, xn, y - bn + 2, zn);
          if (L.label[sn]) {
            a00 += (1.0 - t) * (1.0 - t);
            a01 += (1.0 - t) * t;
            a11 += t * t;
            add(2 * c, n0, sn, -(1.0 - t));
            add(2 * c + 1, n1, sn, -t);
          } else {
            const double inv = 1.0 / ghost_theta_d(ph, L.phi[sn]);
            a00 += (1.0 - t) * (1.0 - t) * inv;
            a01 += (1.0 - t) * t * inv;
            a11 += t * t * inv;
          }
        }
        // rows [bn + band, b) face air above the neighbour's band (phi 0.5)
        self_sums(max(bn + L.band, 0), b, 1.0 / ghost_theta_d(ph, 0.5f));
        add(2 * c, n0, m0, -c00);
        add(2 * c, n0, m1, -c01);
        add(2 * c + 1, n1, m0, -c10);
        add(2 * c + 1, n1, m1, -c11);
      }
      L.diag[s0] = float(a00);
      L.diag[s1] = float(a11);
      L.a01[c] = float(a01);
      if (L.diag64) {
        L.diag64[s0] = a00;
        L.diag64[s1] = a11;
        L.a0164[c] = a01;
      }
    } else {
      L.diag[s0] = 1.0f;
      L.diag[s1] = 1.0f;
      L.a01[c] = 0.0f;
      if (L.diag64) {
        L.diag64[s0] = 1.0;
        L.diag64[s1] = 1.0;
        L.a0164[c] = 0.0;
      }
    }
    for (int s = n0; s < kTallW; ++s) {
      L.tidx[s * nrow + 2 * c] = s0;
      L.tval[s * nrow + 2 * c] = 0.0f;
      if (L.tval64) L.tval64[s * nrow + 2 * c] = 0.0;
    }
    for (int s = n1; s < kTallW; ++s) {
      L.tidx[s * nrow + 2 * c + 1] = s1;
      L.tval[s * nrow + 2 * c + 1] = 0.0f;
      if (L.tval64) L.tval64[s * nrow + 2 * c + 1] = 0.0;
    }
  }
}

// Off-diagonal part of band row (x, j >= 2, z) of a column of base b applied
// to v, in float64.
__device__ __forceinline__ double band_off(const TLevel& L, int x, int j, int z, int b, const float* v) {
  double s = 0.0;
  band_entries(L, x, j, z, b, [&](int sn, double w) { s += double(float(w)) * double(v[sn]); });
  return s;
}

// Off-block part of tall row j of column col applied to v (the 2 x 2 block
// excluded), in float64.  Entries are packed from slot 0 and padded with
// weight 0 on a valid index, so each chunk of 8 slots is loaded at once and a
// chunk ending in padding is the last.
__device__ __forceinline__ double tall_off(const TLevel& L, int col, int j, const float* v) {
  const int nrow = 2 * L.ncol, row = 2 * col + j;
  double s = 0.0;
  for (int e0 = 0; e0 < kTallW; e0 += 8) {
    float a[8], vv[8];
    int id[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      a[e] = L.tval[(e0 + e) * nrow + row];
      id[e] = L.tidx[(e0 + e) * nrow + row];
    }
#pragma unroll
    for (int e = 0; e < 8; ++e) vv[e] = v[id[e]];
#pragma unroll
    for (int e = 0; e < 8; ++e) s += double(a[e]) * double(vv[e]);
    if (a[7] == 0.0f) break;
  }
  return s;
}

// tall_off for both tall rows of column col (rows 2 col and 2 col + 1 are
// adjacent in every slot: one 8-byte load per slot for the pair).
template <class VP>
__device__ __forceinline__ void tall_off_pair(const TLevel& L, int col, VP v, double& o0, double& o1) {
  const float2* tv = reinterpret_cast<const float2*>(L.tval);
  const int2* ti = reinterpret_cast<const int2*>(L.tidx);
  double s0 = 0.0, s1 = 0.0;
  for (int e0 = 0; e0 < kTallW; e0 += 8) {
    float2 a[8];
    int2 id[8];
    float v0[8], v1[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      a[e] = tv[(e0 + e) * L.ncol + col];
      id[e] = ti[(e0 + e) * L.ncol + col];
    }
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      v0[e] = v[id[e].x];
      v1[e] = v[id[e].y];
    }
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      s0 += double(a[e].x) * double(v0[e]);
      s1 += double(a[e].y) * double(v1[e]);
    }
    if (a[7].x == 0.0f && a[7].y == 0.0f) break;
  }
  o0 = s0;
  o1 = s1;
}

// (A v)_k in float64 for a liquid sample (x, j, z) of a column of base b.
__device__ __forceinline__ double apply_row(const TLevel& L, int k, int x, int j, int z, int b, const float* v) {
  const int col = x + L.nx * z;
  double s = double(L.diag[k]) * double(v[k]);
  if (j >= 2) return s + band_off(L, x, j, z, b, v);
  s += tall_off(L, col, j, v);
  return s + double(L.a01[col]) * double(v[sidx(L, x, 1 - j, z)]);
}

// A band work item's column: its base b and, per lateral neighbour d in
// band_entries' order (x - 1, x + 1, z - 1, z + 1), e = bn - b (band row jb
// faces the neighbour's tall cell for jb < e, its band rows for e <= jb <
// e + band, air above; outside the grid e = -2^30, always air), the index
// offset from row jb's own sample to the neighbour's band sample of the same
// dense row (the same for every row), the neighbour's bottom sample and base.
struct BandCol {
  int x, z, b;
  int e[4], off[4], tn[4];
  float rbn[4];   // 1 / (bn - 1): a tall neighbour row interpolates with t = y / (bn - 1)
};

__device__ __forceinline__ void band_col(const TLevel& L, int col, BandCol& c) {
  c.z = int(divq(unsigned(col), L.mnx));
  c.x = col - c.z * L.nx;
  c.b = L.bases[col];
  const int dx[4] = {-1, 1, 0, 0}, dz[4] = {0, 0, -1, 1};
  const bool in[4] = {c.x > 0, c.x + 1 < L.nx, c.z > 0, c.z + 1 < L.nz};
  int bn[4];
#pragma unroll
  for (int d = 0; d < 4; ++d) bn[d] = in[d] ? L.bases[col + dx[d] + L.nx * dz[d]] : 2;
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    c.e[d] = in[d] ? bn[d] - c.b : -(1 << 30);
    c.off[d] = dx[d] + L.nx * (c.b - bn[d]) + L.nx * L.P * dz[d];
    c.tn[d] = in[d] ? sidx(L, c.x + dx[d], 0, c.z + dz[d]) : 0;
    c.rbn[d] = __frcp_rn(float(bn[d] - 1));
  }
}

// The off-diagonal operands of band row jb (own sample k): per lateral
// neighbour its band sample, or its tall pair, or nothing (0); then the
// sample below (the tall cell's top sample for jb = 0: also k - nx) and above.
template <class VP>
__device__ __forceinline__ void band_row_loads(const TLevel& L, const BandCol& c, int jb, int k, VP v,
                                               float (&vv)[10]) {
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    const bool tall = jb < c.e[d], band = !tall && jb < c.e[d] + L.band;
    vv[2 * d] = tall ? v[c.tn[d]] : (band ? v[k + c.off[d]] : 0.0f);
    vv[2 * d + 1] = tall ? v[c.tn[d] + L.nx] : 0.0f;
  }
  vv[8] = v[k - L.nx];
  vv[9] = jb + 1 < L.band && c.b + jb + 1 < L.fine_ny ? v[k + L.nx] : 0.0f;
}

// Off-diagonal part of band row jb applied to the operands of band_row_loads,
// in float: the weights of band_entries (a tall neighbour row interpolates
// with t = y / (bn - 1), here y times the float reciprocal), without the label
// tests (the vectors are 0 on every sample that is not liquid).
__device__ __forceinline__ float band_row_off(const TLevel& L, const BandCol& c, int jb, const float (&vv)[10]) {
  float s = 0.0f;
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    const bool tall = jb < c.e[d];
    const float t = float(c.b + jb) * c.rbn[d];
    const float wa = tall ? t - 1.0f : (jb < c.e[d] + L.band ? -1.0f : 0.0f);
    const float wb = tall ? -t : 0.0f;
    s = fmaf(wa, vv[2 * d], s);
    s = fmaf(wb, vv[2 * d + 1], s);
  }
  s -= vv[8];
  s -= vv[9];
  return s;
}

// Operator applies over every sample run over work items: items 0 .. ncol - 1
// are the columns' tall row pairs, item ncol + column + ncol * group the G
// band rows group * G .. group * G + G - 1 of a column (a warp's lanes are
// adjacent columns).  A band item loads its column's base and lateral bases
// once and issues the loads of all its rows before the first result.
constexpr int kApplyGroup = 2;

__host__ __device__ inline long long apply_items(int ncol, int band, int G) {
  return 1LL * ncol * (1 + (band + G - 1) / G);
}

// (A v)_k of both tall rows of column col: out(k, liquid, Av, v_k).
template <class VP, class Out>
__device__ __forceinline__ void tall_pair_apply(const TLevel& L, int col, VP v, Out out) {
  const int z = int(divq(unsigned(col), L.mnx)), x = col - z * L.nx;
  const int s0 = sidx(L, x, 0, z), s1 = s0 + L.nx;
  const bool l0 = L.label[s0] != 0, l1 = L.label[s1] != 0;
  const float v0 = v[s0], v1 = v[s1];
  double a0 = 0.0, a1 = 0.0;
  if (l0 || l1) {
    double o0, o1;
    tall_off_pair(L, col, v, o0, o1);
    const double a01 = L.a01[col];
    a0 = double(L.diag[s0]) * double(v0);
    a0 += o0;
    a0 = a0 + a01 * double(v1);
    a1 = double(L.diag[s1]) * double(v1);
    a1 += o1;
    a1 = a1 + a01 * double(v0);
  }
  out(s0, l0, a0, v0);
  out(s1, l1, a1, v1);
}

// (A v)_k of the G band rows of band item it, in float: out(k,
// liquid, Av, v_k, e) for each row inside the band (inactive rows above the
// fine grid as not liquid), e = extra(k) loaded with the row's operands.  v
// must be 0 on every sample that is not liquid.
template <int G, class VP, class Extra, class Out>
__device__ __forceinline__ void band_rows_apply(const TLevel& L, int it, VP v, Extra extra, Out out) {
  const int g = int(divq(unsigned(it), L.mnc));
  BandCol c;
  band_col(L, it - g * L.ncol, c);
  float vv[G][10], vk[G], dg[G], ex[G];
  bool liq[G];
#pragma unroll
  for (int r = 0; r < G; ++r) {
    const int jb = g * G + r;
    const int k = sidx(L, c.x, jb + 2, c.z);
    liq[r] = false;
    vk[r] = dg[r] = ex[r] = 0.0f;
    if (jb < L.band && c.b + jb < L.fine_ny) {
      liq[r] = L.label[k] != 0;
      dg[r] = L.diag[k];
      ex[r] = extra(k);
      vk[r] = v[k];
      band_row_loads(L, c, jb, k, v, vv[r]);
    }
  }
#pragma unroll
  for (int r = 0; r < G; ++r) {
    const int jb = g * G + r;
    if (jb >= L.band) continue;
    const float av = liq[r] ? fmaf(dg[r], vk[r], band_row_off(L, c, jb, vv[r])) : 0.0f;
    out(sidx(L, c.x, jb + 2, c.z), liq[r], av, vk[r], ex[r]);
  }
}

// Dense inverse of the coarsest level (air and inactive samples identity rows).
__global__ void k_tall_factor(TInst* I) {
  extern __shared__ double A[];
  __shared__ double prow[kMaxCoarse], pcol[kMaxCoarse];
  const TLevel& L = I->lv[I->nlev - 1];
  const int m = L.n;
  for (int e = threadIdx.x; e < m * m; e += blockDim.x) A[e] = 0.0;
  __syncthreads();
  for (int k = threadIdx.x; k < m; k += blockDim.x) {
    int x, j, z, b;
    const bool act = sample_active(L, k, x, j, z, b);
    if (!act || !L.label[k]) {
      A[k * m + k] = 1.0;
      continue;
    }
    const int col = x + L.nx * z;
    A[k * m + k] = L.diag[k];
    if (j >= 2) {
      band_entries(L, x, j, z, b, [&](int sn, double w) { A[k * m + sn] += float(w); });
    } else {
      const int nrow = 2 * L.ncol, row = 2 * col + j;
      A[k * m + sidx(L, x, 1 - j, z)] += L.a01[col];
      for (int e = 0; e < kTallW; ++e) A[k * m + L.tidx[e * nrow + row]] += L.tval[e * nrow + row];
    }
  }
  __syncthreads();
  gauss_jordan_inplace(A, m, prow, pcol);
  for (int e = threadIdx.x; e < m * m; e += blockDim.x) I->coarse_inv[e] = A[e];
}

// b = T^T (-div u) over liquid dense cells; tall samples sum their rows.
__device__ __forceinline__ double dense_div(const TInst& I, const TLevel& L, int x, int y, int z) {
  const double du = dense_val(L, I.u, x, y, z) - (x > 0 ? dense_val(L, I.u, x - 1, y, z) : 0.0);
  const double dv = dense_val(L, I.v, x, y, z) - (y > 0 ? dense_val(L, I.v, x, y - 1, z) : 0.0);
  const double dw = dense_val(L, I.w, x, y, z) - (z > 0 ? dense_val(L, I.w, x, y, z - 1) : 0.0);
  return (du + dw) + dv;
}

__global__ void k_tall_rhs(TInst* I) {
  const TLevel& L = I->lv[0];
  // Tall segments, a warp per column: b0 = sum (1 - t) (-div), b1 = sum t (-div)
  // over the column's tall rows, the lanes splitting the rows.
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int c = gw; c < L.ncol; c += nw) {
    const int z = int(divq(unsigned(c), L.mnx)), x = c - z * L.nx;
    const int b = L.bases[c];
    const int s0 = sidx(L, x, 0, z);
    double b0 = 0.0, b1 = 0.0;
    if (L.label[s0]) {
      for (int y = lane; y < b; y += 32) {
        const double t = double(y) / double(b - 1);
        const double dv = -dense_div(*I, L, x, y, z);
        b0 += (1.0 - t) * dv;
        b1 += t * dv;
      }
      for (int o = 16; o > 0; o >>= 1) {
        b0 += __shfl_xor_sync(0xffffffffu, b0, o);
        b1 += __shfl_xor_sync(0xffffffffu, b1, o);
      }
    }
    if (lane == 0) {
      I->b[s0] = float(b0);
      I->b[s0 + L.nx] = float(b1);
    }
  }
  // Band samples, a thread each.
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < L.n; k += gridDim.x * blockDim.x) {
    int x, j, z, b;
    const bool act = sample_active(L, k, x, j, z, b);
    if (j < 2) continue;
    I->b[k] = (act && L.label[k]) ? float(-dense_div(*I, L, x, b + j - 2, z)) : 0.0f;
  }
}

// ---------------------------------------------------------- reductions
// Grid-stride partial sums in a fixed order, published per block; the last
// block to arrive folds them (deterministic for a fixed grid).
template <int N>
__device__ __forceinline__ bool reduce_grid(TInst* I, int stage, const double (&v)[N], const bool (&is_max)[N],
                                            double (&out)[N]) {
  __shared__ double sh[32];
  __shared__ int flag;
  double r[N];
#pragma unroll
  for (int s = 0; s < N; ++s) r[s] = is_max[s] ? block_max(v[s], sh) : block_sum(v[s], sh);
  if (threadIdx.x == 0)
#pragma unroll
    for (int s = 0; s < N; ++s) I->partial[s * kTGrid + blockIdx.x] = r[s];
  if (!arrive_last(&I->ctrl->arrive[stage], gridDim.x, &flag)) return false;
#pragma unroll
  for (int s = 0; s < N; ++s) out[s] = gather_slot(I->partial + s * kTGrid, 0, gridDim.x, is_max[s] ? 1 : 0, sh);
  return true;
}

// ------------------------------------------------------------------ CG
__global__ void k_tall_reset(TInst* I) {
  Ctrl* c = I->ctrl;
  c->liquid = 0;
  c->air = 0;
  c->nonfinite = 0;
  c->done = 0;
  c->candidate = 0;
  c->status = 0;
  c->converged = 0;
  c->iter = 0;
  *I->err = 0;
}

// r = b (cold start: x = 0), ||b||^2, ||b||_inf, thresholds.
__global__ void k_tall_cg_init(TInst* I, double rel_tol, double abs_tol, int max_iter, int true_every,
                               double rel_tol_inf) {
  const TLevel& L = I->lv[0];
  double bb = 0.0, bmax = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < L.n; k += gridDim.x * blockDim.x) {
    const float bv = L.label[k] ? I->b[k] : 0.0f;
    L.rhs[k] = bv;
    I->x[k] = 0.0f;
    I->xlo[k] = 0.0f;
    I->d[k] = 0.0f;
    bb += double(bv) * bv;
    bmax = fmax(bmax, fabs(double(bv)));
  }
  const double v[2] = {bb, bmax};
  const bool mx[2] = {false, true};
  double o[2];
  if (reduce_grid<2>(I, 0, v, mx, o) && threadIdx.x == 0) {
    Ctrl* c = I->ctrl;
    c->anchored = 1;
    c->bmean = 0.0;
    c->bb = o[0];
    c->rr = o[0];
    c->rr_true = o[0];
    const double thr = fmax(abs_tol, rel_tol * sqrt(o[0]));
    c->thr2 = thr * thr;
    c->bmax = o[1];
    c->rmax = o[1];
    c->thr_inf = rel_tol_inf > 0 ? rel_tol_inf * o[1] : 0.0;
    c->iter = 0;
    c->max_iter = max_iter;
    c->true_every = true_every;
    c->first = 1;
    c->candidate = 0;
    c->converged = 0;
    c->done = 0;
    c->status = FLUID_PP_OK;
    c->dsel = 0;
    set_sigma(c, o[0]);
    if (c->nonfinite) {
      c->done = 1;
      c->status = FLUID_PP_NONFINITE;
    } else if (*I->err) {
      c->done = 1;
      c->status = FLUID_PP_UNSUPPORTED;
    } else if (c->liquid == 0 || o[0] <= c->thr2) {
      c->done = 1;
      c->converged = 1;
    }
  }
}

// gamma = r . z
__global__ void k_tall_dot(TInst* I) {
  const Ctrl* c = I->ctrl;
  if (c->done) return;
  const TLevel& L = I->lv[0];
  double rz = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < L.n; k += gridDim.x * blockDim.x)
    if (L.label[k]) rz += double(L.rhs[k]) * double(L.z[k]);
  const double v[1] = {rz};
  const bool mx[1] = {false};
  double o[1];
  if (reduce_grid<1>(I, 1, v, mx, o) && threadIdx.x == 0) finish_gamma(I->ctrl, o[0], 0.0, 0.0);
}

// d = z + beta d
__global__ void k_tall_dir(TInst* I) {
  const Ctrl* c = I->ctrl;
  if (c->done) return;
  const float beta = float(c->beta);
  const TLevel& L = I->lv[0];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < L.n; k += gridDim.x * blockDim.x)
    I->d[k] = L.label[k] ? (beta == 0.0f ? L.z[k] : L.z[k] + beta * I->d[k]) : 0.0f;
}

// d = d on liquid samples, 0 elsewhere (the operator apply reads d without
// label tests).
__global__ void k_tall_mask_d(TInst* I) {
  const TLevel& L = I->lv[0];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < L.n; k += gridDim.x * blockDim.x)
    if (!L.label[k]) I->d[k] = 0.0f;
}

// q = A d, delta = d . q
__global__ void k_tall_spmv(TInst* I) {
  const Ctrl* c = I->ctrl;
  if (c->done) return;
  const TLevel& L = I->lv[0];
  double dq = 0.0;
  auto put = [&](int k, bool liq, double av, float dk) {
    const float q = liq ? float(av) : 0.0f;
    if (liq) dq += double(dk) * double(q);
    I->q[k] = q;
  };
  const long long items = apply_items(L.ncol, L.band, kApplyGroup);
  for (long long it = blockIdx.x * blockDim.x + threadIdx.x; it < items; it += gridDim.x * blockDim.x) {
    if (it < L.ncol) {
      tall_pair_apply(L, int(it), I->d, put);
    } else {
      band_rows_apply<kApplyGroup>(L, int(it - L.ncol), I->d, [](int) { return 0.0f; },
                                   [&](int k, bool liq, double av, float dk, float) { put(k, liq, av, dk); });
    }
  }
  const double v[1] = {dq};
  const bool mx[1] = {false};
  double o[1];
  if (reduce_grid<1>(I, 2, v, mx, o) && threadIdx.x == 0) finish_delta(I->ctrl, o[0]);
}

// x += alpha d (double-single), r -= alpha q
__global__ void k_tall_update(TInst* I) {
  const Ctrl* c = I->ctrl;
  if (c->done) return;
  const double alpha = c->alpha;
  const float af = float(alpha);
  const TLevel& L = I->lv[0];
  double rr = 0.0, mr = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < L.n; k += gridDim.x * blockDim.x) {
    if (!L.label[k]) continue;
    const double xv = double(I->x[k]) + double(I->xlo[k]) + alpha * double(I->d[k]);
    const float hi = float(xv);
    I->x[k] = hi;
    I->xlo[k] = float(xv - double(hi));
    const float rv = L.rhs[k] - af * I->q[k];
    L.rhs[k] = rv;
    rr += double(rv) * rv;
    mr = fmax(mr, fabs(double(rv)));
  }
  const double v[2] = {rr, mr};
  const bool mx[2] = {false, true};
  double o[2];
  if (reduce_grid<2>(I, 3, v, mx, o) && threadIdx.x == 0) finish_update(I->ctrl, o[0], o[1]);
}

// float64 r = b - A x with the double-single x
__global__ void k_tall_true(TInst* I) {
  const Ctrl* c = I->ctrl;
  if (c->done || (!c->candidate && !(c->true_every > 0 && c->iter % c->true_every == 0))) return;
  const TLevel& L = I->lv[0];
  double rr = 0.0, mr = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < L.n; k += gridDim.x * blockDim.x) {
    if (!L.label[k]) continue;
    int x, j, z, b;
    sample_active(L, k, x, j, z, b);
    const int col = x + L.nx * z;
    auto X = [&](int s) { return double(I->x[s]) + double(I->xlo[s]); };
    // the float64 operator (the assembly's values, band weights unrounded)
    double s = L.diag64[k] * X(k);
    if (j >= 2) {
      band_entries(L, x, j, z, b, [&](int sn, double w) { s += w * X(sn); });
    } else {
      const int nrow = 2 * L.ncol, row = 2 * col + j;
      s += L.a0164[col] * X(sidx(L, x, 1 - j, z));
      for (int e = 0; e < kTallW; ++e) s += L.tval64[e * nrow + row] * X(L.tidx[e * nrow + row]);
    }
    const double rv = double(I->b[k]) - s;
    L.rhs[k] = float(rv);
    rr += rv * rv;
    mr = fmax(mr, fabs(rv));
  }
  const double v[2] = {rr, mr};
  const bool mx[2] = {false, true};
  double o[2];
  if (reduce_grid<2>(I, 4, v, mx, o) && threadIdx.x == 0) finish_true(I->ctrl, o[0], o[1]);
}

// Loop condition of the iteration graph: one more iteration while the solve
// is not done and fewer than loop[1] iterations have run.
__global__ void k_tall_loop_cond(const TInst* I, unsigned* loop, cudaGraphConditionalHandle handle) {
  const unsigned c = loop[0] + 1;
  loop[0] = c;
  cudaGraphSetConditional(handle, (!I->ctrl->done && c < loop[1]) ? 1u : 0u);
}

__global__ void k_tall_loop_reset(unsigned* loop, unsigned cap) {
  loop[0] = 0u;
  loop[1] = cap;
}

// ------------------------------------------------------------------ V-cycle
// Each V-cycle stage is a device function over the samples t0, t0 + ts, ...;
// the grid kernels call it with the grid's threads, the single-CTA block for
// the small levels (k_tall_vblock) with the CTA's.
template <class S>
__device__ __forceinline__ void tv_zero(TInst* I, int l, int t0, int ts) {
  const TLevel& L = I->lv[l];
  S* z = stor<S>(L.z);
  for (int k = t0; k < L.n; k += ts) z[k] = fromf<S>(0.0f);
}

// The start of a grid level's pre-smoothing in one pass: with from_acc the
// restricted right-hand side out of the fixed-point accumulators (as
// tv_restrict_finish), then z = 0 everywhere except the liquid red band
// rows, which take rhs / diag: the red band sweep from zero, whose neighbour
// terms all vanish.  Same values as tv_restrict_finish + tv_zero +
// tv_smooth_band(colour 0).
template <class S>
__device__ __forceinline__ void tv_start(TInst* I, int l, int from_acc, int t0, int ts) {
  const TLevel& L = I->lv[l];
  S* z = stor<S>(L.z);
  S* rhs = stor<S>(L.rhs);
  for (int k = t0; k < L.n; k += ts) {
    const bool liq = L.label[k] != 0;
    float rh;
    if (from_acc) {
      const long long a = (long long)L.acc[k];
      const S r = fromf<S>(liq ? float(double(a) / kFix) : 0.0f);
      rhs[k] = r;
      L.acc[k] = 0ull;
      rh = tof(r);
    } else {
      rh = tof(rhs[k]);
    }
    int x, j, zc, b;
    const bool act = sample_active(L, k, x, j, zc, b);
    const bool red = j >= 2 && act && j - 2 < L.band && ((x + (b + j - 2) + zc) & 1) == 0;
    z[k] = fromf<S>(red && liq ? (rh - 0.0f) / L.diag[k] : 0.0f);
  }
}

// Band colour sweeps run over work items of G consecutive band rows of one
// column (item = column + ncol * group, so a warp's lanes are adjacent
// columns): an item loads its column's base and the four lateral bases once,
// then issues every load of its G / 2 rows of the colour before the first
// update.  Rows of one colour never neighbour each other, so the loads see no
// update of the same sweep.  Grid launches take kBandGroup rows per item, the
// single-CTA block (64 registers a thread) kBlockBandGroup.
constexpr int kBandGroup = 4;
constexpr int kBlockBandGroup = 2;

template <int G, class S>
__device__ __forceinline__ void tv_smooth_band(TInst* I, int l, int colour, int t0, int ts) {
  static_assert(G % 2 == 0, "a band row group holds both colours");
  const TLevel& L = I->lv[l];
  const VecView<S> Z = view<S>(L.z), Rh = view<S>(L.rhs);
  S* zw = stor<S>(L.z);
  constexpr int R = G / 2;
  const int items = ((L.band + G - 1) / G) * L.ncol;
  for (int it = t0; it < items; it += ts) {
    const int g = int(divq(unsigned(it), L.mnc));
    BandCol c;
    band_col(L, it - g * L.ncol, c);
    const int jb0 = g * G + ((colour + c.x + c.b + c.z) & 1);   // (x + y + z) & 1 == colour
    float vv[R][10], rh[R], dg[R];
    bool act[R], liq[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int jb = jb0 + 2 * r;
      const int k = sidx(L, c.x, jb + 2, c.z);
      act[r] = jb < L.band && c.b + jb < L.fine_ny;
      liq[r] = false;
      rh[r] = dg[r] = 0.0f;
      if (act[r]) {
        liq[r] = L.label[k] != 0;
        rh[r] = Rh[k];
        dg[r] = L.diag[k];
        band_row_loads(L, c, jb, k, Z, vv[r]);
      }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (!act[r]) continue;
      const int jb = jb0 + 2 * r;
      const int k = sidx(L, c.x, jb + 2, c.z);
      zw[k] = fromf<S>(liq[r] ? (rh[r] - band_row_off(L, c, jb, vv[r])) / dg[r] : 0.0f);
    }
  }
}

// One colour of the block Gauss-Seidel sweep: 0/1 band cells with (x + y + z)
// even/odd (items of G band rows), 2/3 tall blocks of columns with (x + z)
// even/odd.
template <int G, class S>
__device__ __forceinline__ void tv_smooth(TInst* I, int l, int colour, int t0, int ts) {
  const TLevel& L = I->lv[l];
  if (colour < 2) {
    tv_smooth_band<G, S>(I, l, colour, t0, ts);
  } else {
    const VecView<S> Z = view<S>(L.z), Rh = view<S>(L.rhs);
    S* zw = stor<S>(L.z);
    for (int c = t0; c < L.ncol; c += ts) {
      const int z = int(divq(unsigned(c), L.mnx)), x = c - z * L.nx;
      if (((x + z) & 1) != colour - 2) continue;
      const int s0 = sidx(L, x, 0, z), s1 = sidx(L, x, 1, z);
      if (!L.label[s0]) {
        zw[s0] = zw[s1] = fromf<S>(0.0f);
        continue;
      }
      double o0, o1;
      tall_off_pair(L, c, Z, o0, o1);
      const double r0 = double(Rh[s0]) - o0;
      const double r1 = double(Rh[s1]) - o1;
      const double a00 = L.diag[s0], a11 = L.diag[s1], a01 = L.a01[c];
      const double det = a00 * a11 - a01 * a01;
      zw[s0] = fromf<S>(float((a11 * r0 - a01 * r1) / det));
      zw[s1] = fromf<S>(float((a00 * r1 - a01 * r0) / det));
    }
  }
}

// res = scale (rhs - A z); level 0 scales by sigma.  Work items as in the
// operator apply, G band rows each.
template <int G, class S>
__device__ __forceinline__ void tv_residual(TInst* I, int l, int t0, int ts) {
  const TLevel& L = I->lv[l];
  const double scale = l == 0 ? I->ctrl->sigma : 1.0;
  const VecView<S> Z = view<S>(L.z), Rh = view<S>(L.rhs);
  S* res = stor<S>(L.res);
  const long long items = apply_items(L.ncol, L.band, G);
  for (long long it = t0; it < items; it += ts) {
    if (it < L.ncol) {
      tall_pair_apply(L, int(it), Z, [&](int k, bool liq, double av, float) {
        res[k] = fromf<S>(liq ? float(scale * (double(Rh[k]) - av)) : 0.0f);
      });
    } else {
      band_rows_apply<G>(L, int(it - L.ncol), Z, [&](int k) { return Rh[k]; },
                         [&](int k, bool liq, float av, float, float rhs) {
                           res[k] = fromf<S>(liq ? float(scale * double(rhs - av)) : 0.0f);
                         });
    }
  }
}

// acc_c += 1/2 P^T res_f in 32.32 fixed point, each term rounded from float
// (order-independent integer sums; sums
// that land on samples that are not liquid are dropped by tv_restrict_finish,
// which reads only liquid accumulators and clears them all).  The
// fine sample at dense (x, row y, z) takes the 2 x 2 x 2 trilinear taps of the
// coarse dense cells around it (taps2: a dropped tap has weight 0); a coarse
// tall cell passes its share to the column's two samples (1 - t, t), a coarse
// band cell to its sample, air cells take nothing.
template <class SF>
__device__ __forceinline__ void tv_restrict(TInst* I, int l, int t0, int ts) {
  const TLevel& F = I->lv[l];
  const TLevel& C = I->lv[l + 1];
  const VecView<SF> Res = view<SF>(F.res);
  constexpr float kFixF = 4294967296.0f;
  for (int k = t0; k < F.n; k += ts) {
    int x, j, z;
    decode(F, k, x, j, z);
    const bool liq = F.label[k] != 0;   // the three loads issue together
    const float r = Res[k];
    const int b = F.bases[x + F.nx * z];
    if (!liq || r == 0.0f) continue;
    int cx[2], cy[2], cz[2];
    float wx[2], wy[2], wz[2];
    taps2(x, 2, C.nx, cx, wx);
    taps2(sample_row(j, b), 2, C.fine_ny, cy, wy);
    taps2(z, 2, C.nz, cz, wz);
    const float hr = 0.5f * r;
    int bc[2][2];
#pragma unroll
    for (int c2 = 0; c2 < 2; ++c2)
#pragma unroll
      for (int c0 = 0; c0 < 2; ++c0) bc[c2][c0] = C.bases[cx[c0] + C.nx * cz[c2]];
#pragma unroll
    for (int c2 = 0; c2 < 2; ++c2)
#pragma unroll
      for (int c0 = 0; c0 < 2; ++c0) {
        const float wxz = wx[c0] * wz[c2];   // products of quarters: exact
        if (wxz == 0.0f) continue;
        const int B = bc[c2][c0];
        const float rB = __frcp_rn(float(B - 1));
        const int s0 = sidx(C, cx[c0], 0, cz[c2]);
        long long t0acc = 0, t1acc = 0;   // the column's tall samples, summed over the y taps
#pragma unroll
        for (int c1 = 0; c1 < 2; ++c1) {
          if (wy[c1] == 0.0f) continue;
          const int Y = cy[c1];
          const float v = hr * (wxz * wy[c1]) * kFixF;
          if (Y < B) {
            const float t = float(Y) * rB;
            t0acc += __float2ll_rn(v * (1.0f - t));
            t1acc += __float2ll_rn(v * t);
          } else if (Y < B + C.band) {
            atomicAdd(&C.acc[s0 + C.nx * (Y - B + 2)], (unsigned long long)__float2ll_rn(v));
          }
        }
        if (t0acc != 0) atomicAdd(&C.acc[s0], (unsigned long long)t0acc);
        if (t1acc != 0) atomicAdd(&C.acc[s0 + C.nx], (unsigned long long)t1acc);
      }
  }
}

template <class SC>
__device__ __forceinline__ void tv_restrict_finish(TInst* I, int l, int t0, int ts) {
  const TLevel& C = I->lv[l];
  SC* rhs = stor<SC>(C.rhs);
  for (int k = t0; k < C.n; k += ts) {
    const long long a = (long long)C.acc[k];
    rhs[k] = fromf<SC>(C.label[k] ? float(double(a) / kFix) : 0.0f);
    C.acc[k] = 0ull;
  }
}

// z_f += P z_c on liquid fine samples (the taps of tv_restrict, a coarse tall
// cell interpolating its column's two samples); into level 0 the sigma scale
// is undone.
template <class SF, class SC>
__device__ __forceinline__ void tv_prolong(TInst* I, int l, int t0, int ts) {
  const TLevel& F = I->lv[l];
  const TLevel& C = I->lv[l + 1];
  const VecView<SF> Zf = view<SF>(F.z);
  const VecView<SC> Zc = view<SC>(C.z);
  SF* zw = stor<SF>(F.z);
  const float unscale = l == 0 ? float(1.0 / I->ctrl->sigma) : 1.0f;
  for (int k = t0; k < F.n; k += ts) {
    int x, j, z;
    decode(F, k, x, j, z);
    const bool liq = F.label[k] != 0;   // the three loads issue together
    const float zf = Zf[k];
    const int b = F.bases[x + F.nx * z];
    if (!liq) continue;
    int cx[2], cy[2], cz[2];
    float wx[2], wy[2], wz[2];
    taps2(x, 2, C.nx, cx, wx);
    taps2(sample_row(j, b), 2, C.fine_ny, cy, wy);
    taps2(z, 2, C.nz, cz, wz);
    int bc[2][2];
#pragma unroll
    for (int c2 = 0; c2 < 2; ++c2)
#pragma unroll
      for (int c0 = 0; c0 < 2; ++c0) bc[c2][c0] = C.bases[cx[c0] + C.nx * cz[c2]];
    float s = 0.0f;
#pragma unroll
    for (int c2 = 0; c2 < 2; ++c2)
#pragma unroll
      for (int c1 = 0; c1 < 2; ++c1)
#pragma unroll
        for (int c0 = 0; c0 < 2; ++c0) {
          const float w = wx[c0] * wy[c1] * wz[c2];   // exact
          if (w == 0.0f) continue;
          const int B = bc[c2][c0], Y = cy[c1];
          const int s0 = sidx(C, cx[c0], 0, cz[c2]);
          float val = 0.0f;
          if (Y < B) {
            const float t = float(Y) * __frcp_rn(float(B - 1));
            val = (1.0f - t) * Zc[s0] + t * Zc[s0 + C.nx];
          } else if (Y < B + C.band) {
            val = Zc[s0 + C.nx * (Y - B + 2)];
          }
          s = fmaf(w, val, s);
        }
    zw[k] = fromf<SF>(fmaf(s, unscale, zf));
  }
}

// z = A^{-1} rhs on the coarsest level, a warp per row (threads t0 .. t0 + ts of one CTA).
__device__ __forceinline__ void tv_coarse_apply(TInst* I) {
  const TLevel& L = I->lv[I->nlev - 1];
  const int m = L.n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int i = warp; i < m; i += nw) {
    double s = 0.0;
    for (int j = lane; j < m; j += 32) s += I->coarse_inv[(long long)i * m + j] * (L.label[j] ? double(L.rhs[j]) : 0.0);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) L.z[i] = L.label[i] ? float(s) : 0.0f;
  }
}

#define TALL_GRID_KERNEL(name, tparams, call)                                               \
  template <tparams>                                                                         \
  __global__ void name(TInst* I, int l, int arg) {                                           \
    if (I->ctrl->done) return;                                                               \
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x, ts = gridDim.x * blockDim.x;      \
    (void)arg;                                                                               \
    call;                                                                                    \
  }
#define TALL_COMMA ,
TALL_GRID_KERNEL(k_tall_zero, class S, tv_zero<S>(I, l, t0, ts))
TALL_GRID_KERNEL(k_tall_start, class S, tv_start<S>(I, l, arg, t0, ts))
TALL_GRID_KERNEL(k_tall_smooth, class S, (tv_smooth<kBandGroup, S>(I, l, arg, t0, ts)))
TALL_GRID_KERNEL(k_tall_residual, class S, (tv_residual<kApplyGroup, S>(I, l, t0, ts)))
TALL_GRID_KERNEL(k_tall_restrict, class S, tv_restrict<S>(I, l, t0, ts))
TALL_GRID_KERNEL(k_tall_restrict_finish, class S, tv_restrict_finish<S>(I, l, t0, ts))
TALL_GRID_KERNEL(k_tall_prolong, class SF TALL_COMMA class SC, (tv_prolong<SF, SC>(I, l, t0, ts)))
#undef TALL_COMMA
#undef TALL_GRID_KERNEL

__global__ void k_tall_coarse_apply(TInst* I) {
  if (I->ctrl->done) return;
  tv_coarse_apply(I);
}

// Shared-memory layout of the block levels when they are held on chip: per
// level first .. nlev - 1 the float z, rhs and diag and the byte label of
// every sample, the int bases and float a01 of every column, each array
// 16-byte aligned.  The same walk sizes it on the host and carves it on the
// device.
constexpr size_t kVBlockSmemMax = 200 * 1024;

template <class Take>
__host__ __device__ inline void vblock_carve(TInst& W, int first, Take take) {
  for (int l = first; l < W.nlev; ++l) {
    TLevel& V = W.lv[l];
    V.z = static_cast<float*>(take(4 * size_t(V.n)));
    V.rhs = static_cast<float*>(take(4 * size_t(V.n)));
    V.diag = static_cast<float*>(take(4 * size_t(V.n)));
    V.label = static_cast<uint8_t*>(take(size_t(V.n)));
    V.bases = static_cast<int*>(take(4 * size_t(V.ncol)));
    V.a01 = static_cast<float*>(take(4 * size_t(V.ncol)));
    if (l > first) V.acc = static_cast<unsigned long long*>(take(8 * size_t(V.n)));
  }
}

// Copy of `bytes` between 16-byte aligned buffers by the CTA's threads, four
// 16-byte words in flight per thread.
__device__ __forceinline__ void cta_copy16(void* dst, const void* src, size_t bytes) {
  const uint4* s4 = static_cast<const uint4*>(src);
  uint4* d4 = static_cast<uint4*>(dst);
  const int n4 = int(bytes / 16), t0 = threadIdx.x, ts = blockDim.x;
  for (int i = t0; i < n4; i += 4 * ts) {
    uint4 v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (i + u * ts < n4) v[u] = s4[i + u * ts];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (i + u * ts < n4) d4[i + u * ts] = v[u];
  }
  const unsigned char* sb = static_cast<const unsigned char*>(src);
  unsigned char* db = static_cast<unsigned char*>(dst);
  for (size_t i = size_t(n4) * 16 + t0; i < bytes; i += ts) db[i] = sb[i];
}

// The small levels first .. nlev-1 of the V-cycle in one CTA: the same stages
// as the grid kernels, separated by barriers instead of launches (memory
// written before a barrier is visible to the CTA after it).  With on_chip
// the stages run on a shared-memory copy of the instance whose block-level z,
// rhs, diag, label, bases and a01 and the coarser levels' restriction
// accumulators live in shared memory (vblock_carve): the operator and the
// level-first rhs are loaded once, the level-first z is written back at the
// end; residuals, the tall-row couplings and the coarsest inverse stay in
// global memory.
__global__ void __launch_bounds__(1024) k_tall_vblock(TInst* I, int first, int on_chip) {
  if (I->ctrl->done) return;
  extern __shared__ __align__(16) unsigned char vsm[];
  __shared__ __align__(16) TInst SI;
  const int t0 = threadIdx.x, ts = blockDim.x, last = I->nlev - 1;
  TInst* W = I;
  if (on_chip) {
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(I);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(&SI);
    for (int w = t0; w < int(sizeof(TInst) / 8); w += ts) dst[w] = src[w];
    __syncthreads();
    if (t0 == 0) {
      size_t off = 0;
      vblock_carve(SI, first, [&](size_t bytes) {
        void* p = vsm + off;
        off += (bytes + 15) & ~size_t(15);
        return p;
      });
    }
    __syncthreads();
    for (int l = first; l <= last; ++l) {
      const TLevel& G = I->lv[l];
      const TLevel& V = SI.lv[l];
      cta_copy16(V.diag, G.diag, 4 * size_t(V.n));
      cta_copy16(V.label, G.label, size_t(V.n));
      cta_copy16(V.bases, G.bases, 4 * size_t(V.ncol));
      cta_copy16(V.a01, G.a01, 4 * size_t(V.ncol));
      if (l == first) cta_copy16(V.rhs, G.rhs, 4 * size_t(V.n));
      else
        for (int k = t0; k < V.n; k += ts) V.acc[k] = 0ull;   // cleared again by every restrict_finish
    }
    __syncthreads();
    W = &SI;
  }
  for (int l = first; l < last; ++l) {
    tv_zero<float>(W, l, t0, ts);
    __syncthreads();
    for (int c = 0; c < 4; ++c) {
      tv_smooth<kBlockBandGroup, float>(W, l, c, t0, ts);
      __syncthreads();
    }
    tv_residual<1, float>(W, l, t0, ts);
    __syncthreads();
    tv_restrict<float>(W, l, t0, ts);
    __syncthreads();
    tv_restrict_finish<float>(W, l + 1, t0, ts);
    __syncthreads();
  }
  tv_coarse_apply(W);
  __syncthreads();
  for (int l = last - 1; l >= first; --l) {
    tv_prolong<float, float>(W, l, t0, ts);
    __syncthreads();
    for (int c = 3; c >= 0; --c) {
      tv_smooth<kBlockBandGroup, float>(W, l, c, t0, ts);
      __syncthreads();
    }
  }
  if (on_chip) cta_copy16(I->lv[first].z, SI.lv[first].z, 4 * size_t(SI.lv[first].n));
}

// ------------------------------------------------------------------ finish
__device__ __forceinline__ double pressure_at(const TInst& I, const TLevel& L, int x, int y, int z) {
  const Rep r = rep_of(L, x, y, z);
  if (!r.liq) return 0.0;
  auto X = [&](int s) { return double(I.x[s]) + double(I.xlo[s]); };
  return r.n == 2 ? r.w0 * X(r.s0) + r.w1 * X(r.s1) : X(r.s0);
}

// Each sample's own +x/+y/+z faces: u -= (p_j - p_i) / theta at the sample's
// row; faces with no liquid side and wall faces are zero.  Pressure in Pa.
__global__ void k_tall_grad(TInst* I) {
  if (I->ctrl->status == FLUID_PP_NONFINITE) return;
  const TLevel& L = I->lv[0];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < L.n; k += gridDim.x * blockDim.x) {
    int x, j, z, b;
    const bool act = sample_active(L, k, x, j, z, b);
    if (!act) {
      I->u[k] = I->v[k] = I->w[k] = 0.0f;
      I->p_si[k] = 0.0f;
      continue;
    }
    const int y = sample_row(j, b);
    const Rep ri = rep_of(L, x, y, z);
    const double pi = pressure_at(*I, L, x, y, z);
    auto face = [&](float u, int xn, int yn, int zn, bool in) -> float {
      if (!in) return 0.0f;
      const Rep rn = rep_of(L, xn, yn, zn);
      if (!ri.liq && !rn.liq) return 0.0f;
      const double th = (ri.liq && rn.liq) ? 1.0 : (ri.liq ? ghost_theta_d(ri.phi, rn.phi) : ghost_theta_d(rn.phi, ri.phi));
      return float(double(u) - (pressure_at(*I, L, xn, yn, zn) - pi) / th);
    };
    const float un = face(I->u[k], x + 1, y, z, x + 1 < L.nx);
    const float vn = face(I->v[k], x, y + 1, z, y + 1 < L.fine_ny);
    const float wn = face(I->w[k], x, y, z + 1, z + 1 < L.nz);
    I->p_si[k] = L.label[k] ? float((double(I->x[k]) + double(I->xlo[k])) * double(I->pscale)) : 0.0f;
    I->u[k] = un;
    I->v[k] = vn;
    I->w[k] = wn;
  }
}

// Divergence receipts over the liquid band cells the packed faces represent
// exactly: rows inside the bands of the column and of its four neighbours
// (every face of such a cell is a sample's own face or a tall cell's top
// face).  max |div| and sum div^2 of the current packed velocities.
__global__ void k_tall_receipt(TInst* I, int slot) {
  const TLevel& L = I->lv[0];
  double mx = 0.0, ss = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < L.n; k += gridDim.x * blockDim.x) {
    int x, j, z, b;
    const bool act = sample_active(L, k, x, j, z, b);
    if (j < 2 || !act || !L.label[k]) continue;
    int lo = b, hi = b;   // rows [lo, hi + band) are inside every band
    auto nb = [&](int c) {
      lo = max(lo, L.bases[c]);
      hi = min(hi, L.bases[c]);
    };
    if (x > 0) nb(x - 1 + L.nx * z);
    if (x + 1 < L.nx) nb(x + 1 + L.nx * z);
    if (z > 0) nb(x + L.nx * (z - 1));
    if (z + 1 < L.nz) nb(x + L.nx * (z + 1));
    const int y = b + j - 2;
    if (y < lo || y >= hi + L.band) continue;
    const double dv = dense_div(*I, L, x, b + j - 2, z);
    mx = fmax(mx, fabs(dv));
    ss += dv * dv;
  }
  const double v[2] = {mx, ss};
  const bool m2[2] = {true, false};
  double o[2];
  if (reduce_grid<2>(I, 5, v, m2, o) && threadIdx.x == 0) {
    I->ctrl->red[2 * slot] = o[0];
    I->ctrl->red[2 * slot + 1] = o[1];
  }
}

}  // namespace tall
}  // namespace fpp

// ==================================================================== host
using namespace fpp;
using namespace fpp::tall;

struct fluid_pp_tall {
  fluid_pp_tall_config cfg{};
  TallPlan plan;
  cudaStream_t stream = nullptr;
  std::string err;
  char* arena = nullptr;
  TInst inst{};
  TInst* d_inst = nullptr;
  Ctrl* h_ctrl = nullptr;
  bool has_state = false;
  bool solving = false;   // between fluid_pp_tall_project_begin and _end
  bool solved = false;    // the CG loop reported done
  int it = 0, cap = 0;    // CG iterations launched, iteration cap (+2 slack)
  // CUDA graphs of the CG iteration, captured once per handle (the launches
  // depend only on the hierarchy): x_body is one iteration (the sliced solve
  // replays it), x_loop a conditional WHILE node around it that ends on the
  // device when the solve is done or after d_loop[1] iterations.
  cudaGraph_t g_body = nullptr, g_loop = nullptr;
  cudaGraphExec_t x_body = nullptr, x_loop = nullptr;
  unsigned* d_loop = nullptr;   // [0] iterations run, [1] iteration cap
  bool graphs_tried = false;
  int pre = 1, post = 1;   // red-black block sweeps on the grid levels (the block levels sweep once)
  int set_error(int code, const std::string& m) {
    err = m;
    return code;
  }
};

namespace {

int grid_for(long long n) { return int(std::max(1LL, std::min<long long>((n + kTB - 1) / kTB, kTGrid))); }
// Grid of a band colour sweep: one thread per (column, kBandGroup rows) item.
int grid_band(const TLevel& L) { return grid_for(1LL * ((L.band + kBandGroup - 1) / kBandGroup) * L.ncol); }

size_t up256(size_t v) { return (v + 255) / 256 * 256; }

// Levels below kTallBlockSamples run in the single-CTA block; the finer ones
// launch one grid kernel per stage.
constexpr long long kTallBlockSamples = 8192;

// Dynamic shared memory of the block levels held on chip, 0 if they do not fit.
size_t vblock_smem_bytes(const TInst& I, int first) {
  TInst W = I;
  size_t off = 0;
  vblock_carve(W, first, [&](size_t bytes) {
    off += (bytes + 15) & ~size_t(15);
    return static_cast<void*>(nullptr);
  });
  return off <= kVBlockSmemMax ? off : 0;
}

// Shared-memory limits of the tall kernels, set once per device: the largest
// coarsest level any tall grid can have and the block levels held on chip.
// Setting a kernel's attribute while another thread launches that kernel is a
// race, so later handle creations (which may run beside other handles'
// solves) never touch them again.
std::mutex g_tall_cfg_mutex;
bool g_tall_cfg_done[64] = {};

cudaError_t configure_tall_kernels() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_tall_cfg_mutex);
  if (dev >= 0 && dev < 64 && g_tall_cfg_done[dev]) return cudaSuccess;
  e = cudaFuncSetAttribute((const void*)k_tall_factor, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           int(kMaxCoarse * kMaxCoarse * sizeof(double)));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)k_tall_vblock, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(kVBlockSmemMax));
  if (e == cudaSuccess && dev >= 0 && dev < 64) g_tall_cfg_done[dev] = true;
  return e;
}

int tall_first_block(const TallPlan& plan) {
  const int L = int(plan.levels.size());
  for (int l = 1; l < L; ++l)
    if (plan.levels[l].samples() <= kTallBlockSamples) return l;
  return L - 1;
}

// The V-cycle's launches: grid levels 0 .. first - 1 (level 0 in float,
// levels 1 .. first - 1 in the storage type S), then the block levels in one
// CTA, then back up.
template <class S>
void launch_vcycle_t(fluid_pp_tall* T, int first) {
  TInst& I = T->inst;
  cudaStream_t s = T->stream;
  TInst* D = T->d_inst;
  // grid level l's vectors are float on level 0, S above it; the block levels are float
  // zero + (restricted rhs) + red band sweep from zero, in one launch
  auto start = [&](int l, int g) {
    if (l == 0) k_tall_start<float><<<g, kTB, 0, s>>>(D, l, 0);
    else k_tall_start<S><<<g, kTB, 0, s>>>(D, l, 1);
  };
  auto smooth = [&](int l, int g, int colour) {
    if (l == 0) k_tall_smooth<float><<<g, kTB, 0, s>>>(D, l, colour);
    else k_tall_smooth<S><<<g, kTB, 0, s>>>(D, l, colour);
  };
  for (int l = 0; l < first; ++l) {
    const int g = grid_for(I.lv[l].n), gc = grid_for(I.lv[l].ncol), gb = grid_band(I.lv[l]);
    const int gr = grid_for(apply_items(I.lv[l].ncol, I.lv[l].band, kApplyGroup));
    const int gf = grid_for(I.lv[l + 1].n);
    start(l, g);
    smooth(l, gb, 1);
    smooth(l, gc, 2);
    smooth(l, gc, 3);
    for (int k = 1; k < T->pre; ++k)
      for (int c = 0; c < 4; ++c) smooth(l, c < 2 ? gb : gc, c);
    if (l == 0) {
      k_tall_residual<float><<<gr, kTB, 0, s>>>(D, l, 0);
      k_tall_restrict<float><<<g, kTB, 0, s>>>(D, l, 0);
    } else {
      k_tall_residual<S><<<gr, kTB, 0, s>>>(D, l, 0);
      k_tall_restrict<S><<<g, kTB, 0, s>>>(D, l, 0);
    }
    // the next grid level finishes its rhs in its start pass; the block levels here
    if (l + 1 >= first) k_tall_restrict_finish<float><<<gf, kTB, 0, s>>>(D, l + 1, 0);
  }
  const size_t sm = vblock_smem_bytes(I, first);
  k_tall_vblock<<<1, 1024, sm, s>>>(D, first, sm > 0 ? 1 : 0);
  for (int l = first - 1; l >= 0; --l) {
    const int g = grid_for(I.lv[l].n), gc = grid_for(I.lv[l].ncol), gb = grid_band(I.lv[l]);
    const bool fine_s = l > 0, coarse_s = l + 1 < first;
    if (!fine_s && !coarse_s) k_tall_prolong<float, float><<<g, kTB, 0, s>>>(D, l, 0);
    else if (!fine_s) k_tall_prolong<float, S><<<g, kTB, 0, s>>>(D, l, 0);
    else if (!coarse_s) k_tall_prolong<S, float><<<g, kTB, 0, s>>>(D, l, 0);
    else k_tall_prolong<S, S><<<g, kTB, 0, s>>>(D, l, 0);
    for (int k = 0; k < T->post; ++k)
      for (int c = 3; c >= 0; --c) smooth(l, c < 2 ? gb : gc, c);
  }
}

void launch_vcycle(fluid_pp_tall* T, int first) {
  switch (T->cfg.precision) {
    case FLUID_PP_FP16: launch_vcycle_t<__half>(T, first); break;
    case FLUID_PP_BF16: launch_vcycle_t<__nv_bfloat16>(T, first); break;
    default: launch_vcycle_t<float>(T, first);
  }
}

// One CG iteration on the handle's stream: the V-cycle (or the dense coarsest
// apply of a single-level hierarchy), gamma, direction, A d, update, float64
// true residual.
void launch_iteration(fluid_pp_tall* T) {
  TInst& I = T->inst;
  cudaStream_t s = T->stream;
  const int g0 = grid_for(I.lv[0].n);
  if (I.nlev > 1) {
    launch_vcycle(T, tall_first_block(T->plan));
  } else {
    k_tall_coarse_apply<<<1, 1024, 0, s>>>(T->d_inst);
  }
  k_tall_dot<<<g0, kTB, 0, s>>>(T->d_inst);
  k_tall_dir<<<g0, kTB, 0, s>>>(T->d_inst);
  k_tall_spmv<<<g0, kTB, 0, s>>>(T->d_inst);
  k_tall_update<<<g0, kTB, 0, s>>>(T->d_inst);
  k_tall_true<<<g0, kTB, 0, s>>>(T->d_inst);
}

void destroy_tall_graphs(fluid_pp_tall* T) {
  for (cudaGraphExec_t* x : {&T->x_body, &T->x_loop})
    if (*x) {
      cudaGraphExecDestroy(*x);
      *x = nullptr;
    }
  for (cudaGraph_t* g : {&T->g_body, &T->g_loop})
    if (*g) {
      cudaGraphDestroy(*g);
      *g = nullptr;
    }
}

// Captures the iteration graphs once; on any failure the handle keeps direct
// launches (same kernels, same order, same bits).
void ensure_tall_graphs(fluid_pp_tall* T) {
  if (T->graphs_tried) return;
  T->graphs_tried = true;
  cudaStream_t cs = nullptr;
  if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  cudaStream_t saved = T->stream;
  T->stream = cs;
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    launch_iteration(T);
    e = cudaStreamEndCapture(cs, &T->g_body);
  }
  cudaGraphConditionalHandle handle{};
  cudaGraph_t body = nullptr;
  if (e == cudaSuccess) e = cudaGraphCreate(&T->g_loop, 0);
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&handle, T->g_loop, 1, cudaGraphCondAssignDefault);
  if (e == cudaSuccess) {
    cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};
    p.conditional.handle = handle;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, T->g_loop, nullptr, 0, &p);
    if (e == cudaSuccess) body = p.conditional.phGraph_out[0];
  }
  if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    launch_iteration(T);
    k_tall_loop_cond<<<1, 1, 0, cs>>>(T->d_inst, T->d_loop, handle);
    e = cudaStreamEndCapture(cs, &body);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&T->x_body, T->g_body, 0);
  if (e == cudaSuccess) e = cudaGraphInstantiate(&T->x_loop, T->g_loop, 0);
  T->stream = saved;
  cudaStreamDestroy(cs);
  if (e != cudaSuccess) {
    destroy_tall_graphs(T);
    cudaGetLastError();
  }
}

void launch_setup(fluid_pp_tall* T) {
  TInst& I = T->inst;
  cudaStream_t s = T->stream;
  k_tall_reset<<<1, 1, 0, s>>>(T->d_inst);
  k_tall_label<<<grid_for(I.lv[0].n), kTB, 0, s>>>(T->d_inst);
  for (int l = 0; l + 1 < I.nlev; ++l) {
    k_tall_coarsen<<<grid_for(I.lv[l + 1].n), kTB, 0, s>>>(T->d_inst, l);
    k_tall_coarse_labels<<<grid_for(I.lv[l + 1].n), kTB, 0, s>>>(T->d_inst, l + 1);
  }
  for (int l = 0; l < I.nlev; ++l) {
    k_tall_assemble_band<<<grid_for(I.lv[l].n), kTB, 0, s>>>(T->d_inst, l);
    k_tall_assemble_tall<<<grid_for(I.lv[l].ncol), kTB, 0, s>>>(T->d_inst, l);
  }
  const size_t m = size_t(I.coarse_m);
  k_tall_factor<<<1, 1024, m * m * sizeof(double), s>>>(T->d_inst);
  k_tall_rhs<<<grid_for(I.lv[0].n), kTB, 0, s>>>(T->d_inst);
}

// Device bytes of one tall handle's arena (every level's arrays and ELL rows,
// the packed state, the CG vectors, partials, coarsest inverse, control).
size_t tall_arena_size(const TallPlan& plan) {
  const int L = int(plan.levels.size());
  size_t bytes = 0;
  auto acc = [&](size_t b) { bytes = up256(bytes + b); };
  for (int l = 0; l < L; ++l) {
    const TallLevel& P = plan.levels[l];
    const size_t n = size_t(P.samples()), nc = size_t(P.nx) * P.nz;
    acc(4 * nc);                                   // bases
    acc(4 * n); acc(n); acc(4 * n); acc(4 * nc);   // phi label diag a01
    acc(4 * kTallW * 2 * nc); acc(4 * kTallW * 2 * nc);
    acc(4 * n); acc(4 * n); acc(4 * n);            // z rhs res
    if (l > 0) acc(8 * n);                         // acc
    if (l == 0) {                                  // float64 operator for the true residual
      acc(8 * n);
      acc(8 * nc);
      acc(8 * kTallW * 2 * nc);
    }
  }
  const size_t n0 = size_t(plan.levels[0].samples());
  for (int k = 0; k < 10; ++k) acc(4 * n0);        // vof u v w b x xlo d q p_si
  acc(sizeof(double) * kSlots * kTGrid);
  const size_t m = size_t(plan.levels[L - 1].samples());
  acc(sizeof(double) * m * m);
  acc(sizeof(Ctrl));
  acc(sizeof(int));
  return bytes;
}

int tall_create(const fluid_pp_tall_config* cfg, const int* bases, fluid_pp_tall** out) {
  if (!cfg || !bases || !out) return FLUID_PP_INVALID_ARG;
  if (cfg->precision != FLUID_PP_FP32 && cfg->precision != FLUID_PP_FP16 && cfg->precision != FLUID_PP_BF16) {
    fpp::set_global_error("unknown precision");
    return FLUID_PP_INVALID_ARG;
  }
  TallPlan plan = plan_tall(cfg->nx, cfg->nz, cfg->fine_ny, cfg->band, bases);
  if (!plan.ok) {
    fpp::set_global_error(plan.rejection ? plan.rejection : "tall layout rejected");
    return FLUID_PP_INVALID_ARG;
  }
  if (cudaSetDevice(cfg->device) != cudaSuccess) {
    fpp::set_global_error("cudaSetDevice failed");
    return FLUID_PP_CUDA;
  }
  auto T = std::make_unique<fluid_pp_tall>();
  T->cfg = *cfg;
  T->plan = plan;
  const int L = int(plan.levels.size());
  const size_t bytes = tall_arena_size(plan);
  const size_t n0 = size_t(plan.levels[0].samples());
  const size_t m = size_t(plan.levels[L - 1].samples());
  if (dev_alloc(reinterpret_cast<void**>(&T->arena), bytes) != cudaSuccess) {
    fpp::set_global_error("tall arena allocation failed");
    return FLUID_PP_OOM;
  }
  cudaMemset(T->arena, 0, bytes);
  size_t used = 0;
  auto take = [&](size_t b) {
    void* p = T->arena + used;
    used = up256(used + b);
    return p;
  };
  TInst& I = T->inst;
  std::memset(&I, 0, sizeof(I));
  I.nlev = L;
  I.h = cfg->h;
  I.rho = cfg->rho;
  for (int l = 0; l < L; ++l) {
    const TallLevel& P = plan.levels[l];
    TLevel& V = I.lv[l];
    V.nx = P.nx;
    V.nz = P.nz;
    V.fine_ny = P.fine_ny;
    V.band = P.band;
    V.P = P.P();
    V.n = int(P.samples());
    V.ncol = P.nx * P.nz;
    V.mnx = magic64(unsigned(V.nx));
    V.mP = magic64(unsigned(V.P));
    V.mnc = magic64(unsigned(V.ncol));
    const size_t n = size_t(V.n), nc = size_t(V.ncol);
    V.bases = static_cast<int*>(take(4 * nc));
    cudaMemcpy(V.bases, P.bases.data(), 4 * nc, cudaMemcpyHostToDevice);
    V.phi = static_cast<float*>(take(4 * n));
    V.label = static_cast<uint8_t*>(take(n));
    V.diag = static_cast<float*>(take(4 * n));
    V.a01 = static_cast<float*>(take(4 * nc));
    V.tidx = static_cast<int*>(take(4 * kTallW * 2 * nc));
    V.tval = static_cast<float*>(take(4 * kTallW * 2 * nc));
    V.z = static_cast<float*>(take(4 * n));
    V.rhs = static_cast<float*>(take(4 * n));
    V.res = static_cast<float*>(take(4 * n));
    V.acc = l > 0 ? static_cast<unsigned long long*>(take(8 * n)) : nullptr;
    V.diag64 = l == 0 ? static_cast<double*>(take(8 * n)) : nullptr;
    V.a0164 = l == 0 ? static_cast<double*>(take(8 * nc)) : nullptr;
    V.tval64 = l == 0 ? static_cast<double*>(take(8 * kTallW * 2 * nc)) : nullptr;
  }
  I.vof = static_cast<float*>(take(4 * n0));
  I.u = static_cast<float*>(take(4 * n0));
  I.v = static_cast<float*>(take(4 * n0));
  I.w = static_cast<float*>(take(4 * n0));
  I.b = static_cast<float*>(take(4 * n0));
  I.x = static_cast<float*>(take(4 * n0));
  I.xlo = static_cast<float*>(take(4 * n0));
  I.d = static_cast<float*>(take(4 * n0));
  I.q = static_cast<float*>(take(4 * n0));
  I.p_si = static_cast<float*>(take(4 * n0));
  I.partial = static_cast<double*>(take(sizeof(double) * kSlots * kTGrid));
  I.coarse_inv = static_cast<double*>(take(sizeof(double) * m * m));
  I.coarse_m = int(m);
  I.ctrl = static_cast<Ctrl*>(take(sizeof(Ctrl)));
  I.err = static_cast<int*>(take(sizeof(int)));
  cudaError_t e = dev_alloc(reinterpret_cast<void**>(&T->d_inst), sizeof(TInst));
  if (e == cudaSuccess) e = host_alloc(reinterpret_cast<void**>(&T->h_ctrl), sizeof(Ctrl));
  if (e == cudaSuccess) e = dev_alloc(reinterpret_cast<void**>(&T->d_loop), 2 * sizeof(unsigned));
  if (e == cudaSuccess) e = configure_tall_kernels();
  if (e != cudaSuccess) {
    fpp::set_global_error(std::string("tall setup: ") + cudaGetErrorString(e));
    dev_release(T->d_inst, T->stream);
    host_release(T->h_ctrl, T->stream);
    dev_release(T->d_loop, T->stream);
    dev_release(T->arena, T->stream);
    return FLUID_PP_OOM;
  }
  cudaMemcpy(T->d_inst, &I, sizeof(TInst), cudaMemcpyHostToDevice);
  *out = T.release();
  return FLUID_PP_OK;
}

}  // namespace

extern "C" {

int fluid_pp_tall_choose_base(int lowest_surface, int highest_surface, int fine_ny, int regular_layers,
                              int liquid_halo, int air_halo) {
  return tall_choose_base(lowest_surface, highest_surface, fine_ny, regular_layers, liquid_halo, air_halo);
}

int fluid_pp_tall_limit_bases(float* bases, int nx, int nz, int max_delta, int passes) {
  if (!bases || nx < 1 || nz < 1 || passes < 0) return FLUID_PP_INVALID_ARG;
  tall_limit_bases(bases, nx, nz, max_delta, passes);
  return FLUID_PP_OK;
}

int fluid_pp_tall_plan(int nx, int nz, int fine_ny, int band, const int* bases, int* level_count, int* level_shapes) {
  if (!bases || !level_count) return FLUID_PP_INVALID_ARG;
  TallPlan p = plan_tall(nx, nz, fine_ny, band, bases);
  if (!p.ok) {
    fpp::set_global_error(p.rejection ? p.rejection : "tall layout rejected");
    return FLUID_PP_INVALID_ARG;
  }
  *level_count = int(p.levels.size());
  if (level_shapes)
    for (size_t l = 0; l < p.levels.size(); ++l) {
      level_shapes[4 * l + 0] = p.levels[l].nx;
      level_shapes[4 * l + 1] = p.levels[l].fine_ny;
      level_shapes[4 * l + 2] = p.levels[l].nz;
      level_shapes[4 * l + 3] = p.levels[l].band;
    }
  return FLUID_PP_OK;
}

int fluid_pp_tall_create(const fluid_pp_tall_config* config, const int* bases, fluid_pp_tall** out) {
  return tall_create(config, bases, out);
}

void fluid_pp_tall_destroy(fluid_pp_tall* T) {
  if (!T) return;
  cudaSetDevice(T->cfg.device);
  destroy_tall_graphs(T);
  dev_release(T->d_inst, T->stream);
  host_release(T->h_ctrl, T->stream);
  dev_release(T->d_loop, T->stream);
  dev_release(T->arena, T->stream);
  delete T;
}

int fluid_pp_tall_set_graphs(fluid_pp_tall* T, int on) {
  if (!T) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(T->cfg.device);
  destroy_tall_graphs(T);
  T->graphs_tried = !on;   // off: no capture is attempted, every launch is direct
  return FLUID_PP_OK;
}

int fluid_pp_tall_set_stream(fluid_pp_tall* T, void* stream) {
  if (!T) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(T->cfg.device);
  const cudaStream_t next = static_cast<cudaStream_t>(stream);
  const cudaError_t e = fpp::order_streams(T->stream, next);
  if (e != cudaSuccess) return T->set_error(FLUID_PP_CUDA, cudaGetErrorString(e));
  T->stream = next;
  return FLUID_PP_OK;
}

static int tall_upload(fluid_pp_tall* T, const float* vof, const float* u, const float* v, const float* w,
                       cudaMemcpyKind kind) {
  if (!T || !vof || !u || !v || !w) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(T->cfg.device);
  const size_t n = size_t(T->inst.lv[0].n) * 4;
  cudaError_t e = cudaMemcpyAsync(T->inst.vof, vof, n, kind, T->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(T->inst.u, u, n, kind, T->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(T->inst.v, v, n, kind, T->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(T->inst.w, w, n, kind, T->stream);
  if (e != cudaSuccess) return T->set_error(FLUID_PP_CUDA, cudaGetErrorString(e));
  T->has_state = true;
  return FLUID_PP_OK;
}

int fluid_pp_tall_upload_state(fluid_pp_tall* T, const float* vof, const float* u, const float* v, const float* w) {
  return tall_upload(T, vof, u, v, w, cudaMemcpyHostToDevice);
}

int fluid_pp_tall_upload_state_device(fluid_pp_tall* T, const float* vof, const float* u, const float* v,
                                      const float* w) {
  return tall_upload(T, vof, u, v, w, cudaMemcpyDeviceToDevice);
}

static void tall_set_dt(fluid_pp_tall* T, float dt) {
  T->inst.dt = dt;
  T->inst.pscale = T->cfg.rho * T->cfg.h / dt;
  cudaMemcpyAsync(reinterpret_cast<char*>(T->d_inst) + offsetof(TInst, dt), &T->inst.dt, sizeof(float),
                  cudaMemcpyHostToDevice, T->stream);
  cudaMemcpyAsync(reinterpret_cast<char*>(T->d_inst) + offsetof(TInst, pscale), &T->inst.pscale, sizeof(float),
                  cudaMemcpyHostToDevice, T->stream);
}

}  // extern "C"

namespace {
// The grid levels' sweep counts of the next solve; the graphs hold the launch
// sequence, so a change drops them for a new capture.
bool tall_sweeps(fluid_pp_tall* T, const fluid_pp_solve_opts& o) {
  if (o.pre_sweeps < 1 || o.post_sweeps < 1 || o.pre_sweeps > 4 || o.post_sweeps > 4) return false;
  if (o.pre_sweeps != T->pre || o.post_sweeps != T->post) {
    T->pre = o.pre_sweeps;
    T->post = o.post_sweeps;
    if (T->x_body || T->x_loop) {
      cudaSetDevice(T->cfg.device);
      destroy_tall_graphs(T);
      T->graphs_tried = false;
    }
  }
  return true;
}
}  // namespace

extern "C" {

int fluid_pp_tall_project_begin(fluid_pp_tall* T, float dt, const fluid_pp_solve_opts* opts) {
  if (!T) return FLUID_PP_INVALID_ARG;
  if (!(dt > 0) || !std::isfinite(dt)) return T->set_error(FLUID_PP_INVALID_ARG, "dt must be positive and finite");
  if (!T->has_state) return T->set_error(FLUID_PP_INVALID_ARG, "state not uploaded");
  fluid_pp_solve_opts o{1e-6, 0.0, 200, 2, 2, 4, 0, 0.0, 0};   // two sweeps on the grid levels
  if (opts) o = *opts;
  if (!(o.rel_tol >= 0) || !(o.abs_tol >= 0) || o.max_iters < 1)
    return T->set_error(FLUID_PP_INVALID_ARG, "invalid solve options");
  if (o.cycle != 0) return T->set_error(FLUID_PP_INVALID_ARG, "the tall grid solves with the V-cycle only (cycle 0)");
  if (!tall_sweeps(T, o)) return T->set_error(FLUID_PP_INVALID_ARG, "tall sweeps: 1 to 4 before and after");
  cudaSetDevice(T->cfg.device);
  cudaStream_t s = T->stream;
  TInst& I = T->inst;
  tall_set_dt(T, dt);
  launch_setup(T);
  const int g0 = grid_for(I.lv[0].n);
  k_tall_receipt<<<g0, kTB, 0, s>>>(T->d_inst, 0);
  k_tall_cg_init<<<g0, kTB, 0, s>>>(T->d_inst, o.rel_tol, o.abs_tol, o.max_iters, o.true_residual_every,
                                    o.rel_tol_inf);
  T->solving = true;
  T->solved = false;
  T->it = 0;
  T->cap = o.max_iters + 2;
  return FLUID_PP_OK;
}

int fluid_pp_tall_project_continue(fluid_pp_tall* T, int max_iterations, int* finished) {
  if (!T || !finished) return FLUID_PP_INVALID_ARG;
  if (!T->solving) return T->set_error(FLUID_PP_INVALID_ARG, "no projection begun");
  cudaSetDevice(T->cfg.device);
  cudaStream_t s = T->stream;
  TInst& I = T->inst;
  int budget = max_iterations > 0 ? max_iterations : T->cap;
  ensure_tall_graphs(T);
  while (!T->solved && T->it < T->cap && budget > 0) {
    const int burst = std::min({4, T->cap - T->it, budget});
    for (int k = 0; k < burst; ++k) {
      if (T->x_body)
        cudaGraphLaunch(T->x_body, s);
      else
        launch_iteration(T);
    }
    T->it += burst;
    budget -= burst;
    cudaMemcpyAsync(T->h_ctrl, I.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      T->solving = false;
      return T->set_error(FLUID_PP_CUDA, std::string("tall solve: ") + cudaGetErrorString(e));
    }
    if (T->h_ctrl->done) T->solved = true;
  }
  *finished = (T->solved || T->it >= T->cap) ? 1 : 0;
  return FLUID_PP_OK;
}

int fluid_pp_tall_project_end(fluid_pp_tall* T, fluid_pp_receipt* receipt) {
  if (!T) return FLUID_PP_INVALID_ARG;
  if (!T->solving) return T->set_error(FLUID_PP_INVALID_ARG, "no projection begun");
  T->solving = false;
  cudaSetDevice(T->cfg.device);
  cudaStream_t s = T->stream;
  TInst& I = T->inst;
  const int g0 = grid_for(I.lv[0].n);
  k_tall_grad<<<g0, kTB, 0, s>>>(T->d_inst);
  k_tall_receipt<<<g0, kTB, 0, s>>>(T->d_inst, 1);
  cudaMemcpyAsync(T->h_ctrl, I.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return T->set_error(FLUID_PP_CUDA, std::string("tall finish: ") + cudaGetErrorString(e));
  const Ctrl& c = *T->h_ctrl;
  int status = c.status;
  if (!c.done && status == FLUID_PP_OK) status = FLUID_PP_NONCONVERGENCE;
  if (receipt) {
    std::memset(receipt, 0, sizeof(*receipt));
    receipt->status = status;
    receipt->iterations = c.iter;
    receipt->liquid_cells = c.liquid;
    receipt->levels = I.nlev;
    receipt->b_norm = std::sqrt(std::max(0.0, c.bb));
    receipt->rel_residual = c.bb > 0 ? std::sqrt(std::max(0.0, c.rr) / c.bb) : 0.0;
    receipt->true_rel_residual = c.bb > 0 ? std::sqrt(std::max(0.0, c.rr_true) / c.bb) : 0.0;
    const double hh = T->cfg.h;
    receipt->max_div_before = c.red[0] / hh;
    receipt->l2_div_before = std::sqrt(std::max(0.0, c.red[1]) * hh);
    receipt->max_div_after = c.red[2] / hh;
    receipt->l2_div_after = std::sqrt(std::max(0.0, c.red[3]) * hh);
  }
  if (status == FLUID_PP_UNSUPPORTED)
    T->err = "a tall row has more neighbour entries than its ELL width (column bases differ too much)";
  return status;
}

int fluid_pp_tall_project(fluid_pp_tall* T, float dt, const fluid_pp_solve_opts* opts, fluid_pp_receipt* receipt) {
  int rc = fluid_pp_tall_project_begin(T, dt, opts);
  if (rc != FLUID_PP_OK) return rc;
  ensure_tall_graphs(T);
  if (T->x_loop) {
    // the whole CG loop as one graph launch; it ends on the device
    k_tall_loop_reset<<<1, 1, 0, T->stream>>>(T->d_loop, unsigned(T->cap));
    cudaGraphLaunch(T->x_loop, T->stream);
    T->it = T->cap;
    return fluid_pp_tall_project_end(T, receipt);
  }
  int finished = 0;
  rc = fluid_pp_tall_project_continue(T, 0, &finished);
  if (rc != FLUID_PP_OK) return rc;
  return fluid_pp_tall_project_end(T, receipt);
}

int fluid_pp_tall_download(fluid_pp_tall* T, float* p, float* u, float* v, float* w) {
  if (!T) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(T->cfg.device);
  const size_t n = size_t(T->inst.lv[0].n) * 4;
  cudaError_t e = cudaSuccess;
  if (p) e = cudaMemcpyAsync(p, T->inst.p_si, n, cudaMemcpyDeviceToHost, T->stream);
  if (e == cudaSuccess && u) e = cudaMemcpyAsync(u, T->inst.u, n, cudaMemcpyDeviceToHost, T->stream);
  if (e == cudaSuccess && v) e = cudaMemcpyAsync(v, T->inst.v, n, cudaMemcpyDeviceToHost, T->stream);
  if (e == cudaSuccess && w) e = cudaMemcpyAsync(w, T->inst.w, n, cudaMemcpyDeviceToHost, T->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(T->stream);
  if (e != cudaSuccess) return T->set_error(FLUID_PP_CUDA, cudaGetErrorString(e));
  return FLUID_PP_OK;
}

int fluid_pp_tall_get_pressure(fluid_pp_tall* T, float* p) {
  if (!T || !p) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(T->cfg.device);
  const size_t n = size_t(T->inst.lv[0].n);
  std::vector<float> lo(n);
  cudaError_t e = cudaMemcpy(p, T->inst.x, 4 * n, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(lo.data(), T->inst.xlo, 4 * n, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return T->set_error(FLUID_PP_CUDA, cudaGetErrorString(e));
  for (size_t i = 0; i < n; ++i) p[i] = float(double(p[i]) + double(lo[i]));
  return FLUID_PP_OK;
}

int fluid_pp_tall_prepare(fluid_pp_tall* T, float dt) {
  if (!T || !T->has_state || !(dt > 0)) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(T->cfg.device);
  tall_set_dt(T, dt);
  launch_setup(T);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(T->stream);
  if (e != cudaSuccess) return T->set_error(FLUID_PP_CUDA, cudaGetErrorString(e));
  int err = 0;
  cudaMemcpy(&err, T->inst.err, sizeof(int), cudaMemcpyDeviceToHost);
  if (err) return T->set_error(FLUID_PP_UNSUPPORTED, "a tall row overflowed its ELL width");
  return FLUID_PP_OK;
}

int fluid_pp_tall_get_rhs(fluid_pp_tall* T, float* b) {
  if (!T || !b) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(T->cfg.device);
  cudaError_t e = cudaMemcpy(b, T->inst.b, size_t(T->inst.lv[0].n) * 4, cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? FLUID_PP_OK : T->set_error(FLUID_PP_CUDA, cudaGetErrorString(e));
}

int fluid_pp_tall_get_labels(fluid_pp_tall* T, int level, unsigned char* label) {
  if (!T || !label || level < 0 || level >= T->inst.nlev) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(T->cfg.device);
  cudaError_t e = cudaMemcpy(label, T->inst.lv[level].label, size_t(T->inst.lv[level].n), cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? FLUID_PP_OK : T->set_error(FLUID_PP_CUDA, cudaGetErrorString(e));
}

// out = A p on level 0 (after fluid_pp_tall_prepare); air entries of p ignored.
int fluid_pp_tall_apply_operator(fluid_pp_tall* T, const float* p, float* out) {
  if (!T || !p || !out) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(T->cfg.device);
  const size_t n = size_t(T->inst.lv[0].n);
  TInst& I = T->inst;
  cudaMemcpyAsync(I.d, p, 4 * n, cudaMemcpyHostToDevice, T->stream);
  k_tall_reset<<<1, 1, 0, T->stream>>>(T->d_inst);
  k_tall_mask_d<<<grid_for(n), kTB, 0, T->stream>>>(T->d_inst);
  k_tall_spmv<<<grid_for(n), kTB, 0, T->stream>>>(T->d_inst);
  cudaMemcpyAsync(out, I.q, 4 * n, cudaMemcpyDeviceToHost, T->stream);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(T->stream);
  return e == cudaSuccess ? FLUID_PP_OK : T->set_error(FLUID_PP_CUDA, cudaGetErrorString(e));
}

// Solves the assembled level-0 system A x = b for a caller-given b (finest-cell
// units; entries on air samples are ignored) with the projection's MGPCG, for
// parity tests that refine a float64 solution with the device solver; x is the
// solution in finest-cell units.  Labels, hierarchy and operator come from the
// uploaded state and dt, as in fluid_pp_tall_prepare.
int fluid_pp_tall_solve_rhs(fluid_pp_tall* T, float dt, const float* b, const fluid_pp_solve_opts* opts, float* x,
                            fluid_pp_receipt* receipt) {
  if (!T || !b || !x) return FLUID_PP_INVALID_ARG;
  if (!(dt > 0) || !std::isfinite(dt)) return T->set_error(FLUID_PP_INVALID_ARG, "dt must be positive and finite");
  if (!T->has_state) return T->set_error(FLUID_PP_INVALID_ARG, "state not uploaded");
  fluid_pp_solve_opts o{1e-6, 0.0, 200, 2, 2, 4, 0, 0.0, 0};   // two sweeps on the grid levels
  if (opts) o = *opts;
  if (!(o.rel_tol >= 0) || !(o.abs_tol >= 0) || o.max_iters < 1)
    return T->set_error(FLUID_PP_INVALID_ARG, "invalid solve options");
  if (o.cycle != 0) return T->set_error(FLUID_PP_INVALID_ARG, "the tall grid solves with the V-cycle only (cycle 0)");
  if (!tall_sweeps(T, o)) return T->set_error(FLUID_PP_INVALID_ARG, "tall sweeps: 1 to 4 before and after");
  cudaSetDevice(T->cfg.device);
  cudaStream_t s = T->stream;
  TInst& I = T->inst;
  tall_set_dt(T, dt);
  launch_setup(T);
  cudaMemcpyAsync(I.b, b, size_t(I.lv[0].n) * 4, cudaMemcpyHostToDevice, s);
  k_tall_cg_init<<<grid_for(I.lv[0].n), kTB, 0, s>>>(T->d_inst, o.rel_tol, o.abs_tol, o.max_iters,
                                                      o.true_residual_every, o.rel_tol_inf);
  T->solving = true;
  T->solved = false;
  T->it = 0;
  T->cap = o.max_iters + 2;
  int finished = 0;
  int rc = fluid_pp_tall_project_continue(T, 0, &finished);
  T->solving = false;
  if (rc != FLUID_PP_OK) return rc;
  const Ctrl& c = *T->h_ctrl;
  int status = c.status;
  if (!c.done && status == FLUID_PP_OK) status = FLUID_PP_NONCONVERGENCE;
  if (receipt) {
    std::memset(receipt, 0, sizeof(*receipt));
    receipt->status = status;
    receipt->iterations = c.iter;
    receipt->liquid_cells = c.liquid;
    receipt->levels = I.nlev;
    receipt->b_norm = std::sqrt(std::max(0.0, c.bb));
    receipt->rel_residual = c.bb > 0 ? std::sqrt(std::max(0.0, c.rr) / c.bb) : 0.0;
    receipt->true_rel_residual = c.bb > 0 ? std::sqrt(std::max(0.0, c.rr_true) / c.bb) : 0.0;
  }
  rc = fluid_pp_tall_get_pressure(T, x);
  return rc != FLUID_PP_OK ? rc : status;
}

const char* fluid_pp_tall_last_error(fluid_pp_tall* T) { return T ? T->err.c_str() : ""; }

int fluid_pp_tall_required_bytes(const fluid_pp_tall_config* cfg, const int* bases, unsigned long long* bytes) {
  if (!cfg || !bases || !bytes) return FLUID_PP_INVALID_ARG;
  TallPlan plan = plan_tall(cfg->nx, cfg->nz, cfg->fine_ny, cfg->band, bases);
  if (!plan.ok) {
    fpp::set_global_error(plan.rejection ? plan.rejection : "tall layout rejected");
    return FLUID_PP_INVALID_ARG;
  }
  *bytes = tall_arena_size(plan) + sizeof(TInst);
  return FLUID_PP_OK;
}

}  // extern "C"
