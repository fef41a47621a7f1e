// Sparse brick-atlas pressure projection: the default adaptive method's
// projection (lib/methods/adaptive-mass/webgpu-sparse-cm12-resident.ts, whose
// CPU statement is projectSparseAtlasVelocity,
// lib/methods/adaptive-mass/sparse-atlas-composite-projection.ts:978-1566)
// for atlases whose bricks all carry the finest resolution.
//
// Storage is brick-compact: only the present bricks of 8^3 cells exist; a
// brick table over the brick grid maps coordinates to slots (-1 absent).
// Cell i of the level-0 arrays is slot i / 512, local (x, y, z) = i % 512 in
// x-fastest order.  Faces are stored per brick as the dense MAC layout of the
// brick (u [8][8][9], v [8][9][8], w [9][8][8]: face f of an axis sits between
// local cells f - 1 and f), so the face between two present bricks has two
// copies: the lower brick's f = 8 copy is the one read, both are written.
//
// The system is the atlas's (buildLiquidSystem, :978-1168): a cell is liquid
// iff phi = 0.5 - rho <= 0; every face that is not a domain wall is a row:
// inside a brick, between present bricks (ports), or to an absent brick inside
// the domain (sparse-air rows, air phi 0.5); a row with a liquid and an air
// side weighs 1 / theta, theta = clamp(|phi_l| / max(|phi_l| + |phi_a|, 1e-12),
// 0.05, 1); b = G^T u over liquid cells; liquid components with no cut row are
// pure Neumann problems whose mean is projected out (projectNullspace,
// :1194-1213).  Units: finest cells, so the solve gives p' = p dt / (rho h)
// and a face takes u - jump / theta (pressureCorrection, :1263-1279); faces of
// rows without a liquid side become 0 (:1474-1493).
//
// The solve is PCG (float64 x, r, d, q and scalars) preconditioned by one
// V-cycle on a block hierarchy: levels with 4, 2 and 1 cells per brick edge
// (children 2 x 2 x 2 inside the brick), then levels of one cell per block
// whose block grid halves (a block exists if any child exists), until at most
// kAtCoarseMax cells remain, solved by a dense inverse.  Coarse phi is the mean
// of the children's phi (absent children inside the domain count as air,
// 0.5); coarse rows are rediscretised by the same rule.  Red-black
// Gauss-Seidel by global coordinate parity, one sweep before and one after
// (reversed), restriction R = P^T / 2 with P piecewise constant, so the
// preconditioner is symmetric.  Jacobi (precond = 0) is the reference's own
// preconditioner.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "alloc.h"
#include "../../include/fluid_pp.h"
#include "device_util.cuh"

namespace fpp {
namespace atlas {

constexpr int kRes = 8;            // finest cells per brick edge
constexpr int kCells = kRes * kRes * kRes;
constexpr int kFaces = (kRes + 1) * kRes * kRes;   // faces per axis per brick
constexpr int kAT = 256;           // threads per CTA
constexpr int kAGrid = 148 * 8;    // grid cap
constexpr int kAtMaxLevels = 16;
constexpr int kAtCoarseMax = 64;   // the dense coarsest level
constexpr long long kAtSmallCells = 2048;   // levels this small run in one CTA (k_at_vsmall)
constexpr int kRedGrid = 1184;     // fixed reduction grid (partials folded in block order)

struct ALevel {
  int B;                    // cells per block edge
  int dx, dy, dz;           // domain in this level's cells
  int gx, gy, gz;           // block grid
  int nblocks;
  long long n;              // nblocks * B^3
  const int* table;         // gx gy gz -> slot or -1
  const int* coords;        // nblocks x 3 block coordinates
  const int* children;      // levels made by halving a block grid: 8 finer slots per block (-1 absent)
  const int* parent;        // levels whose next coarser level halves the block grid: coarser slot per block
  uint8_t* label;
  float* phi;
  float* diag;
  float* z;
  float* rhs;
  float* res;
};

struct ACtrl {
  double bb, thr2, gamma, rr, rr_true;
  double div[4];     // max |b| and sum b^2 of the faces before and after the projection
  double red[4];     // last folded reductions
  double liquid;     // liquid cells
  int iter, max_iter, done, status, converged;
};

struct AInst {
  ALevel lv[kAtMaxLevels];
  int nlev;
  int precond;              // 1: V-cycle, 0: Jacobi
  int nb;                   // bricks
  const int* bnb;           // nb x 6 neighbour slots of each brick (kBrickAbsent, kBrickWall)
  float* faces;             // nb x 3 x kFaces, per brick u, v, w
  double* b;
  double* x;
  double* r;
  double* d;
  double* q;
  double* part;             // kRedGrid x 4
  double* bpart;            // one partial per brick (the brick-tiled reductions)
  double* coarse_inv;       // dense inverse of the coarsest level
  int coarse_m;
  int ncomp;                // liquid components without a cut row
  const int* comp_off;      // ncomp + 1
  const int* comp_cells;    // their level-0 cells
  double* comp_mean;
  ACtrl* ctrl;
};

// ----------------------------------------------------------------- geometry
struct Cell {
  int slot, lx, ly, lz;     // block slot and local coordinates
  int gx, gy, gz;           // level coordinates
};

__device__ __forceinline__ Cell cell_of(const ALevel& L, long long i) {
  const int B3 = L.B * L.B * L.B;
  Cell c;
  c.slot = int(i / B3);
  const int loc = int(i - (long long)c.slot * B3);
  c.lx = loc % L.B;
  c.ly = (loc / L.B) % L.B;
  c.lz = loc / (L.B * L.B);
  c.gx = L.coords[3 * c.slot] * L.B + c.lx;
  c.gy = L.coords[3 * c.slot + 1] * L.B + c.ly;
  c.gz = L.coords[3 * c.slot + 2] * L.B + c.lz;
  return c;
}

// Neighbour of cell c across its face on axis a, side s (+1 / -1):
// kWall outside the domain, kAbsent in an absent block inside it, else the
// neighbour's index.
constexpr long long kWall = -1, kAbsent = -2;

__device__ __forceinline__ long long neighbour(const ALevel& L, const Cell& c, int a, int s) {
  int g[3] = {c.gx, c.gy, c.gz};
  int l[3] = {c.lx, c.ly, c.lz};
  const int dom[3] = {L.dx, L.dy, L.dz};
  g[a] += s;
  if (g[a] < 0 || g[a] >= dom[a]) return kWall;
  l[a] += s;
  const int B = L.B;
  if (l[a] >= 0 && l[a] < B) return (long long)c.slot * B * B * B + l[0] + B * (l[1] + B * l[2]);
  const int bx = g[0] / B, by = g[1] / B, bz = g[2] / B;
  if (bx >= L.gx || by >= L.gy || bz >= L.gz) return kAbsent;
  const int t = L.table[bx + L.gx * (by + L.gy * bz)];
  if (t < 0) return kAbsent;
  l[a] = s > 0 ? 0 : B - 1;
  return (long long)t * B * B * B + l[0] + B * (l[1] + B * l[2]);
}

__device__ __forceinline__ double theta_d(double lphi, double aphi) {
  const double a = fabs(lphi);
  return fmin(1.0, fmax(0.05, a / fmax(a + fabs(aphi), 1e-12)));
}

// Row weight of cell i's face (a, s) for a liquid i: 0 on walls, 1 to a liquid
// neighbour, 1 / theta to an air cell or an absent block (phi 0.5).
__device__ __forceinline__ double face_weight(const ALevel& L, long long i, const Cell& c, int a, int s, long long& j) {
  j = neighbour(L, c, a, s);
  if (j == kWall) return 0.0;
  if (j == kAbsent) return 1.0 / theta_d(L.phi[i], 0.5);
  if (L.label[j]) return 1.0;
  return 1.0 / theta_d(L.phi[i], L.phi[j]);
}

// ------------------------------------------------------------------ kernels
// Cells of level L taken by thread t0 of ts (a grid-stride walk).
#define A_RANGE(L, t0, ts) for (long long i = (t0); i < (L).n; i += (ts))
#define A_CELLS(L)                                                                                   \
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (L).n;                  \
       i += (long long)gridDim.x * blockDim.x)

// Level 0 labels and phi from the bricks' density.
__global__ void k_at_label(AInst* I, const float* __restrict__ rho) {
  const ALevel& L = I->lv[0];
  A_CELLS(L) {
    const float ph = 0.5f - rho[i];
    L.phi[i] = ph;
    L.label[i] = ph <= 0.0f ? 1 : 0;
  }
}

// Coarse phi: mean of the children's phi; children in absent blocks inside the
// fine domain count as air (0.5), children outside it are left out.
__global__ void k_at_coarsen(AInst* I, int l) {
  const ALevel& F = I->lv[l];
  const ALevel& C = I->lv[l + 1];
  A_CELLS(C) {
    const Cell c = cell_of(C, i);
    double s = 0.0;
    int cnt = 0;
    for (int k = 0; k < 8; ++k) {
      const int ox = k & 1, oy = (k >> 1) & 1, oz = (k >> 2) & 1;
      const int fx = 2 * c.gx + ox, fy = 2 * c.gy + oy, fz = 2 * c.gz + oz;
      if (fx >= F.dx || fy >= F.dy || fz >= F.dz) continue;
      ++cnt;
      long long fi = -1;
      if (C.children) {   // one cell per block: the child block
        const int t = C.children[8 * (long long)c.slot + k];
        fi = t;           // B == 1 on the finer level too
      } else {            // children inside the same block
        const int B = F.B;
        fi = (long long)c.slot * B * B * B + (2 * c.lx + ox) + B * ((2 * c.ly + oy) + B * (2 * c.lz + oz));
      }
      s += fi >= 0 ? double(F.phi[fi]) : 0.5;
    }
    const float ph = float(s / double(max(cnt, 1)));
    C.phi[i] = ph;
    C.label[i] = ph <= 0.0f ? 1 : 0;
  }
}

// Diagonal of every level: the sum of the row weights (1 for air cells, which
// are identity rows of the smoother).
__global__ void k_at_diag(AInst* I, int l) {
  const ALevel& L = I->lv[l];
  A_CELLS(L) {
    if (!L.label[i]) {
      L.diag[i] = 1.0f;
      continue;
    }
    const Cell c = cell_of(L, i);
    double d = 0.0;
    long long j;
    for (int a = 0; a < 3; ++a) {
      d += face_weight(L, i, c, a, -1, j);
      d += face_weight(L, i, c, a, +1, j);
    }
    L.diag[i] = float(d);
  }
}

// Face f (0 .. 8) of a brick's axis-a array at the local tangential
// coordinates of cell c.
__device__ __forceinline__ long long face_index(int slot, int a, int lx, int ly, int lz) {
  long long off;
  if (a == 0) off = lx + (kRes + 1) * (ly + kRes * lz);
  else if (a == 1) off = lx + kRes * (ly + (kRes + 1) * lz);
  else off = lx + kRes * (ly + kRes * lz);
  return (long long)slot * 3 * kFaces + (long long)a * kFaces + off;
}

// (A v)_i for a liquid level-0 cell, float64.
__device__ __forceinline__ double apply0(const AInst* I, const double* v, long long i) {
  const ALevel& L = I->lv[0];
  const Cell c = cell_of(L, i);
  double s = double(L.diag[i]) * v[i];
  for (int a = 0; a < 3; ++a)
    for (int sd = -1; sd <= 1; sd += 2) {
      const long long j = neighbour(L, c, a, sd);
      if (j >= 0 && L.label[j]) s -= v[j];
    }
  return s;
}

// Fixed-grid float64 reductions: per-CTA tree sums into part[4 blockIdx + k],
// folded by one CTA in CTA order.
template <int K>
__device__ __forceinline__ void block_reduce(double (&v)[K], double* part) {
  __shared__ double sh[K][kAT];
#pragma unroll
  for (int k = 0; k < K; ++k) sh[k][threadIdx.x] = v[k];
  __syncthreads();
  for (int o = kAT / 2; o > 0; o >>= 1) {
    if (int(threadIdx.x) < o)
#pragma unroll
      for (int k = 0; k < K; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) part[4 * blockIdx.x + k] = sh[k][0];
}

__device__ __forceinline__ void at_fold(AInst* I, int K, int slot0) {
  __shared__ double sh[4][kAT];
  double v[4] = {0, 0, 0, 0};
  for (int b = threadIdx.x; b < kRedGrid; b += kAT)
    for (int k = 0; k < K; ++k) v[k] += I->part[4 * b + k];
  for (int k = 0; k < 4; ++k) sh[k][threadIdx.x] = v[k];
  __syncthreads();
  for (int o = kAT / 2; o > 0; o >>= 1) {
    if (int(threadIdx.x) < o)
      for (int k = 0; k < 4; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < K; ++k) I->ctrl->red[slot0 + k] = sh[k][0];
}

__global__ void __launch_bounds__(kAT) k_at_fold(AInst* I, int K, int slot0) { at_fold(I, K, slot0); }

// Nullspace: mean of each unanchored component (one CTA each, fixed order),
// then the subtraction.
__global__ void __launch_bounds__(kAT) k_at_comp_mean(AInst* I, const double* v) {
  __shared__ double sh[kAT];
  const int c = blockIdx.x;
  const int b0 = I->comp_off[c], b1 = I->comp_off[c + 1];
  double s = 0.0;
  for (int k = b0 + threadIdx.x; k < b1; k += kAT) s += v[I->comp_cells[k]];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = kAT / 2; o > 0; o >>= 1) {
    if (int(threadIdx.x) < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) I->comp_mean[c] = sh[0] / double(b1 - b0);
}

__global__ void k_at_comp_sub(AInst* I, double* v) {
  const int c = blockIdx.y;
  const int b0 = I->comp_off[c], b1 = I->comp_off[c + 1];
  const double m = I->comp_mean[c];
  for (int k = b0 + blockIdx.x * kAT + threadIdx.x; k < b1; k += gridDim.x * kAT) v[I->comp_cells[k]] -= m;
}

// ------------------------------------------------------------ the V-cycle
// One colour of red-black Gauss-Seidel on level l (from a zero guess when
// zero_init: the first colour then reads no neighbours).
__device__ __forceinline__ void at_smooth(AInst* I, int l, int colour, int zero_init, long long t0, long long ts) {
  const ALevel& L = I->lv[l];
  A_RANGE(L, t0, ts) {
    if (!L.label[i]) {
      if (zero_init) L.z[i] = 0.0f;
      continue;
    }
    const Cell c = cell_of(L, i);
    if (((c.gx + c.gy + c.gz) & 1) != colour) {
      if (zero_init && colour == 0) L.z[i] = 0.0f;
      continue;
    }
    float s = L.rhs[i];
    if (!(zero_init && colour == 0)) {
      for (int a = 0; a < 3; ++a)
        for (int sd = -1; sd <= 1; sd += 2) {
          const long long j = neighbour(L, c, a, sd);
          if (j >= 0 && L.label[j]) s += L.z[j];
        }
    }
    L.z[i] = s / L.diag[i];
  }
}

// res = rhs - A z on level l.
__device__ __forceinline__ void at_residual(AInst* I, int l, long long t0, long long ts) {
  const ALevel& L = I->lv[l];
  A_RANGE(L, t0, ts) {
    if (!L.label[i]) {
      L.res[i] = 0.0f;
      continue;
    }
    const Cell c = cell_of(L, i);
    float s = L.rhs[i] - L.diag[i] * L.z[i];
    for (int a = 0; a < 3; ++a)
      for (int sd = -1; sd <= 1; sd += 2) {
        const long long j = neighbour(L, c, a, sd);
        if (j >= 0 && L.label[j]) s += L.z[j];
      }
    L.res[i] = s;
  }
}

__device__ __forceinline__ long long grid_t0() { return blockIdx.x * (long long)blockDim.x + threadIdx.x; }
__device__ __forceinline__ long long grid_ts() { return (long long)gridDim.x * blockDim.x; }

__global__ void k_at_smooth(AInst* I, int l, int colour, int zero_init) {
  if (I->ctrl->done) return;
  at_smooth(I, l, colour, zero_init, grid_t0(), grid_ts());
}

__global__ void k_at_residual(AInst* I, int l) {
  if (I->ctrl->done) return;
  at_residual(I, l, grid_t0(), grid_ts());
}

// ----------------------------------------------- level 0, one CTA per brick
// The brick's values and its six face halos staged in shared memory as a
// 10^3 tile (index (z + 1) 100 + (y + 1) 10 + x + 1; edges and corners
// unused).  A halo cell in an absent brick or beyond a wall holds 0, which is
// what the stencils need: air and absent cells carry z = 0 and d = 0, and a
// liquid cell's diagonal already holds its walls' and air faces' weights.
constexpr int kTile = (kRes + 2) * (kRes + 2) * (kRes + 2);

__device__ __forceinline__ int tix(int x, int y, int z) { return (z + 1) * 100 + (y + 1) * 10 + (x + 1); }

// A brick's six neighbours, index 2 a + (side > 0): a slot, kBrickAbsent for
// an absent brick inside the domain, kBrickWall beyond a domain face.
constexpr int kBrickAbsent = -1, kBrickWall = -2;

// Threads 0 .. 5 fetch the brick's neighbours into nb (shared); the caller
// synchronises before reading them.
__device__ __forceinline__ void brick_nbrs(const AInst* I, int slot, int* nb) {
  if (threadIdx.x < 6) nb[threadIdx.x] = I->bnb[6 * slot + threadIdx.x];
}

// Two adjacent values of a brick row as one aligned load (cells 2q, 2q + 1).
template <class T> struct Pair;
template <> struct Pair<float> { using V = float2; };
template <> struct Pair<double> { using V = double2; };
template <> struct Pair<uint8_t> { using V = uchar2; };

// Stage the brick's values and its halos (nb: the brick's neighbours, already
// visible to every thread); ends with a barrier.  The body is read as row
// pairs; halo entry e (face f = e / 64, face cell u = e % 8, w = e / 8 % 8)
// is the neighbour's cell on the shared face (f = 2 a + (side > 0)).
template <class T>
__device__ __forceinline__ void load_tile(int slot, const int* nb, const T* v, T* t) {
  using V = typename Pair<T>::V;
  const V* src = reinterpret_cast<const V*>(v + (long long)slot * kCells);
  for (int q = threadIdx.x; q < kCells / 2; q += blockDim.x) {
    const V p = src[q];
    const int k = 2 * q, c = tix(k & 7, (k >> 3) & 7, k >> 6);
    t[c] = p.x;
    t[c + 1] = p.y;
  }
  for (int e = threadIdx.x; e < 6 * 64; e += blockDim.x) {
    const int f = e >> 6, u = e & 7, w = (e >> 3) & 7;
    int c, o;   // tile index, cell of the neighbour brick
    switch (f) {
      case 0: c = (w + 1) * 100 + (u + 1) * 10; o = (kRes - 1) + kRes * (u + kRes * w); break;
      case 1: c = (w + 1) * 100 + (u + 1) * 10 + kRes + 1; o = kRes * (u + kRes * w); break;
      case 2: c = (w + 1) * 100 + (u + 1); o = u + kRes * ((kRes - 1) + kRes * w); break;
      case 3: c = (w + 1) * 100 + (kRes + 1) * 10 + (u + 1); o = u + kRes * kRes * w; break;
      case 4: c = (w + 1) * 10 + (u + 1); o = u + kRes * (w + kRes * (kRes - 1)); break;
      default: c = (kRes + 1) * 100 + (w + 1) * 10 + (u + 1); o = u + kRes * w; break;
    }
    const int ns = nb[f];
    t[c] = ns >= 0 ? v[(long long)ns * kCells + o] : T(0);
  }
  __syncthreads();
}

template <class T>
__device__ __forceinline__ T nbr_sum(const T* t, int x, int y, int z) {
  const int c = tix(x, y, z);
  return ((t[c - 1] + t[c + 1]) + (t[c - 10] + t[c + 10])) + (t[c - 100] + t[c + 100]);
}

// One colour of the level-0 smoother (z in place; the other colour's values,
// inside and across the brick, are not written by this launch): thread t
// takes the t-th cell of the colour, (x + y + z) & 1 == colour.
__global__ void __launch_bounds__(256) k_at_smooth0(AInst* I, int colour) {
  if (I->ctrl->done) return;
  const ALevel& L = I->lv[0];
  __shared__ float t[kTile];
  __shared__ int nb[6];
  const int slot = blockIdx.x;
  brick_nbrs(I, slot, nb);
  const int ty = (threadIdx.x >> 2) & 7, tz = threadIdx.x >> 5;
  const int tx = 2 * (threadIdx.x & 3) + ((ty + tz + colour) & 1);
  const long long i = (long long)slot * kCells + tx + kRes * (ty + kRes * tz);
  const bool liq = L.label[i];   // the cell's own inputs load while the tile comes in
  const float r = L.rhs[i], d = L.diag[i];
  __syncthreads();
  load_tile<float>(slot, nb, L.z, t);
  if (!liq) return;
  L.z[i] = (r + nbr_sum(t, tx, ty, tz)) / d;
}

// The first colour of the level-0 pre-smoothing from zero: red liquid cells
// z = rhs / diag, every other cell 0 (no neighbour terms).
__global__ void __launch_bounds__(256) k_at_smooth0_zero(AInst* I) {
  if (I->ctrl->done) return;
  const ALevel& L = I->lv[0];
  const int slot = blockIdx.x;
  for (int k = threadIdx.x; k < kCells; k += 256) {
    const int x = k & 7, y = (k >> 3) & 7, z = k >> 6;
    const long long i = (long long)slot * kCells + k;
    L.z[i] = (L.label[i] && ((x + y + z) & 1) == 0) ? L.rhs[i] / L.diag[i] : 0.0f;
  }
}

// res = rhs - A z on level 0 (two cells per thread, kept in shared memory)
// and its restriction into the brick's own block of level 1 (4^3 cells):
// rhs_c = 1/2 sum of the 8 children's residuals in child order, 0 on air,
// as k_at_restrict forms it.
__global__ void __launch_bounds__(256) k_at_residual0(AInst* I) {
  if (I->ctrl->done) return;
  const ALevel& L = I->lv[0];
  const ALevel& C = I->lv[1];
  constexpr int CB = kRes / 2, CC = CB * CB * CB;
  __shared__ float t[kTile];
  __shared__ float rs[kCells];
  __shared__ int nb[6];
  const int slot = blockIdx.x;
  brick_nbrs(I, slot, nb);
  bool liq[2];   // the cells' own inputs load while the tile comes in
  float r[2], d[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const long long i = (long long)slot * kCells + threadIdx.x + 256 * h;
    liq[h] = L.label[i];
    r[h] = L.rhs[i];
    d[h] = L.diag[i];
  }
  const bool cl = threadIdx.x < CC && C.label[(long long)slot * CC + threadIdx.x];
  __syncthreads();
  load_tile<float>(slot, nb, L.z, t);
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int k = threadIdx.x + 256 * h;
    const int x = k & 7, y = (k >> 3) & 7, z = k >> 6;
    rs[k] = liq[h] ? (r[h] - d[h] * t[tix(x, y, z)]) + nbr_sum(t, x, y, z) : 0.0f;
  }
  __syncthreads();
  if (threadIdx.x < CC) {
    const int cx = threadIdx.x % CB, cy = (threadIdx.x / CB) % CB, cz = threadIdx.x / (CB * CB);
    float sum = 0.0f;
    if (cl)
      for (int k = 0; k < 8; ++k)
        sum += rs[(2 * cx + (k & 1)) + kRes * ((2 * cy + ((k >> 1) & 1)) + kRes * (2 * cz + ((k >> 2) & 1)))];
    C.rhs[(long long)slot * CC + threadIdx.x] = cl ? 0.5f * sum : 0.0f;
  }
}

// q = A d and the CTA's d . q partial (level 0, float64).  One CTA per
// brick; the partials go to part[4 brick] (the fold reads kRedGrid of them
// per pass, so the brick kernels write a per-brick array folded separately).
__global__ void __launch_bounds__(256) k_at_spmv0(AInst* I, double* bpart) {
  if (I->ctrl->done) return;
  const ALevel& L = I->lv[0];
  __shared__ double t[kTile];
  __shared__ int nb[6];
  const int slot = blockIdx.x;
  brick_nbrs(I, slot, nb);
  bool liq[2];   // the cells' own inputs load while the tile comes in
  float dg[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const long long i = (long long)slot * kCells + threadIdx.x + 256 * h;
    liq[h] = L.label[i];
    dg[h] = L.diag[i];
  }
  __syncthreads();
  load_tile<double>(slot, nb, I->d, t);
  double acc = 0.0;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int k = threadIdx.x + 256 * h;
    const int x = k & 7, y = (k >> 3) & 7, z = k >> 6;
    const long long i = (long long)slot * kCells + k;
    double q = 0.0;
    if (liq[h]) {
      const double dv = t[tix(x, y, z)];
      q = double(dg[h]) * dv - nbr_sum(t, x, y, z);
      acc += dv * q;
    }
    I->q[i] = q;
  }
  __shared__ double sh[256];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (int(threadIdx.x) < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) bpart[slot] = sh[0];
}

// Folds the per-brick partials into ctrl->red[0]: 256 threads each sum a
// fixed stride of bricks, then a fixed tree.
// keep_gamma: first move the folded gamma (red[0]) to ctrl->gamma, which
// red[0] is about to be overwritten by delta (the CG's set-gamma step).
__global__ void __launch_bounds__(256) k_at_fold_bricks(AInst* I, const double* bpart, int keep_gamma) {
  __shared__ double sh[256];
  double s = 0.0;
  for (int b = threadIdx.x; b < I->nb; b += 256) s += bpart[b];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (int(threadIdx.x) < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (keep_gamma && !I->ctrl->done) I->ctrl->gamma = I->ctrl->red[0];
    I->ctrl->red[0] = sh[0];
  }
}

// Finer level index of child k (0 .. 7) of coarse cell c, -1 if none.
__device__ __forceinline__ long long child_of(const ALevel& F, const ALevel& C, const Cell& c, int k) {
  const int ox = k & 1, oy = (k >> 1) & 1, oz = (k >> 2) & 1;
  if (2 * c.gx + ox >= F.dx || 2 * c.gy + oy >= F.dy || 2 * c.gz + oz >= F.dz) return -1;
  if (C.children) return C.children[8 * (long long)c.slot + k];
  const int B = F.B;
  return (long long)c.slot * B * B * B + (2 * c.lx + ox) + B * ((2 * c.ly + oy) + B * (2 * c.lz + oz));
}

// rhs_c = 1/2 sum of the liquid children's residuals (R = P^T / 2).
__device__ __forceinline__ void at_restrict(AInst* I, int l, long long t0, long long ts) {
  const ALevel& F = I->lv[l];
  const ALevel& C = I->lv[l + 1];
  A_RANGE(C, t0, ts) {
    if (!C.label[i]) {
      C.rhs[i] = 0.0f;
      continue;
    }
    const Cell c = cell_of(C, i);
    float s = 0.0f;
    for (int k = 0; k < 8; ++k) {
      const long long f = child_of(F, C, c, k);
      if (f >= 0) s += F.res[f];   // res is 0 on air children
    }
    C.rhs[i] = 0.5f * s;
  }
}

// z_f += z_c on liquid fine cells (P piecewise constant).
__device__ __forceinline__ void at_prolong(AInst* I, int l, long long t0, long long ts) {
  const ALevel& F = I->lv[l];
  const ALevel& C = I->lv[l + 1];
  A_RANGE(F, t0, ts) {
    if (!F.label[i]) continue;
    long long ci;
    if (F.parent) {
      const Cell f = cell_of(F, i);   // B == 1: the block is the cell
      ci = F.parent[f.slot];
    } else {
      const Cell f = cell_of(F, i);
      const int B = C.B;
      ci = (long long)f.slot * B * B * B + (f.lx / 2) + B * ((f.ly / 2) + B * (f.lz / 2));
    }
    if (ci >= 0 && C.label[ci]) F.z[i] += C.z[ci];
  }
}

__global__ void k_at_restrict(AInst* I, int l) {
  if (I->ctrl->done) return;
  at_restrict(I, l, grid_t0(), grid_ts());
}

__global__ void k_at_prolong(AInst* I, int l) {
  if (I->ctrl->done) return;
  at_prolong(I, l, grid_t0(), grid_ts());
}

// Dense inverse of the coarsest level's operator (one CTA, shared memory):
// air cells are identity rows; a level with no cut row gets the rank-one
// term mean(diag) / m 1 1^T so the inverse is SPD.
__global__ void __launch_bounds__(1024) k_at_coarse_factor(AInst* I) {
  const ALevel& L = I->lv[I->nlev - 1];
  const int m = int(L.n);
  __shared__ double A[kAtCoarseMax * kAtCoarseMax];
  __shared__ double prow[kAtCoarseMax], pcol[kAtCoarseMax];
  __shared__ int anchored;
  if (threadIdx.x == 0) anchored = 0;
  for (int e = threadIdx.x; e < m * m; e += blockDim.x) A[e] = 0.0;
  __syncthreads();
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    if (!L.label[i]) {
      A[i * m + i] = 1.0;
      atomicOr(&anchored, 1);
      continue;
    }
    const Cell c = cell_of(L, i);
    A[i * m + i] = L.diag[i];
    for (int a = 0; a < 3; ++a)
      for (int sd = -1; sd <= 1; sd += 2) {
        const long long j = neighbour(L, c, a, sd);
        if (j == kAbsent) atomicOr(&anchored, 1);
        if (j >= 0 && L.label[j]) A[i * m + j] = -1.0;
      }
  }
  __syncthreads();
  if (!anchored) {
    __shared__ double add;
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int i = 0; i < m; ++i) s += A[i * m + i];
      add = s / double(m) / double(m);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) A[e] += add;
    __syncthreads();
  }
  gauss_jordan_inplace(A, m, prow, pcol);
  for (int e = threadIdx.x; e < m * m; e += blockDim.x) I->coarse_inv[e] = A[e];
}

// z = A^{-1} rhs on the coarsest level, a warp per row.
__device__ __forceinline__ void at_coarse_apply(AInst* I) {
  const ALevel& L = I->lv[I->nlev - 1];
  const int m = int(L.n);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int i = warp; i < m; i += nw) {
    double s = 0.0;
    for (int j = lane; j < m; j += 32) s += I->coarse_inv[i * m + j] * (L.label[j] ? double(L.rhs[j]) : 0.0);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) L.z[i] = L.label[i] ? float(s) : 0.0f;
  }
}

__global__ void k_at_coarse_apply(AInst* I) {
  if (I->ctrl->done) return;
  at_coarse_apply(I);
}

// The small levels first .. nlev - 1 of the V-cycle in one CTA: the same
// stages in the same order as the per-level launches (pre-smoothing from
// zero, residual, restriction down to the dense coarsest level, then
// prolongation and post-smoothing up to level first), separated by barriers
// instead of launches.  Each stage computes every cell from values the
// previous stages wrote, as the launches do, so the results are the same.
__global__ void __launch_bounds__(1024) k_at_vsmall(AInst* I, int first, int pre, int post) {
  if (I->ctrl->done) return;
  const long long t0 = threadIdx.x, ts = blockDim.x;
  const int last = I->nlev - 1;
  for (int l = first; l < last; ++l) {
    at_smooth(I, l, 0, 1, t0, ts);
    __syncthreads();
    at_smooth(I, l, 1, 0, t0, ts);
    __syncthreads();
    for (int k = 1; k < pre; ++k) {
      at_smooth(I, l, 0, 0, t0, ts);
      __syncthreads();
      at_smooth(I, l, 1, 0, t0, ts);
      __syncthreads();
    }
    at_residual(I, l, t0, ts);
    __syncthreads();
    at_restrict(I, l, t0, ts);
    __syncthreads();
  }
  at_coarse_apply(I);
  __syncthreads();
  for (int l = last - 1; l >= first; --l) {
    at_prolong(I, l, t0, ts);
    __syncthreads();
    for (int k = 0; k < post; ++k) {
      at_smooth(I, l, 1, 0, t0, ts);
      __syncthreads();
      at_smooth(I, l, 0, 0, t0, ts);
      __syncthreads();
    }
  }
}

// Level-0 rhs of the V-cycle from the CG residual (float).
__global__ void k_at_vin(AInst* I) {
  if (I->ctrl->done) return;
  const ALevel& L = I->lv[0];
  A_CELLS(L) L.rhs[i] = L.label[i] ? float(I->r[i]) : 0.0f;
}

// ------------------------------------------------------------ CG kernels
// z as a float64 vector (for the nullspace projection of z before the dot):
// the preconditioned residual is written to q temporarily.
__global__ void k_at_zvec(AInst* I) {
  if (I->ctrl->done) return;
  const ALevel& L = I->lv[0];
  A_CELLS(L) {
    I->q[i] = L.label[i] ? (I->precond ? double(L.z[i]) : I->r[i] / double(L.diag[i])) : 0.0;
  }
}

__global__ void __launch_bounds__(kAT) k_at_dot_rq(AInst* I) {
  if (I->ctrl->done) return;
  const ALevel& L = I->lv[0];
  double v[1] = {0.0};
  A_CELLS(L) if (L.label[i]) v[0] += I->r[i] * I->q[i];
  block_reduce<1>(v, I->part);
}

// zvec and dot_rq in one pass (no nullspace projection between them).
__global__ void __launch_bounds__(kAT) k_at_zdot(AInst* I) {
  if (I->ctrl->done) return;
  const ALevel& L = I->lv[0];
  double v[1] = {0.0};
  A_CELLS(L) {
    const double z = L.label[i] ? (I->precond ? double(L.z[i]) : I->r[i] / double(L.diag[i])) : 0.0;
    I->q[i] = z;
    if (L.label[i]) v[0] += I->r[i] * z;
  }
  block_reduce<1>(v, I->part);
}

__global__ void __launch_bounds__(kAT) k_at_rr(AInst* I) {
  if (I->ctrl->done) return;
  const ALevel& L = I->lv[0];
  double v[1] = {0.0};
  A_CELLS(L) if (L.label[i]) v[0] += I->r[i] * I->r[i];
  block_reduce<1>(v, I->part);
}

// beta and d = z + beta d (first iteration: d = z); z is in q.
__global__ void k_at_dir(AInst* I) {
  ACtrl* C = I->ctrl;
  if (C->done) return;
  const double gnew = C->red[0];
  const double beta = C->iter == 0 ? 0.0 : gnew / C->gamma;
  const ALevel& L = I->lv[0];
  A_CELLS(L) I->d[i] = L.label[i] ? I->q[i] + beta * I->d[i] : 0.0;
}



// q = A d, delta = d . q
__global__ void __launch_bounds__(kAT) k_at_spmv(AInst* I) {
  if (I->ctrl->done) return;
  const ALevel& L = I->lv[0];
  double v[1] = {0.0};
  A_CELLS(L) {
    double q = 0.0;
    if (L.label[i]) {
      q = apply0(I, I->d, i);
      v[0] += I->d[i] * q;
    }
    I->q[i] = q;
  }
  block_reduce<1>(v, I->part);
}

// x += alpha d, r -= alpha q, rr = r . r; with VIN also the next V-cycle's level-0 input
template <bool VIN>
__global__ void __launch_bounds__(kAT) k_at_update(AInst* I) {
  ACtrl* C = I->ctrl;
  if (C->done) return;
  const double alpha = C->gamma / C->red[0];
  const ALevel& L = I->lv[0];
  double v[1] = {0.0};
  A_CELLS(L) {
    if (!L.label[i]) continue;
    I->x[i] += alpha * I->d[i];
    const double r = I->r[i] - alpha * I->q[i];
    I->r[i] = r;
    if (VIN) L.rhs[i] = float(r);   // the next V-cycle's input (air cells keep rhs 0)
    v[0] += r * r;
  }
  block_reduce<1>(v, I->part);
}

// r = b - A x (float64), rr = r . r
__global__ void __launch_bounds__(kAT) k_at_true(AInst* I) {
  if (I->ctrl->done) return;
  const ALevel& L = I->lv[0];
  double v[1] = {0.0};
  A_CELLS(L) {
    if (!L.label[i]) continue;
    const double r = I->b[i] - apply0(I, I->x, i);
    I->r[i] = r;
    v[0] += r * r;
  }
  block_reduce<1>(v, I->part);
}

// After an update: count the iteration, stop on the tolerance (the
// recursive float64 residual, as projectSparseAtlasVelocity does), the cap,
// or a non-finite residual.
// The stopping test on the folded rr (red[0]).
__device__ __forceinline__ void at_check(AInst* I) {
  ACtrl* C = I->ctrl;
  if (C->done) return;
  const double rr = C->red[0];
  C->iter += 1;
  C->rr = rr;
  if (!(rr == rr) || fabs(rr) > 1e300) {
    C->done = 1;
    C->status = FLUID_PP_NONFINITE;
    return;
  }
  if (rr <= C->thr2) {
    C->done = 1;
    C->converged = 1;
    C->status = FLUID_PP_OK;
    return;
  }
  if (C->iter >= C->max_iter) {
    C->done = 1;
    C->status = FLUID_PP_NONCONVERGENCE;
  }
}

// The fold of rr (red[0]) and the stopping test in one launch.
__global__ void __launch_bounds__(kAT) k_at_fold_check(AInst* I) {
  at_fold(I, 1, 0);
  if (threadIdx.x == 0) at_check(I);   // the thread that wrote red[0]
}

__global__ void k_at_init(AInst* I, double thr_rel, double thr_abs, int max_iter) {
  ACtrl* C = I->ctrl;
  const double bb = C->red[0];
  C->bb = bb;
  C->liquid = C->red[1];
  const double t = fmax(thr_abs, thr_rel * sqrt(bb));
  C->thr2 = t * t;
  C->iter = 0;
  C->max_iter = max_iter;
  C->done = bb <= C->thr2 ? 1 : 0;
  C->converged = C->done;
  C->status = FLUID_PP_OK;
  C->rr = bb;
  C->rr_true = bb;
}

__global__ void __launch_bounds__(kAT) k_at_bb(AInst* I) {
  const ALevel& L = I->lv[0];
  double v[2] = {0.0, 0.0};
  A_CELLS(L) {
    if (!L.label[i]) continue;
    v[0] += I->b[i] * I->b[i];
    v[1] += 1.0;
  }
  block_reduce<2>(v, I->part);
}

__global__ void k_at_start(AInst* I) {
  const ALevel& L = I->lv[0];
  A_CELLS(L) {
    I->x[i] = 0.0;
    I->r[i] = L.label[i] ? I->b[i] : 0.0;
    I->d[i] = 0.0;
    L.rhs[i] = L.label[i] ? float(I->b[i]) : 0.0f;   // the first V-cycle's input
  }
}

// ------------------------------- levels 1 and 2, K blocks of B^3 per CTA
// Levels with B = 4 and 2 cells per brick edge hold the bricks' own blocks
// (same slots, same block grid), so the brick neighbour table serves them.
// Each block and its face halos are staged in a (B + 2)^3 tile; the stencil
// adds the six neighbours in the order of the per-cell kernels (x-, x+, y-,
// y+, z-, z+).  Air cells of these levels hold z = 0 from the first colour of
// the pre-smoothing on (it writes every cell, the prolongation adds only to
// liquid ones), and absent or beyond-wall halo cells are staged as 0, so the
// tile needs no labels.
template <int B>
struct BTile {
  static constexpr int C = B * B * B, W = B + 2, N = W * W * W;
  static __device__ __forceinline__ int ix(int x, int y, int z) { return (z + 1) * W * W + (y + 1) * W + (x + 1); }
};

template <int B, int K>
__device__ __forceinline__ void load_btiles(const ALevel& L, const int (*nb)[6], const float* v, float (*t)[BTile<B>::N]) {
  using T = BTile<B>;
  for (int e = threadIdx.x; e < K * T::C; e += blockDim.x) {
    const int j = e / T::C, k = e - j * T::C;
    const int slot = blockIdx.x * K + j;
    t[j][T::ix(k % B, (k / B) % B, k / (B * B))] = slot < L.nblocks ? v[(long long)slot * T::C + k] : 0.0f;
  }
  for (int e = threadIdx.x; e < K * 6 * B * B; e += blockDim.x) {
    const int j = e / (6 * B * B), r = e - j * 6 * B * B;
    const int f = r / (B * B), u = r % B, w = (r / B) % B;
    const int a = f >> 1, sd = (f & 1) ? 1 : -1;
    int h[3], m[3];
    if (a == 0) { h[0] = sd > 0 ? B : -1; h[1] = u; h[2] = w; }
    else if (a == 1) { h[0] = u; h[1] = sd > 0 ? B : -1; h[2] = w; }
    else { h[0] = u; h[1] = w; h[2] = sd > 0 ? B : -1; }
    m[0] = h[0]; m[1] = h[1]; m[2] = h[2];
    m[a] = sd > 0 ? 0 : B - 1;
    const int ns = nb[j][f];
    t[j][T::ix(h[0], h[1], h[2])] = ns >= 0 ? v[(long long)ns * T::C + m[0] + B * (m[1] + B * m[2])] : 0.0f;
  }
}

// The CTA's K blocks' neighbours (beyond the level's blocks: walls).
template <int K>
__device__ __forceinline__ void block_nbrs(const AInst* I, const ALevel& L, int (*nb)[6]) {
  if (threadIdx.x < 6 * K) {
    const int j = threadIdx.x / 6, f = threadIdx.x - 6 * j, slot = blockIdx.x * K + j;
    nb[j][f] = slot < L.nblocks ? I->bnb[6 * slot + f] : kBrickWall;
  }
}

// One colour of the smoother on level l (B cells per block edge, B even, so a
// cell's colour is its local parity); thread t: block t / B^3, cell t % B^3.
template <int B, int K>
__global__ void __launch_bounds__(K * B * B * B) k_at_smooth_t(AInst* I, int l, int colour, int zero_init) {
  using T = BTile<B>;
  if (I->ctrl->done) return;
  const ALevel& L = I->lv[l];
  __shared__ float t[K][T::N];
  __shared__ int nb[K][6];
  block_nbrs<K>(I, L, nb);
  const int j = threadIdx.x / T::C, k = threadIdx.x - j * T::C;
  const int slot = blockIdx.x * K + j;
  const bool act = slot < L.nblocks;
  const int x = k % B, y = (k / B) % B, z = k / (B * B);
  const long long i = (long long)slot * T::C + k;
  bool liq = false;   // the cell's own inputs load while the tile comes in
  float r = 0.0f, d = 1.0f;
  if (act) {
    liq = L.label[i];
    r = L.rhs[i];
    d = L.diag[i];
  }
  const bool first = zero_init && colour == 0;   // from zero: no neighbour terms
  __syncthreads();
  if (!first) {
    load_btiles<B, K>(L, nb, L.z, t);
    __syncthreads();
  }
  if (!act) return;
  if (!liq) {
    if (zero_init) L.z[i] = 0.0f;
    return;
  }
  if (((x + y + z) & 1) != colour) {
    if (first) L.z[i] = 0.0f;
    return;
  }
  float s = r;
  if (!first) {
    const float* tt = t[j];
    const int c = T::ix(x, y, z);
    s += tt[c - 1];
    s += tt[c + 1];
    s += tt[c - T::W];
    s += tt[c + T::W];
    s += tt[c - T::W * T::W];
    s += tt[c + T::W * T::W];
  }
  L.z[i] = s / d;
}

// res = rhs - A z on level l (B as k_at_smooth_t), kept in shared memory, and
// its restriction into level l + 1, whose blocks are the same bricks' with
// B / 2 cells per edge: rhs_c = 1/2 sum of the 8 children's residuals in
// child order, 0 on air, as k_at_restrict forms it.
template <int B, int K>
__global__ void __launch_bounds__(K * B * B * B) k_at_residual_t(AInst* I, int l) {
  using T = BTile<B>;
  constexpr int CB = B / 2, CC = CB * CB * CB;
  static_assert(K * CC <= K * T::C, "a thread per coarse cell");
  if (I->ctrl->done) return;
  const ALevel& L = I->lv[l];
  const ALevel& Cl = I->lv[l + 1];
  __shared__ float t[K][T::N];
  __shared__ float rs[K][T::C];
  __shared__ int nb[K][6];
  block_nbrs<K>(I, L, nb);
  const int j = threadIdx.x / T::C, k = threadIdx.x - j * T::C;
  const int slot = blockIdx.x * K + j;
  const bool act = slot < L.nblocks;
  const int x = k % B, y = (k / B) % B, z = k / (B * B);
  const long long i = (long long)slot * T::C + k;
  bool liq = false;
  float r = 0.0f, d = 0.0f;
  if (act) {
    liq = L.label[i];
    r = L.rhs[i];
    d = L.diag[i];
  }
  // the coarse cell of thread e < K CC: block e / CC, cell e % CC
  const int cj = threadIdx.x / CC, ck = threadIdx.x - cj * CC, cslot = blockIdx.x * K + cj;
  const bool cown = threadIdx.x < K * CC && cslot < L.nblocks;
  const bool cl = cown && Cl.label[(long long)cslot * CC + ck];
  __syncthreads();
  load_btiles<B, K>(L, nb, L.z, t);
  __syncthreads();
  float res = 0.0f;
  if (act && liq) {
    const float* tt = t[j];
    const int c = T::ix(x, y, z);
    float s = r - d * tt[c];
    s += tt[c - 1];
    s += tt[c + 1];
    s += tt[c - T::W];
    s += tt[c + T::W];
    s += tt[c - T::W * T::W];
    s += tt[c + T::W * T::W];
    res = s;
  }
  rs[j][k] = res;
  __syncthreads();
  if (cown) {
    const int cx = ck % CB, cy = (ck / CB) % CB, cz = ck / (CB * CB);
    float sum = 0.0f;
    if (cl)
      for (int q = 0; q < 8; ++q)
        sum += rs[cj][(2 * cx + (q & 1)) + B * ((2 * cy + ((q >> 1) & 1)) + B * (2 * cz + ((q >> 2) & 1)))];
    Cl.rhs[(long long)cslot * CC + ck] = cl ? 0.5f * sum : 0.0f;
  }
}

// ------------------------------------------ the faces, one CTA per brick
// A brick's six neighbour slots (-1 absent or beyond a wall) and which of its
// faces lie on the domain walls, index 2 a + (side > 0).
__device__ __forceinline__ void brick_sides(const AInst* I, int slot, int* nbs, int* nbw) {
  if (threadIdx.x < 6) {
    const int b = I->bnb[6 * slot + threadIdx.x];
    nbw[threadIdx.x] = b == kBrickWall;
    nbs[threadIdx.x] = b >= 0 ? b : -1;
  }
}

// Face entry k (0 .. 575) of a brick's axis-A array as local (x, y, z), the
// axis coordinate being the face index 0 .. 8; face_off is the inverse.
template <int A>
__device__ __forceinline__ void face_local(int k, int* l) {
  if (A == 0) { l[0] = k % (kRes + 1); l[1] = (k / (kRes + 1)) % kRes; l[2] = k / ((kRes + 1) * kRes); }
  else if (A == 1) { l[0] = k % kRes; l[1] = (k / kRes) % (kRes + 1); l[2] = k / (kRes * (kRes + 1)); }
  else { l[0] = k % kRes; l[1] = (k / kRes) % kRes; l[2] = k / (kRes * kRes); }
}

template <int A>
__device__ __forceinline__ int face_off(int x, int y, int z) {
  if (A == 0) return x + (kRes + 1) * (y + kRes * z);
  if (A == 1) return x + kRes * (y + (kRes + 1) * z);
  return x + kRes * (y + kRes * z);
}

// Stage a brick's axis-A faces in shared memory, the canonical copy of each
// port (a low face shared with a present lower brick is that brick's f = 8
// copy); with sync the brick's own f = 0 copy of such a port is set to it.
template <int A>
__device__ __forceinline__ void stage_faces(const AInst* I, int slot, const int* nbs, int sync, float* fs) {
  for (int k = threadIdx.x; k < kFaces; k += blockDim.x) {
    int l[3];
    face_local<A>(k, l);
    const long long own = (long long)slot * 3 * kFaces + (long long)A * kFaces + k;
    if (l[A] == 0 && nbs[2 * A] >= 0) {
      l[A] = kRes;
      const float v = I->faces[(long long)nbs[2 * A] * 3 * kFaces + (long long)A * kFaces + face_off<A>(l[0], l[1], l[2])];
      fs[k] = v;
      if (sync) I->faces[own] = v;
    } else {
      fs[k] = I->faces[own];
    }
  }
}

// The axis-A part of b for local cell l: its low face minus its high face,
// each only where it is a row (not a domain wall).
template <int A>
__device__ __forceinline__ double div_axis(const float* fs, const int* nbw, const int* l) {
  int h[3] = {l[0], l[1], l[2]};
  h[A] += 1;
  double b = 0.0;
  if (!(l[A] == 0 && nbw[2 * A])) b += double(fs[face_off<A>(l[0], l[1], l[2])]);
  if (!(l[A] == kRes - 1 && nbw[2 * A + 1])) b -= double(fs[face_off<A>(h[0], h[1], h[2])]);
  return b;
}

// b = G^T u of every cell of the brick (0 off the liquid), written to I->b
// when write_b, and the brick's max |b| and sum b^2 over liquid cells into
// bpart[2 brick ..].  With write_b the brick's own f = 0 copy of each port is
// also set to the canonical value, so that the projection can read its own
// copies.  No CTA writes a face another CTA reads here: f = 8 copies are only
// read.
__global__ void __launch_bounds__(256) k_at_div0(AInst* I, int write_b, double* bpart) {
  const ALevel& L = I->lv[0];
  const int slot = blockIdx.x;
  __shared__ float fs[3][kFaces];
  __shared__ int nbs[6], nbw[6];
  brick_sides(I, slot, nbs, nbw);
  __syncthreads();
  stage_faces<0>(I, slot, nbs, write_b, fs[0]);
  stage_faces<1>(I, slot, nbs, write_b, fs[1]);
  stage_faces<2>(I, slot, nbs, write_b, fs[2]);
  __syncthreads();
  double mx = 0.0, ss = 0.0;
  for (int k = threadIdx.x; k < kCells; k += 256) {
    const int l[3] = {k & 7, (k >> 3) & 7, k >> 6};
    const long long i = (long long)slot * kCells + k;
    double b = 0.0;
    if (L.label[i]) {
      b += div_axis<0>(fs[0], nbw, l);
      b += div_axis<1>(fs[1], nbw, l);
      b += div_axis<2>(fs[2], nbw, l);
      mx = fmax(mx, fabs(b));
      ss += b * b;
    }
    if (write_b) I->b[i] = b;
  }
  __shared__ double sm[256], sq[256];
  sm[threadIdx.x] = mx;
  sq[threadIdx.x] = ss;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (int(threadIdx.x) < o) {
      sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + o]);
      sq[threadIdx.x] += sq[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    bpart[2 * slot] = sm[0];
    bpart[2 * slot + 1] = sq[0];
  }
}

// The divergence receipt from the per-brick partials (fixed stride and tree).
__global__ void __launch_bounds__(256) k_at_div_fold_bricks(AInst* I, const double* bpart, int slot0) {
  __shared__ double sm[256], sq[256];
  double m = 0.0, q = 0.0;
  for (int b = threadIdx.x; b < I->nb; b += 256) {
    m = fmax(m, bpart[2 * b]);
    q += bpart[2 * b + 1];
  }
  sm[threadIdx.x] = m;
  sq[threadIdx.x] = q;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (int(threadIdx.x) < o) {
      sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + o]);
      sq[threadIdx.x] += sq[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    I->ctrl->div[slot0] = sm[0];
    I->ctrl->div[slot0 + 1] = sq[0];
  }
}

// The projection of a brick's own faces: u - jump / theta on rows with a
// liquid side, 0 on rows without, walls kept.  A port (a face shared with a
// present neighbour brick) is computed by both bricks from the same values:
// the pressures and levels of its two cells, and the face value, whose two
// copies k_at_div0 made equal.  Each CTA reads and writes only its own faces.
template <int A>
__device__ __forceinline__ void project_axis(AInst* I, int slot, const int* nbs, const int* nbw, const double* xs,
                                             const float* ph, const uint8_t* lb) {
  for (int k = threadIdx.x; k < kFaces; k += blockDim.x) {
    int l[3];
    face_local<A>(k, l);
    const int f = l[A];
    if ((f == 0 && nbw[2 * A]) || (f == kRes && nbw[2 * A + 1])) continue;   // a domain wall keeps its value
    const bool lo_absent = f == 0 && nbs[2 * A] < 0, hi_absent = f == kRes && nbs[2 * A + 1] < 0;
    int lo[3] = {l[0], l[1], l[2]};
    lo[A] = f - 1;
    const int tlo = tix(lo[0], lo[1], lo[2]), thi = tix(l[0], l[1], l[2]);
    const bool li = !lo_absent && lb[tlo] != 0, lj = !hi_absent && lb[thi] != 0;
    const long long own = (long long)slot * 3 * kFaces + (long long)A * kFaces + k;
    float val = 0.0f;
    if (li || lj) {
      const float u0 = I->faces[own];
      const double jump = (lj ? xs[thi] : 0.0) - (li ? xs[tlo] : 0.0);
      double th = 1.0;
      if (li != lj) {
        const double lphi = li ? ph[tlo] : ph[thi];
        const bool air_absent = li ? hi_absent : lo_absent;
        const double aphi = air_absent ? 0.5 : (li ? ph[thi] : ph[tlo]);
        th = theta_d(lphi, aphi);
      }
      val = float(double(u0) - jump / th);
    }
    I->faces[own] = val;
  }
}

__global__ void __launch_bounds__(256) k_at_project0(AInst* I) {
  const ALevel& L = I->lv[0];
  const int slot = blockIdx.x;
  __shared__ double xs[kTile];
  __shared__ float ph[kTile];
  __shared__ uint8_t lb[kTile];
  __shared__ int nbs[6], nbw[6];
  brick_sides(I, slot, nbs, nbw);
  __syncthreads();
  load_tile<double>(slot, nbs, I->x, xs);
  load_tile<float>(slot, nbs, L.phi, ph);
  load_tile<uint8_t>(slot, nbs, L.label, lb);
  project_axis<0>(I, slot, nbs, nbw, xs, ph, lb);
  project_axis<1>(I, slot, nbs, nbw, xs, ph, lb);
  project_axis<2>(I, slot, nbs, nbw, xs, ph, lb);
}

__global__ void k_at_pressure(AInst* I, float* out, double pscale) {
  const ALevel& L = I->lv[0];
  A_CELLS(L) out[i] = L.label[i] ? float(I->x[i] * pscale) : 0.0f;
}

#undef A_CELLS

}  // namespace atlas
}  // namespace fpp

// ==================================================================== host
using namespace fpp;
using namespace fpp::atlas;

namespace {

struct HostLevel {
  int B, dx, dy, dz, gx, gy, gz;
  std::vector<int> table, coords, children, parent;
  long long n() const { return (long long)coords.size() / 3 * B * B * B; }
};

// The block hierarchy: levels with 4, 2, 1 cells per brick edge, then block
// grids halved until at most kAtCoarseMax cells remain.
std::vector<HostLevel> plan_levels(int nx, int ny, int nz, const std::vector<int>& coords) {
  std::vector<HostLevel> lv;
  HostLevel L0;
  L0.B = kRes;
  L0.dx = nx;
  L0.dy = ny;
  L0.dz = nz;
  L0.gx = nx / kRes;
  L0.gy = ny / kRes;
  L0.gz = nz / kRes;
  L0.coords = coords;
  L0.table.assign(size_t(L0.gx) * L0.gy * L0.gz, -1);
  for (size_t s = 0; s < coords.size() / 3; ++s)
    L0.table[coords[3 * s] + size_t(L0.gx) * (coords[3 * s + 1] + size_t(L0.gy) * coords[3 * s + 2])] = int(s);
  lv.push_back(std::move(L0));
  while (lv.back().n() > kAtCoarseMax && int(lv.size()) < kAtMaxLevels) {
    const HostLevel& F = lv.back();
    HostLevel C;
    if (F.B > 1) {
      C = F;
      C.B = F.B / 2;
      C.dx = F.dx / 2;
      C.dy = F.dy / 2;
      C.dz = F.dz / 2;
      C.children.clear();
      C.parent.clear();
    } else {
      C.B = 1;
      C.dx = (F.dx + 1) / 2;
      C.dy = (F.dy + 1) / 2;
      C.dz = (F.dz + 1) / 2;
      C.gx = C.dx;
      C.gy = C.dy;
      C.gz = C.dz;
      C.table.assign(size_t(C.gx) * C.gy * C.gz, -1);
      const int nf = int(F.coords.size() / 3);
      std::vector<int> parent(nf);
      for (int s = 0; s < nf; ++s) {
        const int cx = F.coords[3 * s] / 2, cy = F.coords[3 * s + 1] / 2, cz = F.coords[3 * s + 2] / 2;
        int& t = C.table[cx + size_t(C.gx) * (cy + size_t(C.gy) * cz)];
        if (t < 0) {
          t = int(C.coords.size() / 3);
          C.coords.insert(C.coords.end(), {cx, cy, cz});
        }
        parent[s] = t;
      }
      const int nc = int(C.coords.size() / 3);
      C.children.assign(size_t(8) * nc, -1);
      for (int s = 0; s < nf; ++s) {
        const int k = (F.coords[3 * s] & 1) | ((F.coords[3 * s + 1] & 1) << 1) | ((F.coords[3 * s + 2] & 1) << 2);
        C.children[8 * size_t(parent[s]) + k] = s;
      }
      lv.back().parent = std::move(parent);
    }
    lv.push_back(std::move(C));
  }
  return lv;
}

// Liquid components without a cut row (no face to an air cell or an absent
// brick): union-find over the level-0 cells, CSR of their cells.
void plan_components(const HostLevel& L, const std::vector<float>& rho, std::vector<int>& off, std::vector<int>& cells) {
  const long long n = L.n();
  std::vector<int> par(n);
  std::iota(par.begin(), par.end(), 0);
  std::function<int(int)> find = [&](int a) {
    while (par[a] != a) {
      par[a] = par[par[a]];
      a = par[a];
    }
    return a;
  };
  auto liquid = [&](long long i) { return 0.5f - rho[i] <= 0.0f; };
  std::vector<uint8_t> anchored(n, 0);
  for (long long i = 0; i < n; ++i) {
    if (!liquid(i)) continue;
    const int slot = int(i / kCells), loc = int(i % kCells);
    const int l[3] = {loc % kRes, (loc / kRes) % kRes, loc / (kRes * kRes)};
    const int g[3] = {L.coords[3 * slot] * kRes + l[0], L.coords[3 * slot + 1] * kRes + l[1],
                      L.coords[3 * slot + 2] * kRes + l[2]};
    const int dom[3] = {L.dx, L.dy, L.dz};
    for (int a = 0; a < 3; ++a)
      for (int s = -1; s <= 1; s += 2) {
        int gg[3] = {g[0], g[1], g[2]};
        gg[a] += s;
        if (gg[a] < 0 || gg[a] >= dom[a]) continue;   // wall
        const int t = L.table[gg[0] / kRes + size_t(L.gx) * (gg[1] / kRes + size_t(L.gy) * (gg[2] / kRes))];
        if (t < 0) {
          anchored[i] = 1;   // sparse-air row
          continue;
        }
        const long long j = (long long)t * kCells + (gg[0] % kRes) + kRes * ((gg[1] % kRes) + kRes * (gg[2] % kRes));
        if (!liquid(j)) {
          anchored[i] = 1;
          continue;
        }
        const int ra = find(int(i)), rb = find(int(j));
        if (ra != rb) par[std::max(ra, rb)] = std::min(ra, rb);
      }
  }
  std::vector<uint8_t> root_anchor(n, 0);
  for (long long i = 0; i < n; ++i)
    if (liquid(i) && anchored[i]) root_anchor[find(int(i))] = 1;
  std::vector<int> comp_of(n, -1);
  std::vector<int> roots;
  for (long long i = 0; i < n; ++i) {
    if (!liquid(i)) continue;
    const int r = find(int(i));
    if (root_anchor[r]) continue;
    if (comp_of[r] < 0) {
      comp_of[r] = int(roots.size());
      roots.push_back(r);
    }
  }
  off.assign(roots.size() + 1, 0);
  for (long long i = 0; i < n; ++i)
    if (liquid(i) && !root_anchor[find(int(i))]) ++off[comp_of[find(int(i))] + 1];
  for (size_t c = 0; c < roots.size(); ++c) off[c + 1] += off[c];
  cells.assign(off.back(), 0);
  std::vector<int> fill(off.begin(), off.end() - 1);
  for (long long i = 0; i < n; ++i)
    if (liquid(i) && !root_anchor[find(int(i))]) cells[fill[comp_of[find(int(i))]]++] = int(i);
}

int grid_n(long long n) { return int(std::max(1LL, std::min<long long>((n + kAT - 1) / kAT, kAGrid))); }

}  // namespace

struct fluid_pp_atlas {
  fluid_pp_atlas_config cfg{};
  cudaStream_t stream = nullptr;
  std::string err;
  char* arena = nullptr;   // level arrays, CG vectors, tables, faces
  size_t arena_bytes = 0;
  AInst inst{};
  AInst* d_inst = nullptr;
  ACtrl* h_ctrl = nullptr;  // pinned
  int nb = 0;
  float dt = 0.0f;
  bool has_state = false;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};   // one iteration: Jacobi, V-cycle
  bool graph_failed[2] = {false, false};
  bool use_graphs = true;
  int pre = 1, post = 1;   // red-black sweeps before and after the coarse correction (every level)
  int small_first = 0;     // first level of the one-CTA V-cycle tail (k_at_vsmall), 0 = none
  int set_error(int code, const std::string& m) {
    err = m;
    return code;
  }
};

namespace {

std::mutex g_atlas_err_mutex;
std::string g_atlas_err;

int global_error(int code, const std::string& m) {
  std::lock_guard<std::mutex> lock(g_atlas_err_mutex);
  g_atlas_err = m;
  return code;
}

void proj(fluid_pp_atlas* A, double* v, cudaStream_t s) {
  if (A->inst.ncomp == 0) return;
  k_at_comp_mean<<<A->inst.ncomp, kAT, 0, s>>>(A->d_inst, v);
  k_at_comp_sub<<<dim3(8, A->inst.ncomp), kAT, 0, s>>>(A->d_inst, v);
}

void vcycle(fluid_pp_atlas* A, cudaStream_t s, bool vin) {
  const AInst& I = A->inst;
  if (vin) k_at_vin<<<grid_n(I.lv[0].n), kAT, 0, s>>>(A->d_inst);
  const int last = I.nlev - 1;
  const int fs = A->small_first;   // levels fs .. last in one CTA
  const int grid_last = fs > 0 ? fs : last;
  // levels 1 and 2 (4 and 2 cells per brick edge) run block-tiled kernels
  auto smooth = [&](int l, int colour, int zero) {
    const ALevel& L = I.lv[l];
    if (L.B == 4) k_at_smooth_t<4, 2><<<(L.nblocks + 1) / 2, 128, 0, s>>>(A->d_inst, l, colour, zero);
    else if (L.B == 2) k_at_smooth_t<2, 16><<<(L.nblocks + 15) / 16, 128, 0, s>>>(A->d_inst, l, colour, zero);
    else k_at_smooth<<<grid_n(L.n), kAT, 0, s>>>(A->d_inst, l, colour, zero);
  };
  // the residual and its restriction into level l + 1 (one kernel where level
  // l + 1 holds the same bricks' blocks)
  auto residual_restrict = [&](int l) {
    const ALevel& L = I.lv[l];
    if (l == 0) k_at_residual0<<<I.nb, 256, 0, s>>>(A->d_inst);
    else if (L.B == 4) k_at_residual_t<4, 2><<<(L.nblocks + 1) / 2, 128, 0, s>>>(A->d_inst, l);
    else if (L.B == 2) k_at_residual_t<2, 16><<<(L.nblocks + 15) / 16, 128, 0, s>>>(A->d_inst, l);
    else {
      k_at_residual<<<grid_n(L.n), kAT, 0, s>>>(A->d_inst, l);
      k_at_restrict<<<grid_n(I.lv[l + 1].n), kAT, 0, s>>>(A->d_inst, l);
    }
  };
  for (int l = 0; l < grid_last; ++l) {
    const int g = grid_n(I.lv[l].n);
    if (l == 0) k_at_smooth0_zero<<<I.nb, 256, 0, s>>>(A->d_inst);   // first colour from zero
    else smooth(l, 0, 1);
    if (l == 0) {
      k_at_smooth0<<<I.nb, 256, 0, s>>>(A->d_inst, 1);
      for (int k = 1; k < A->pre; ++k) {
        k_at_smooth0<<<I.nb, 256, 0, s>>>(A->d_inst, 0);
        k_at_smooth0<<<I.nb, 256, 0, s>>>(A->d_inst, 1);
      }
    } else {
      smooth(l, 1, 0);
      for (int k = 1; k < A->pre; ++k) {
        smooth(l, 0, 0);
        smooth(l, 1, 0);
      }
    }
    residual_restrict(l);
  }
  if (fs > 0) k_at_vsmall<<<1, 1024, 0, s>>>(A->d_inst, fs, A->pre, A->post);
  else k_at_coarse_apply<<<1, 1024, 0, s>>>(A->d_inst);
  for (int l = grid_last - 1; l >= 0; --l) {
    const int g = grid_n(I.lv[l].n);
    k_at_prolong<<<g, kAT, 0, s>>>(A->d_inst, l);
    for (int k = 0; k < A->post; ++k) {
      if (l == 0) {
        k_at_smooth0<<<I.nb, 256, 0, s>>>(A->d_inst, 1);
        k_at_smooth0<<<I.nb, 256, 0, s>>>(A->d_inst, 0);
      } else {
        smooth(l, 1, 0);
        smooth(l, 0, 0);
      }
    }
  }
}

// One PCG iteration on stream s (kernels skip their work once the solve is done).
// Without liquid components free of air (no projections) the V-cycle's input
// is written by the previous update (and by the start for the first
// iteration), and z is formed with its dot product in one pass.
void iteration(fluid_pp_atlas* A, cudaStream_t s) {
  const AInst& I = A->inst;
  const int g0 = grid_n(I.lv[0].n);
  const bool fused = I.ncomp == 0;
  if (I.precond) vcycle(A, s, !fused);
  if (fused) {
    k_at_zdot<<<kRedGrid, kAT, 0, s>>>(A->d_inst);
  } else {
    k_at_zvec<<<g0, kAT, 0, s>>>(A->d_inst);
    proj(A, I.q, s);
    k_at_dot_rq<<<kRedGrid, kAT, 0, s>>>(A->d_inst);
  }
  k_at_fold<<<1, kAT, 0, s>>>(A->d_inst, 1, 0);
  k_at_dir<<<g0, kAT, 0, s>>>(A->d_inst);
  proj(A, I.d, s);
  k_at_spmv0<<<I.nb, 256, 0, s>>>(A->d_inst, I.bpart);
  k_at_fold_bricks<<<1, 256, 0, s>>>(A->d_inst, I.bpart, 1);   // also sets gamma from red[0]
  if (fused && I.precond) k_at_update<true><<<kRedGrid, kAT, 0, s>>>(A->d_inst);
  else k_at_update<false><<<kRedGrid, kAT, 0, s>>>(A->d_inst);
  if (I.ncomp) {
    proj(A, I.x, s);
    proj(A, I.r, s);
    k_at_rr<<<kRedGrid, kAT, 0, s>>>(A->d_inst);
  }
  k_at_fold_check<<<1, kAT, 0, s>>>(A->d_inst);
}

// The iteration as a CUDA graph, captured once per upload and preconditioner
// on a private stream (the caller's may be the legacy stream); on any
// failure the solve launches the same kernels directly.
cudaGraphExec_t iteration_graph(fluid_pp_atlas* A) {
  const int k = A->inst.precond ? 1 : 0;
  if (A->graph[k] || A->graph_failed[k]) return A->graph[k];
  cudaStream_t cs = nullptr;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    iteration(A, cs);
    e = cudaStreamEndCapture(cs, &g);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&A->graph[k], g, 0);
  if (g) cudaGraphDestroy(g);
  if (cs) cudaStreamDestroy(cs);
  if (e != cudaSuccess) {
    A->graph[k] = nullptr;
    A->graph_failed[k] = true;
    cudaGetLastError();
  }
  return A->graph[k];
}

void drop_graphs(fluid_pp_atlas* A) {
  for (int k = 0; k < 2; ++k) {
    if (A->graph[k]) cudaGraphExecDestroy(A->graph[k]);
    A->graph[k] = nullptr;
    A->graph_failed[k] = false;
  }
}

}  // namespace

extern "C" {

const char* fluid_pp_atlas_last_error(fluid_pp_atlas* A) {
  if (A) return A->err.c_str();
  std::lock_guard<std::mutex> lock(g_atlas_err_mutex);
  return g_atlas_err.c_str();
}

int fluid_pp_atlas_plan(int nx, int ny, int nz, int nbricks, const int* coords, const float* density,
                        int* level_count, long long* level_cells, int* components, int* component_cells) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || nx % kRes || ny % kRes || nz % kRes || nbricks <= 0 || !coords || !level_count)
    return global_error(FLUID_PP_INVALID_ARG, "atlas plan: bad arguments");
  const int gx = nx / kRes, gy = ny / kRes, gz = nz / kRes;
  std::vector<int> c(coords, coords + 3 * size_t(nbricks));
  std::vector<uint8_t> seen(size_t(gx) * gy * gz, 0);
  for (int b = 0; b < nbricks; ++b) {
    const int x = c[3 * b], y = c[3 * b + 1], z = c[3 * b + 2];
    if (x < 0 || y < 0 || z < 0 || x >= gx || y >= gy || z >= gz)
      return global_error(FLUID_PP_INVALID_ARG, "a brick lies outside the domain");
    uint8_t& m = seen[x + size_t(gx) * (y + size_t(gy) * z)];
    if (m) return global_error(FLUID_PP_INVALID_ARG, "a brick is given twice");
    m = 1;
  }
  const std::vector<HostLevel> lv = plan_levels(nx, ny, nz, c);
  *level_count = int(lv.size());
  if (level_cells)
    for (size_t l = 0; l < lv.size(); ++l) level_cells[l] = lv[l].n();
  if (density && (components || component_cells)) {
    std::vector<float> rho(density, density + size_t(nbricks) * kCells);
    std::vector<int> off, cells;
    plan_components(lv[0], rho, off, cells);
    if (components) *components = int(off.size()) - 1;
    if (component_cells) *component_cells = int(cells.size());
  }
  return FLUID_PP_OK;
}

int fluid_pp_atlas_create(const fluid_pp_atlas_config* cfg, fluid_pp_atlas** out) {
  if (!cfg || !out) return FLUID_PP_INVALID_ARG;
  *out = nullptr;
  if (cfg->nx <= 0 || cfg->ny <= 0 || cfg->nz <= 0 || cfg->nx % kRes || cfg->ny % kRes || cfg->nz % kRes)
    return global_error(FLUID_PP_INVALID_ARG, "atlas domain must be positive multiples of 8 cells per axis");
  if (!(cfg->h > 0.0f) || !(cfg->rho > 0.0f) || !std::isfinite(cfg->h) || !std::isfinite(cfg->rho))
    return global_error(FLUID_PP_INVALID_ARG, "h and rho must be positive and finite");
  const long long bricks = (long long)(cfg->nx / kRes) * (cfg->ny / kRes) * (cfg->nz / kRes);
  if (bricks > (1LL << 22)) return global_error(FLUID_PP_INVALID_ARG, "brick grid too large");
  if (cudaSetDevice(cfg->device) != cudaSuccess) return global_error(FLUID_PP_CUDA, "cannot select the device");
  auto A = std::make_unique<fluid_pp_atlas>();
  A->cfg = *cfg;
  cudaError_t e = dev_alloc(reinterpret_cast<void**>(&A->d_inst), sizeof(AInst));
  if (e == cudaSuccess) e = host_alloc(reinterpret_cast<void**>(&A->h_ctrl), sizeof(ACtrl));
  if (e != cudaSuccess) {
    dev_release(A->d_inst, A->stream);
    return global_error(FLUID_PP_OOM, std::string("atlas: ") + cudaGetErrorString(e));
  }
  *out = A.release();
  return FLUID_PP_OK;
}

void fluid_pp_atlas_destroy(fluid_pp_atlas* A) {
  if (!A) return;
  cudaSetDevice(A->cfg.device);
  drop_graphs(A);
  dev_release(A->arena, A->stream);
  dev_release(A->d_inst, A->stream);
  host_release(A->h_ctrl, A->stream);
  delete A;
}

int fluid_pp_atlas_set_graphs(fluid_pp_atlas* A, int on) {
  if (!A) return FLUID_PP_INVALID_ARG;
  A->use_graphs = on != 0;
  return FLUID_PP_OK;
}

int fluid_pp_atlas_set_stream(fluid_pp_atlas* A, void* stream) {
  if (!A) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(A->cfg.device);
  const cudaStream_t next = static_cast<cudaStream_t>(stream);
  const cudaError_t e = order_streams(A->stream, next);
  if (e != cudaSuccess) return A->set_error(FLUID_PP_CUDA, cudaGetErrorString(e));
  A->stream = next;
  return FLUID_PP_OK;
}

int fluid_pp_atlas_upload(fluid_pp_atlas* A, int nbricks, const int* coords, const float* density, const float* faces) {
  if (!A || nbricks <= 0 || !coords || !density || !faces) return FLUID_PP_INVALID_ARG;
  const int gx = A->cfg.nx / kRes, gy = A->cfg.ny / kRes, gz = A->cfg.nz / kRes;
  std::vector<int> c(coords, coords + 3 * size_t(nbricks));
  std::vector<uint8_t> seen(size_t(gx) * gy * gz, 0);
  for (int s = 0; s < nbricks; ++s) {
    const int x = c[3 * s], y = c[3 * s + 1], z = c[3 * s + 2];
    if (x < 0 || y < 0 || z < 0 || x >= gx || y >= gy || z >= gz)
      return A->set_error(FLUID_PP_INVALID_ARG, "a brick lies outside the domain");
    uint8_t& m = seen[x + size_t(gx) * (y + size_t(gy) * z)];
    if (m) return A->set_error(FLUID_PP_INVALID_ARG, "a brick is given twice");
    m = 1;
  }
  const long long n0 = (long long)nbricks * kCells;
  std::vector<float> rho(density, density + n0);
  for (long long i = 0; i < n0; ++i)
    if (!std::isfinite(rho[i])) return A->set_error(FLUID_PP_NONFINITE, "non-finite density");
  std::vector<HostLevel> lv = plan_levels(A->cfg.nx, A->cfg.ny, A->cfg.nz, c);
  if (lv.back().n() > kAtCoarseMax)
    return A->set_error(FLUID_PP_UNSUPPORTED, "the brick hierarchy does not reach a small coarsest level");
  std::vector<int> comp_off, comp_cells;
  plan_components(lv[0], rho, comp_off, comp_cells);
  const int ncomp = int(comp_off.size()) - 1;
  if (ncomp > 65535) return A->set_error(FLUID_PP_UNSUPPORTED, "more than 65535 liquid components without air");
  // arena: per level 1 + 5 x 4 bytes per cell and its int tables; level-0
  // CG vectors (b x r d q float64), density, faces, partials, components
  size_t bytes = 0;
  auto up = [](size_t v) { return (v + 255) / 256 * 256; };
  for (const HostLevel& L : lv) {
    const size_t n = size_t(L.n());
    bytes += up(n) + 5 * up(4 * n) + up(4 * L.table.size()) + up(4 * L.coords.size()) + up(4 * L.children.size()) +
             up(4 * L.parent.size());
  }
  bytes += 5 * up(8 * size_t(n0)) + up(4 * size_t(n0)) + up(4 * size_t(nbricks) * 3 * kFaces);
  bytes += up(8 * size_t(nbricks)) + up(8 * 4 * kRedGrid) + up(8 * kAtCoarseMax * kAtCoarseMax) + up(4 * comp_off.size()) +
           up(4 * comp_cells.size()) + up(8 * std::max(ncomp, 1)) + up(sizeof(ACtrl));
  cudaSetDevice(A->cfg.device);
  cudaStream_t s = A->stream;
  drop_graphs(A);   // the graphs hold the old hierarchy's launch shapes
  if (bytes > A->arena_bytes) {
    dev_release(A->arena, s);
    A->arena_bytes = 0;
    const cudaError_t e = dev_alloc(reinterpret_cast<void**>(&A->arena), bytes);
    if (e != cudaSuccess) return A->set_error(FLUID_PP_OOM, std::string("atlas arena: ") + cudaGetErrorString(e));
    A->arena_bytes = bytes;
  }
  char* p = A->arena;
  auto take = [&](size_t b) {
    void* r = p;
    p += up(b);
    return r;
  };
  AInst& I = A->inst;
  I = AInst{};
  I.nlev = int(lv.size());
  I.nb = nbricks;
  // the levels from the first one of at most kAtSmallCells cells (not level
  // 0, whose kernels are brick-tiled) down to the coarsest run in one CTA
  A->small_first = 0;
  for (int l = 1; l + 1 < I.nlev; ++l)
    if (lv[l].n() <= kAtSmallCells) {
      A->small_first = l;
      break;
    }
  cudaError_t e = cudaSuccess;
  auto put = [&](const void* src, size_t b) -> void* {
    void* d = take(b);
    if (b && e == cudaSuccess) e = cudaMemcpyAsync(d, src, b, cudaMemcpyHostToDevice, s);
    return d;
  };
  for (int l = 0; l < I.nlev; ++l) {
    const HostLevel& H = lv[l];
    ALevel& L = I.lv[l];
    const size_t n = size_t(H.n());
    L.B = H.B;
    L.dx = H.dx;
    L.dy = H.dy;
    L.dz = H.dz;
    L.gx = H.gx;
    L.gy = H.gy;
    L.gz = H.gz;
    L.nblocks = int(H.coords.size() / 3);
    L.n = (long long)n;
    L.label = static_cast<uint8_t*>(take(n));
    L.phi = static_cast<float*>(take(4 * n));
    L.diag = static_cast<float*>(take(4 * n));
    L.z = static_cast<float*>(take(4 * n));
    L.rhs = static_cast<float*>(take(4 * n));
    L.res = static_cast<float*>(take(4 * n));
    L.table = static_cast<const int*>(put(H.table.data(), 4 * H.table.size()));
    L.coords = static_cast<const int*>(put(H.coords.data(), 4 * H.coords.size()));
    L.children = H.children.empty() ? nullptr : static_cast<const int*>(put(H.children.data(), 4 * H.children.size()));
    L.parent = H.parent.empty() ? nullptr : static_cast<const int*>(put(H.parent.data(), 4 * H.parent.size()));
  }
  I.b = static_cast<double*>(take(8 * size_t(n0)));
  I.x = static_cast<double*>(take(8 * size_t(n0)));
  I.r = static_cast<double*>(take(8 * size_t(n0)));
  I.d = static_cast<double*>(take(8 * size_t(n0)));
  I.q = static_cast<double*>(take(8 * size_t(n0)));
  float* d_rho = static_cast<float*>(put(rho.data(), 4 * size_t(n0)));
  {   // each brick's six neighbours: a slot, absent, or beyond a domain face
    const HostLevel& H = lv[0];
    std::vector<int> bnb(6 * size_t(nbricks));
    for (int k = 0; k < nbricks; ++k)
      for (int f = 0; f < 6; ++f) {
        int b[3] = {H.coords[3 * k], H.coords[3 * k + 1], H.coords[3 * k + 2]};
        const int a = f >> 1, g[3] = {H.gx, H.gy, H.gz};
        b[a] += (f & 1) ? 1 : -1;
        int t = kBrickWall;
        if (b[a] >= 0 && b[a] < g[a]) {
          t = H.table[b[0] + size_t(H.gx) * (b[1] + size_t(H.gy) * b[2])];
          if (t < 0) t = kBrickAbsent;
        }
        bnb[6 * size_t(k) + f] = t;
      }
    I.bnb = static_cast<const int*>(put(bnb.data(), 4 * bnb.size()));
  }
  I.faces = static_cast<float*>(put(faces, 4 * size_t(nbricks) * 3 * kFaces));
  I.part = static_cast<double*>(take(8 * 4 * kRedGrid));
  I.bpart = static_cast<double*>(take(16 * size_t(nbricks)));
  I.coarse_inv = static_cast<double*>(take(8 * kAtCoarseMax * kAtCoarseMax));
  I.coarse_m = int(lv.back().n());
  I.ncomp = ncomp;
  I.comp_off = static_cast<const int*>(put(comp_off.data(), 4 * comp_off.size()));
  I.comp_cells = static_cast<const int*>(put(comp_cells.data(), 4 * comp_cells.size()));
  I.comp_mean = static_cast<double*>(take(8 * std::max(ncomp, 1)));
  I.ctrl = static_cast<ACtrl*>(take(sizeof(ACtrl)));
  if (e == cudaSuccess) e = cudaMemcpyAsync(A->d_inst, &I, sizeof(AInst), cudaMemcpyHostToDevice, s);
  // labels, phi and diagonals of every level, the coarsest inverse
  if (e == cudaSuccess) {
    k_at_label<<<grid_n(n0), kAT, 0, s>>>(A->d_inst, d_rho);
    for (int l = 0; l + 1 < I.nlev; ++l) k_at_coarsen<<<grid_n(I.lv[l + 1].n), kAT, 0, s>>>(A->d_inst, l);
    for (int l = 0; l < I.nlev; ++l) k_at_diag<<<grid_n(I.lv[l].n), kAT, 0, s>>>(A->d_inst, l);
    k_at_coarse_factor<<<1, 1024, 0, s>>>(A->d_inst);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return A->set_error(FLUID_PP_CUDA, std::string("atlas upload: ") + cudaGetErrorString(e));
  A->nb = nbricks;
  A->has_state = true;
  return FLUID_PP_OK;
}

int fluid_pp_atlas_project(fluid_pp_atlas* A, float dt, const fluid_pp_solve_opts* opts, fluid_pp_receipt* receipt) {
  if (!A) return FLUID_PP_INVALID_ARG;
  if (!A->has_state) return A->set_error(FLUID_PP_INVALID_ARG, "state not uploaded");
  if (!(dt > 0.0f) || !std::isfinite(dt)) return A->set_error(FLUID_PP_INVALID_ARG, "dt must be positive and finite");
  double rel = 1e-6, abs_tol = 0.0;
  int max_iters = 200, cycle = 0;
  if (opts) {
    rel = opts->rel_tol;
    abs_tol = opts->abs_tol;
    max_iters = opts->max_iters;
    cycle = opts->cycle;
  }
  if (cycle != 0 && cycle != 2)
    return A->set_error(FLUID_PP_UNSUPPORTED, "atlas preconditioners: cycle 0 (V-cycle) or 2 (Jacobi)");
  const int pre = opts ? opts->pre_sweeps : 2, post = opts ? opts->post_sweeps : 2;
  if (pre < 1 || post < 1 || pre > 4 || post > 4) return A->set_error(FLUID_PP_INVALID_ARG, "sweeps: 1 to 4");
  if (pre != A->pre || post != A->post) {   // the iteration graphs hold the launch sequence
    A->pre = pre;
    A->post = post;
    drop_graphs(A);
  }
  if (!(rel >= 0.0) || !(abs_tol >= 0.0) || max_iters <= 0) return A->set_error(FLUID_PP_INVALID_ARG, "bad solve options");
  cudaSetDevice(A->cfg.device);
  AInst& I = A->inst;
  I.precond = cycle == 0 ? 1 : 0;
  cudaStream_t s = A->stream;
  cudaError_t e = cudaMemcpyAsync(&A->d_inst->precond, &I.precond, sizeof(int), cudaMemcpyHostToDevice, s);
  const long long n0 = I.lv[0].n;
  const int g0 = grid_n(n0);
  // divergence before, the right-hand side, the start
  k_at_div0<<<I.nb, 256, 0, s>>>(A->d_inst, 1, I.bpart);
  k_at_div_fold_bricks<<<1, 256, 0, s>>>(A->d_inst, I.bpart, 0);
  proj(A, I.b, s);
  k_at_bb<<<kRedGrid, kAT, 0, s>>>(A->d_inst);
  k_at_fold<<<1, kAT, 0, s>>>(A->d_inst, 2, 0);
  k_at_init<<<1, 1, 0, s>>>(A->d_inst, rel, abs_tol, max_iters);
  k_at_start<<<g0, kAT, 0, s>>>(A->d_inst);
  const int poll = 8;
  cudaGraphExec_t gx = A->use_graphs ? iteration_graph(A) : nullptr;
  for (int it = 0; it < max_iters; ++it) {
    if (gx) e = cudaGraphLaunch(gx, s);
    else iteration(A, s);
    if (e != cudaSuccess) break;
    if ((it + 1) % poll == 0) {
      e = cudaMemcpyAsync(A->h_ctrl, I.ctrl, sizeof(ACtrl), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) break;
      if (A->h_ctrl->done) break;
    }
  }
  // float64 true residual, projected faces, receipts
  k_at_true<<<kRedGrid, kAT, 0, s>>>(A->d_inst);
  k_at_fold<<<1, kAT, 0, s>>>(A->d_inst, 1, 1);
  k_at_project0<<<I.nb, 256, 0, s>>>(A->d_inst);
  k_at_div0<<<I.nb, 256, 0, s>>>(A->d_inst, 0, I.bpart);
  k_at_div_fold_bricks<<<1, 256, 0, s>>>(A->d_inst, I.bpart, 2);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(A->h_ctrl, I.ctrl, sizeof(ACtrl), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return A->set_error(FLUID_PP_CUDA, std::string("atlas project: ") + cudaGetErrorString(e));
  const ACtrl& C = *A->h_ctrl;
  int status = C.status;
  if (!C.done) status = FLUID_PP_NONCONVERGENCE;
  A->dt = dt;
  if (receipt) {
    const double h = A->cfg.h;
    receipt->status = status;
    receipt->iterations = C.iter;
    receipt->liquid_cells = int(C.liquid);
    receipt->levels = I.precond ? I.nlev : 1;
    receipt->b_norm = std::sqrt(C.bb);
    receipt->rel_residual = C.bb > 0 ? std::sqrt(C.rr / C.bb) : 0.0;
    receipt->true_rel_residual = C.bb > 0 ? std::sqrt(C.red[1] / C.bb) : 0.0;
    // b = h div u per cell: div in 1/s, the L2 norm over the liquid volume
    receipt->max_div_before = C.div[0] / h;
    receipt->l2_div_before = std::sqrt(C.div[1] * h);
    receipt->max_div_after = C.div[2] / h;
    receipt->l2_div_after = std::sqrt(C.div[3] * h);
  }
  return status;
}

int fluid_pp_atlas_download(fluid_pp_atlas* A, float* pressure, float* faces) {
  if (!A) return FLUID_PP_INVALID_ARG;
  if (!A->has_state) return A->set_error(FLUID_PP_INVALID_ARG, "state not uploaded");
  cudaSetDevice(A->cfg.device);
  cudaStream_t s = A->stream;
  const long long n0 = A->inst.lv[0].n;
  cudaError_t e = cudaSuccess;
  float* tmp = nullptr;
  if (pressure) {
    if (!(A->dt > 0.0f)) return A->set_error(FLUID_PP_INVALID_ARG, "no projection yet");
    e = dev_alloc(reinterpret_cast<void**>(&tmp), sizeof(float) * size_t(n0));
    if (e == cudaSuccess) {
      const double pscale = double(A->cfg.rho) * double(A->cfg.h) / double(A->dt);
      k_at_pressure<<<grid_n(n0), kAT, 0, s>>>(A->d_inst, tmp, pscale);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(pressure, tmp, sizeof(float) * size_t(n0), cudaMemcpyDeviceToHost, s);
  }
  if (e == cudaSuccess && faces)
    e = cudaMemcpyAsync(faces, A->inst.faces, sizeof(float) * size_t(A->nb) * 3 * kFaces, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  dev_release(tmp, s);
  if (e != cudaSuccess) return A->set_error(FLUID_PP_CUDA, std::string("atlas download: ") + cudaGetErrorString(e));
  return FLUID_PP_OK;
}

}  // extern "C"

