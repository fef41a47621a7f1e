// Device-visible descriptors shared by the host orchestration and the kernels.
#pragma once
#include <cstdint>

#include "plan.h"

namespace fpp {

constexpr int kThreads = 256;      // threads per CTA for the grid kernels
constexpr int kFThreads = 512;     // threads per CTA for the fused shared-memory kernels
constexpr int kMaxCoarse = 128;    // largest coarsest level solved densely
constexpr int kSlots = 6;          // reduction quantities per stage
constexpr int kCoarseBlockCells = 4096;          // levels this small run inside one CTA
constexpr int kCoarseBlockSmem = 160 * 1024;     // shared-memory budget of that CTA

// Per-solve control word block, one per instance, resident on the device.
// All scalar CG state lives here so no host round trip is needed inside a solve.
struct Ctrl {
  double bb;          // ||b||^2
  double thr2;        // stopping threshold squared
  double gamma;       // r.z of the current direction
  double beta;
  double delta;       // d.Ad
  double alpha;
  double rr;          // recursive ||r||^2
  double rr_true;     // float64 ||b - A x||^2
  double zmean;       // mean of z over liquid cells (unanchored systems only)
  double bmean;
  double sigma;       // preconditioner input scale (keeps half-precision levels in range)
  double bmax;        // max |b| over liquid cells
  double rmax;        // max |r| of the last residual (recursive or true)
  double thr_inf;     // max-norm threshold (0: criterion off)
  double red[kSlots]; // last finalised reduction values
  double zmean_prev;  // zmean of the previous preconditioned residual (flexible CG)
  int iter;
  int max_iter;
  int true_every;
  int first;          // 1 until the first direction is formed
  int candidate;      // recursive residual below threshold; awaiting float64 check
  int done;           // solve finished (converged or failed)
  int status;         // FLUID_PP_* status of the solve
  int liquid;         // liquid cells on the finest level
  int air;            // air cells on the finest level
  int top_liquid;     // liquid cells in the top row (open-top anchoring)
  int nonfinite;      // non-finite input seen
  int anchored;       // finest system has a Dirichlet contact
  int converged;
  unsigned arrive[8]; // per-stage completion counters (self-resetting)
  int dsel;           // which of d / d2 holds the current search direction
  int fcg;            // 1: full-cycle preconditioner under flexible CG (Polak-Ribiere beta)
};

struct LevelDev {
  int nx, ny, nz;
  int sx, sy, sz;     // coarsening factor from the next finer level (1 or 2)
  long long n;
  int ntiles;
  int depth;          // cells per thread along z in this level's work tiles
  int dcx, dcy, dcz;  // fused down step l -> l+1: coarse cells per tile (level l+1 units)
  int dtiles;         // tiles of that step
  int utx, uty, utz;  // fused up step l+1 -> l: fine cells per tile
  int utiles;
  int cdz;            // column down step l -> l+1: coarse planes per tile (levels coarsened by two on every axis)
  int cuz;            // column up step l+1 -> l: fine planes per tile (a multiple of 8 on level 0)
  int cqz;            // level 0: direction + SpMV, fine planes per tile (a multiple of 8)
  float wx, wy, wz;   // normalised off-diagonal weights w_a / wmax
  float wmax;         // (h0 / h_a)^2 maximum over axes; level operators are stored divided by it
  float ext_phi;      // open-top exterior phi (finest-cell units)
  float to_coarse;    // wmax(l) / wmax(l+1): restriction rescale into the next level's units
  uint8_t* label;     // 1 liquid, 0 air
  float* phi;         // level set, finest-cell units
  float* diag;        // exact float32 diagonal in finest-cell units (A_l), used by SpMV on level 0
  void* diagT;        // normalised diagonal in the storage type (smoother)
  void* z;            // level solution (level 0: float CG vector)
  void* rhs;          // level right-hand side (level 0: the CG residual r, float)
  void* res;          // scratch in the z type: the pre-smoothed z between the fused down and up steps
  const float* ff;    // embedded solids: open fraction of each cell's +x, +y, +z face (planar, 3 x n), or null
  float* pmin;        // embedded solids: the LCP solve's lower bound of z (CM11a p_min), or null
};

struct InstDev {
  LevelDev lv[kMaxLevels];
  int nlev;
  int nx, ny, nz;
  int open_top;
  float h, rho, dt;
  float pscale;       // rho * h / dt : finest-cell pressure -> Pa
  int ntiles0;
  int coarse_m;       // cells of the coarsest level
  int first_block;    // first level solved by the single-CTA coarse block (nlev when none)
  int block_smem;     // shared memory that block needs, bytes
  const float* vof;
  float* u;
  float* v;
  float* w;
  float* b;           // right-hand side, finest-cell units
  float* x;           // pressure, finest-cell units: x + xlo is a double-single value
  float* xlo;         // low part of the double-single pressure
  float* d;           // search direction (double-buffered with d2, see Ctrl::dsel)
  float* d2;
  float* q;           // A d
  float* p_si;        // pressure output in Pa
  // embedded solids (null / 0 without): cell open fraction, face open fractions
  // and solid normal velocities on the MAC faces (layouts of u, v, w)
  int solids;
  const float* open;
  const float* fv[3];
  const float* us[3];
  double* partial;    // kSlots * ntiles0 per-tile reduction partials
  double* coarse_inv; // coarse_m^2 dense inverse of the coarsest operator
  Ctrl* ctrl;
};

}  // namespace fpp
