// Host orchestration and C ABI of the uniform-grid pressure projection.
//
// A handle owns one grid's device arena.  Every solve, single or batched, runs
// through a fluid_pp_batch: a device table of instance descriptors plus tile
// lists per stage, so one launch per stage covers every instance.  The CG
// scalars live on the device (Ctrl); the host only polls the done flags every
// few iterations.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "alloc.h"
#include "../../include/fluid_pp.h"
#include "colmg.cuh"
#include "fused.cuh"
#include "extrap.cuh"
#include "lcp.cuh"
#include "solids.cuh"
#include "transport.cuh"
#include "plan.h"
#include "types.h"

using namespace fpp;

namespace {

constexpr int kMaxGrid = 148 * 8;   // 148 SMs x 8 resident 256-thread CTAs
constexpr int kFillTiles = 148;  // fused-kernel tiles that give every SM one (the default fill count)

// Fused-kernel tile shapes, largest first: coarse cells per down-step tile and
// fine cells per up-step tile (level 0's up step always uses the CG kernels'
// 32 x 8 x 8 tiles, whose reduction partials it shares).
constexpr int kDownShapes[5][3] = {{16, 4, 4}, {8, 4, 4}, {8, 4, 2}, {8, 2, 2}, {4, 2, 2}};
constexpr int kUpShapes[5][3] = {{32, 8, 8}, {32, 8, 4}, {16, 8, 4}, {16, 4, 4}, {8, 4, 4}};

int shape_tiles(int n0, int n1, int n2, const int* t) {
  return ((n0 + t[0] - 1) / t[0]) * ((n1 + t[1] - 1) / t[1]) * ((n2 + t[2] - 1) / t[2]);
}

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

size_t storage_bytes(int precision) { return precision == FLUID_PP_FP32 ? 4 : 2; }

struct Arena {
  char* base = nullptr;
  size_t used = 0, cap = 0;
  void* take(size_t bytes) {
    void* p = base + used;
    used = align_up(used + bytes, 256);
    return p;
  }
};

}  // namespace

struct fluid_pp_batch;

struct fluid_pp {
  fluid_pp_config cfg{};
  HierarchyPlan plan{};
  cudaStream_t stream = nullptr;
  std::string err;
  char* arena = nullptr;
  size_t arena_bytes = 0;
  InstDev inst{};        // host copy of the descriptor (device pointers)
  Ctrl* h_ctrl = nullptr;  // pinned
  bool has_state = false;
  bool has_pressure = false;
  float last_dt = 0.f;
  fluid_pp_batch* self = nullptr;   // batch of one
  char* solid_mem = nullptr;         // embedded solids: open fractions, face fractions and velocities, level fractions
  char* ext_mem = nullptr;           // velocity extrapolation: FIM sides and the known-value hierarchy
  char* tr_mem = nullptr;            // density transport: persistent gamma, scratch fields, fixed-point deposits
  long long plan_cells() const { return (long long)cfg.nx * cfg.ny * cfg.nz; }
  int set_error(int code, const std::string& m) {
    err = m;
    return code;
  }
};

struct List {
  int off = 0, n = 0;
};

struct fluid_pp_batch {
  std::vector<fluid_pp*> h;
  std::vector<float> dev_dt, dev_pscale;   // values last written into d_insts (NaN = not yet)
  int device = 0;
  int precision = 0;
  cudaStream_t stream = nullptr;
  InstDev* d_insts = nullptr;
  Ctrl* d_ctrl = nullptr;
  Ctrl* h_ctrl = nullptr;   // pinned mirror
  Tile* d_tiles = nullptr;
  int* d_ilist = nullptr;
  List l0;
  List lvl[kMaxLevels];      // level-l tiles of instances for which l is not the coarsest
  List rst[kMaxLevels];      // level-(l+1) tiles of instances for which l is not the coarsest
  List crs[kMaxLevels];      // level-l tiles (l >= 1) of every instance having level l
  List dn[kMaxLevels];       // fused down-step tiles (coarse tiles of level l+1) of grid level l
  List cdn[kMaxLevels];      // column down-step tiles of grid level l (next level halves every axis)
  List cup[kMaxLevels];      // column up-step tiles of grid level l (same condition)
  List cq;                   // column direction + SpMV tiles of level 0 (every instance)
  List dot0;                 // level-0 tiles of instances whose level-0 up step is a box kernel (gamma by k_dot_rz_part)
  List up[kMaxLevels];       // fused up-step tiles (fine tiles of level l) of grid level l
  List l0single;             // level-0 tiles of single-level instances
  List bake;
  List multi, single;        // instance lists (offsets into d_ilist) by coarsest level
  bool solids = false;       // the instances have embedded solids (per-pass kernels, face-weighted operators)
  List fcb[kMaxLevels];      // multi-level instances for which level l is a grid level (full-cycle coarse steps)
  int maxL = 0;
  cudaError_t launch_err = cudaSuccess;   // first failed launch since the last check
  size_t smem_factor = 0;
  size_t smem_block = 0;
  size_t smem_down = 0, smem_up = 0;
  std::string err;
  // CUDA graphs: setup, the device-side CG loop (conditional WHILE node), finish
  bool graphs_valid = false;
  fluid_pp_solve_opts graph_key{};
  cudaGraph_t g_setup = nullptr, g_loop = nullptr, g_finish = nullptr;
  cudaGraphExec_t x_setup = nullptr, x_loop = nullptr, x_finish = nullptr;
  unsigned long long n_setup = 0, n_body = 0, n_finish = 0;   // kernels per graph (body: per iteration)
  unsigned* d_loop = nullptr;   // loop-iteration counter (device)
  unsigned* h_loop = nullptr;   // pinned mirror
  bool pending_graph_count = false;
  // per-stage kernel timing (events on the launching stream), off by default
  bool profiling = false;
  // CUDA graphs for the solve (on by default); a batch whose composition changes
  // every few solves runs direct launches instead of paying for a new capture
  bool use_graphs = true;
  // Concurrent parts (batch tuning `parts` > 1): sub-batches of the handles on
  // streams of their own, each with its own graphs, launched together after an
  // event on this batch's stream and joined back to it, so that one part's
  // small launches and last iterations overlap another part's work.  Only
  // graph-mode solves use them; direct launches run the whole batch.
  std::vector<fluid_pp_batch*> parts;
  std::vector<std::vector<int>> part_idx;   // handle indices (into h) of each part
  std::vector<cudaStream_t> part_streams;
  std::vector<cudaEvent_t> part_done;
  cudaEvent_t part_start = nullptr;
  bool parts_pending = false;               // the last solve ran in parts: receipts come from them
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  std::vector<int> ev_stage;
  double prof_ms[FLUID_PP_PROFILE_STAGES] = {};
  long long prof_count[FLUID_PP_PROFILE_STAGES] = {};
};

// ------------------------------------------------------------------ helpers
namespace {

thread_local std::string g_err;

int launch_grid(int tiles) { return std::max(1, std::min(tiles, kMaxGrid)); }


const Tile* tl(const fluid_pp_batch* B, const List& L) { return B->d_tiles + L.off; }
const int* il(const fluid_pp_batch* B, const List& L) { return B->d_ilist + L.off; }

enum ProfStage {
  kPrReset = FLUID_PP_STAGE_RESET, kPrLabel = FLUID_PP_STAGE_LABEL, kPrCoarsen = FLUID_PP_STAGE_COARSEN,
  kPrBake = FLUID_PP_STAGE_BAKE, kPrFactor = FLUID_PP_STAGE_FACTOR, kPrInit = FLUID_PP_STAGE_INIT,
  kPrSmooth0 = FLUID_PP_STAGE_SMOOTH0, kPrSmoothC = FLUID_PP_STAGE_SMOOTHC, kPrResidual0 = FLUID_PP_STAGE_RESIDUAL0,
  kPrResidualC = FLUID_PP_STAGE_RESIDUALC, kPrRestrict0 = FLUID_PP_STAGE_RESTRICT0,
  kPrRestrictC = FLUID_PP_STAGE_RESTRICTC, kPrCoarse = FLUID_PP_STAGE_COARSE, kPrProlong0 = FLUID_PP_STAGE_PROLONG0,
  kPrProlongC = FLUID_PP_STAGE_PROLONGC, kPrDot = FLUID_PP_STAGE_DOT, kPrDir = FLUID_PP_STAGE_DIR,
  kPrSpmv = FLUID_PP_STAGE_SPMV, kPrUpdate = FLUID_PP_STAGE_UPDATE, kPrTrue = FLUID_PP_STAGE_TRUE,
  kPrGrad = FLUID_PP_STAGE_GRAD, kPrReceipt = FLUID_PP_STAGE_RECEIPT, kPrDown0 = FLUID_PP_STAGE_DOWN0,
  kPrDownC = FLUID_PP_STAGE_DOWNC, kPrUp0 = FLUID_PP_STAGE_UP0, kPrUpC = FLUID_PP_STAGE_UPC,
  kPrDirSpmv = FLUID_PP_STAGE_DIRSPMV
};

std::atomic<unsigned long long> g_launches{0};

cudaEvent_t next_event(fluid_pp_batch* B) {
  if (B->ev_used == B->ev_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    B->ev_pool.push_back(e);
  }
  return B->ev_pool[B->ev_used++];
}

void prof_begin(fluid_pp_batch* B, int stage) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (!B->profiling) return;
  B->ev_stage.push_back(stage);
  cudaEventRecord(next_event(B), B->stream);
}

void prof_end(fluid_pp_batch* B, int) {
  if (!B->profiling) return;
  cudaEventRecord(next_event(B), B->stream);
}

// Folds the recorded event pairs into the per-stage totals (synchronises).
void prof_collect(fluid_pp_batch* B) {
  if (B->ev_stage.empty()) return;
  cudaStreamSynchronize(B->stream);
  for (size_t k = 0; k < B->ev_stage.size(); ++k) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, B->ev_pool[2 * k], B->ev_pool[2 * k + 1]);
    B->prof_ms[B->ev_stage[k]] += ms;
    B->prof_count[B->ev_stage[k]] += 1;
  }
  B->ev_stage.clear();
  B->ev_used = 0;
}

}  // namespace


namespace {

// Every launch goes through FPP_LAUNCH: it counts the launch and, when the
// batch is profiling, brackets it with CUDA events on the launching stream.
#define FPP_LAUNCH(B, stage, ...)                                  \
  do {                                                             \
    prof_begin(B, stage);                                          \
    __VA_ARGS__;                                                   \
    const cudaError_t launch_e_ = cudaGetLastError();              \
    if (launch_e_ != cudaSuccess && (B)->launch_err == cudaSuccess) \
      (B)->launch_err = launch_e_;                                 \
    prof_end(B, stage);                                            \
  } while (0)

// Returns and clears the first launch error recorded on the batch.
cudaError_t take_launch_error(fluid_pp_batch* B) {
  const cudaError_t e = B->launch_err;
  B->launch_err = cudaSuccess;
  return e;
}

template <class T>
void setup_launch(fluid_pp_batch* B, const fluid_pp_solve_opts& o) {
  const int warm = o.warm_start;
  cudaStream_t s = B->stream;
  const int n = int(B->h.size());
  const Tile* t0 = tl(B, B->l0);
  const int n0 = B->l0.n, g0 = launch_grid(n0);
  FPP_LAUNCH(B, kPrReset, k_reset_ctrl<<<(n + 127) / 128, 128, 0, s>>>(B->d_insts, n, B->d_loop));
  if (B->solids)
    FPP_LAUNCH(B, kPrLabel, k_label_rhs_solid<<<g0, kThreads, 0, s>>>(B->d_insts, t0, n0, warm));
  else
    FPP_LAUNCH(B, kPrLabel, k_label_rhs<<<g0, kThreads, 0, s>>>(B->d_insts, t0, n0, warm));
  for (int l = 1; l < B->maxL; ++l)
    if (B->crs[l].n)
      FPP_LAUNCH(B, kPrCoarsen, k_coarsen_phi<<<launch_grid(B->crs[l].n), kThreads, 0, s>>>(B->d_insts, tl(B, B->crs[l]),
                                                                                             B->crs[l].n));
  FPP_LAUNCH(B, kPrBake, k_bake_diag<T><<<launch_grid(B->bake.n), kThreads, 0, s>>>(B->d_insts, tl(B, B->bake), B->bake.n));
  if (B->multi.n)
    FPP_LAUNCH(B, kPrFactor, k_coarse_factor<T><<<B->multi.n, kBlockThreads, B->smem_factor, s>>>(B->d_insts, il(B, B->multi)));
  if (B->single.n)
    FPP_LAUNCH(B, kPrFactor,
               k_coarse_factor<T><<<B->single.n, kBlockThreads, B->smem_factor, s>>>(B->d_insts, il(B, B->single)));
  FPP_LAUNCH(B, kPrInit, k_cg_init_part<<<g0, kThreads, 0, s>>>(B->d_insts, t0, n0, warm));
  FPP_LAUNCH(B, kPrInit, k_cg_init_finish<<<B->multi.n + B->single.n, kThreads, 0, s>>>(
                             B->d_insts, il(B, B->multi), o.rel_tol, o.abs_tol, o.max_iters, o.true_residual_every,
                             o.rel_tol_inf, o.cycle == 1));
  FPP_LAUNCH(B, kPrInit, k_project_init<<<g0, kThreads, 0, s>>>(B->d_insts, t0, n0));
}

template <class T>
void smooth_pass(fluid_pp_batch* B, int l, int colour, int zero_init, int project = 0) {
  const List& Ls = B->lvl[l];
  const int g = launch_grid(Ls.n);
  if (l == 0)
    FPP_LAUNCH(B, kPrSmooth0, k_smooth<float, float, T><<<g, kThreads, 0, B->stream>>>(B->d_insts, tl(B, Ls), Ls.n, l,
                                                                                       colour, zero_init, project));
  else
    FPP_LAUNCH(B, kPrSmoothC, k_smooth<T, T, T><<<g, kThreads, 0, B->stream>>>(B->d_insts, tl(B, Ls), Ls.n, l, colour,
                                                                               zero_init, project));
}

// One V-cycle from grid level `from` down to the coarse block and back
// (vCycle, webgpu-uniform-pressure-multigrid.ts:524-538).  Level `from` starts
// from zero, or from the z it holds when `keep` (the full cycle's prolongated
// guess); every deeper level starts from zero.  `coarse` lists the instances
// whose coarse block closes the cycle.
template <class T>
void vcycle_from(fluid_pp_batch* B, int from, int pre, int post, bool keep, const List& coarse) {
  cudaStream_t s = B->stream;
  for (int l = from; l + 1 < B->maxL; ++l) {
    const List& Ls = B->lvl[l];
    if (!Ls.n) continue;
    const bool zero = !(keep && l == from);
    for (int sw = 0; sw < pre; ++sw) {
      smooth_pass<T>(B, l, 0, zero && sw == 0);
      smooth_pass<T>(B, l, 1, 0);
    }
    if (pre == 0 && zero) smooth_pass<T>(B, l, 2, 1);   // z must start at zero
    const List& Lr = B->rst[l];
    if (l == 0)
      FPP_LAUNCH(B, kPrRestrict0, k_residual_restrict<float, float, T, T><<<launch_grid(Lr.n), kThreads, 0, s>>>(
                                      B->d_insts, tl(B, Lr), Lr.n, l));
    else
      FPP_LAUNCH(B, kPrRestrictC, k_residual_restrict<T, T, T, T><<<launch_grid(Lr.n), kThreads, 0, s>>>(
                                      B->d_insts, tl(B, Lr), Lr.n, l));
  }
  if (coarse.n)
    FPP_LAUNCH(B, kPrCoarse, k_coarse_block<T><<<coarse.n, kBlockThreads, B->smem_block, s>>>(
                                 B->d_insts, il(B, coarse), pre, post));
  if (from == 0 && B->single.n)
    FPP_LAUNCH(B, kPrCoarse,
               k_coarse_apply<float, float><<<B->single.n, kThreads, 0, s>>>(B->d_insts, il(B, B->single)));
  for (int l = B->maxL - 2; l >= from; --l) {
    const List& Ls = B->lvl[l];
    if (!Ls.n) continue;
    const int g = launch_grid(Ls.n);
    if (l == 0)
      FPP_LAUNCH(B, kPrProlong0, k_prolong<float, T><<<g, kThreads, 0, s>>>(B->d_insts, tl(B, Ls), Ls.n, l));
    else
      FPP_LAUNCH(B, kPrProlongC, k_prolong<T, T><<<g, kThreads, 0, s>>>(B->d_insts, tl(B, Ls), Ls.n, l));
    for (int sw = 0; sw < post; ++sw) {
      smooth_pass<T>(B, l, 1, 0);
      smooth_pass<T>(B, l, 0, 0);
    }
  }
}

template <class T>
void vcycle_launch(fluid_pp_batch* B, int pre, int post) {
  vcycle_from<T>(B, 0, pre, post, false, B->multi);
}

// One full cycle z = F(r), zero initial guess (fullCycle,
// webgpu-uniform-pressure-multigrid.ts:539-563): the residual restricted down
// every grid level, the coarse block's V-cycle as the coarsest correction,
// then for each grid level from the coarsest up, z_l = P z_{l+1} as the guess
// of a V-cycle started at level l.  The levels inside the coarse block (at
// most 4096 cells each) are not nested: the block's one V-cycle stands for
// their full cycle.
template <class T>
void fcycle_launch(fluid_pp_batch* B, int pre, int post) {
  cudaStream_t s = B->stream;
  // descent: z = 0 on every grid level (so prolongation below assigns), the
  // restricted right-hand side of each level is the residual of that zero guess
  for (int l = 0; l + 1 < B->maxL; ++l) {
    if (!B->lvl[l].n) continue;
    smooth_pass<T>(B, l, 2, 1);
    const List& Lr = B->rst[l];
    if (l == 0)
      FPP_LAUNCH(B, kPrRestrict0, k_residual_restrict<float, float, T, T><<<launch_grid(Lr.n), kThreads, 0, s>>>(
                                      B->d_insts, tl(B, Lr), Lr.n, l));
    else
      FPP_LAUNCH(B, kPrRestrictC, k_residual_restrict<T, T, T, T><<<launch_grid(Lr.n), kThreads, 0, s>>>(
                                      B->d_insts, tl(B, Lr), Lr.n, l));
  }
  if (B->multi.n)
    FPP_LAUNCH(B, kPrCoarse, k_coarse_block<T><<<B->multi.n, kBlockThreads, B->smem_block, s>>>(
                                 B->d_insts, il(B, B->multi), pre, post));
  if (B->single.n)
    FPP_LAUNCH(B, kPrCoarse,
               k_coarse_apply<float, float><<<B->single.n, kThreads, 0, s>>>(B->d_insts, il(B, B->single)));
  for (int l = B->maxL - 2; l >= 0; --l) {
    const List& Ls = B->lvl[l];
    if (!Ls.n) continue;
    const int g = launch_grid(Ls.n);
    if (l == 0)
      FPP_LAUNCH(B, kPrProlong0, k_prolong<float, T><<<g, kThreads, 0, s>>>(B->d_insts, tl(B, Ls), Ls.n, l));
    else
      FPP_LAUNCH(B, kPrProlongC, k_prolong<T, T><<<g, kThreads, 0, s>>>(B->d_insts, tl(B, Ls), Ls.n, l));
    vcycle_from<T>(B, l, pre, post, true, B->fcb[l]);
  }
}

// The default schedule (one sweep down, one up): per grid level one fused down
// launch and one fused up launch; the level-0 up launch also forms gamma.
template <class T>
void vcycle_fused(fluid_pp_batch* B, int with_dot) {
  cudaStream_t s = B->stream;
  for (int l = 0; l + 1 < B->maxL; ++l) {
    const List& Lm = B->cdn[l];
    if (Lm.n) {
      if (l == 0)
        FPP_LAUNCH(B, kPrDown0, k_cdown<float, float, float, T><<<Lm.n, kCDThreads, cdown_smem(), s>>>(
                                    B->d_insts, tl(B, Lm), 0));
      else
        FPP_LAUNCH(B, kPrDownC, k_cdown<T, T, T, T><<<Lm.n, kCDThreads, cdown_smem(), s>>>(B->d_insts, tl(B, Lm), l));
    }
    const List& Ld = B->dn[l];
    if (!Ld.n) continue;
    if (l == 0)
      FPP_LAUNCH(B, kPrDown0, k_down<float, float, T, T><<<Ld.n, kFThreads, B->smem_down, s>>>(B->d_insts, tl(B, Ld), 0));
    else
      FPP_LAUNCH(B, kPrDownC, k_down<T, T, T, T><<<Ld.n, kFThreads, B->smem_down, s>>>(B->d_insts, tl(B, Ld), l));
  }
  if (B->multi.n)
    FPP_LAUNCH(B, kPrCoarse, k_coarse_block<T><<<B->multi.n, kBlockThreads, B->smem_block, s>>>(
                                 B->d_insts, il(B, B->multi), 1, 1));
  if (B->single.n)
    FPP_LAUNCH(B, kPrCoarse,
               k_coarse_apply<float, float><<<B->single.n, kThreads, 0, s>>>(B->d_insts, il(B, B->single)));
  for (int l = B->maxL - 2; l >= 0; --l) {
    const List& Lc = B->cup[l];
    if (Lc.n) {
      if (l == 0 && with_dot)
        FPP_LAUNCH(B, kPrUp0, k_cup<float, float, float, T, true><<<Lc.n, kCUThreads, cup_smem(), s>>>(
                                  B->d_insts, tl(B, Lc), 0));
      else if (l == 0)
        FPP_LAUNCH(B, kPrUp0, k_cup<float, float, float, T><<<Lc.n, kCUThreads, cup_smem(), s>>>(B->d_insts,
                                                                                                 tl(B, Lc), 0));
      else
        FPP_LAUNCH(B, kPrUpC, k_cup<T, T, T, T><<<Lc.n, kCUThreads, cup_smem(), s>>>(B->d_insts, tl(B, Lc), l));
    }
    const List& Lu = B->up[l];
    if (!Lu.n) continue;
    if (l == 0)
      FPP_LAUNCH(B, kPrUp0, k_up<float, float, T, T><<<Lu.n, kFThreads, B->smem_up, s>>>(B->d_insts, tl(B, Lu), 0));
    else
      FPP_LAUNCH(B, kPrUpC, k_up<T, T, T, T><<<Lu.n, kFThreads, B->smem_up, s>>>(B->d_insts, tl(B, Lu), l));
  }
  // gamma = r . (z - zmean) over the fixed level-0 dot tiles of every
  // instance: the column level-0 up step writes the partials of its instances,
  // k_dot_rz_part those of the instances whose level 0 runs the box kernels.
  // Which of the two an instance takes depends only on its lattice, so a solve
  // gives the same bits alone and in any batch
  if (with_dot) {
    if (B->dot0.n)
      FPP_LAUNCH(B, kPrDot, k_dot_rz_part<<<launch_grid(B->dot0.n), kThreads, 0, s>>>(B->d_insts, tl(B, B->dot0),
                                                                                      B->dot0.n));
    // every instance: the multi-level list followed by the single-level one
    FPP_LAUNCH(B, kPrDot, k_dot_rz_finish<<<B->multi.n + B->single.n, kThreads, 0, s>>>(B->d_insts,
                                                                                      il(B, B->multi)));
  }
}

template <class T>
void iter_launch(fluid_pp_batch* B, const fluid_pp_solve_opts& o) {
  cudaStream_t s = B->stream;
  const Tile* t0 = tl(B, B->l0);
  const int n0 = B->l0.n, g = launch_grid(n0);
  const int pre = o.pre_sweeps, post = o.post_sweeps;
  if (o.cycle == 1) {
    // flexible CG: gamma also takes r . z_prev (z_prev kept in d2)
    fcycle_launch<T>(B, pre, post);
    FPP_LAUNCH(B, kPrDot, k_dot_rz<true><<<g, kThreads, 0, s>>>(B->d_insts, t0, n0));
  } else if (pre == 1 && post == 1 && !B->solids) {
    vcycle_fused<T>(B, 1);
    FPP_LAUNCH(B, kPrDirSpmv, k_cdirspmv<<<B->cq.n, kSThreads, 0, s>>>(B->d_insts, tl(B, B->cq)));
    FPP_LAUNCH(B, kPrDirSpmv, k_dirspmv_finish<<<B->multi.n + B->single.n, kThreads, 0, s>>>(B->d_insts,
                                                                                           il(B, B->multi)));
    FPP_LAUNCH(B, kPrUpdate, k_cupdate<<<B->cq.n, kUThreads, 0, s>>>(B->d_insts, tl(B, B->cq)));
    FPP_LAUNCH(B, kPrUpdate, k_update_finish<<<B->multi.n + B->single.n, kThreads, 0, s>>>(B->d_insts,
                                                                                         il(B, B->multi)));
    FPP_LAUNCH(B, kPrTrue, k_ctrue<<<B->cq.n, kSThreads, 0, s>>>(B->d_insts, tl(B, B->cq)));
    return;
  } else {
    vcycle_launch<T>(B, pre, post);
    FPP_LAUNCH(B, kPrDot, k_dot_rz<<<g, kThreads, 0, s>>>(B->d_insts, t0, n0));
  }
  FPP_LAUNCH(B, kPrDir, k_dir<<<g, kThreads, 0, s>>>(B->d_insts, t0, n0));
  FPP_LAUNCH(B, kPrSpmv, k_spmv<<<g, kThreads, 0, s>>>(B->d_insts, t0, n0));
  FPP_LAUNCH(B, kPrUpdate, k_update<<<g, kThreads, 0, s>>>(B->d_insts, t0, n0));
  FPP_LAUNCH(B, kPrTrue, k_true_residual<<<g, kThreads, 0, s>>>(B->d_insts, t0, n0));
}

void finish_launch_any(fluid_pp_batch* B) {
  cudaStream_t s = B->stream;
  const Tile* t0 = tl(B, B->l0);
  const int n0 = B->l0.n, g = launch_grid(n0);
  if (B->solids) {
    FPP_LAUNCH(B, kPrGrad, k_grad_solid<<<g, kThreads, 0, s>>>(B->d_insts, t0, n0));
    FPP_LAUNCH(B, kPrReceipt, k_receipt_solid<<<g, kThreads, 0, s>>>(B->d_insts, t0, n0));
  } else {
    FPP_LAUNCH(B, kPrGrad, k_grad<<<g, kThreads, 0, s>>>(B->d_insts, t0, n0));
    FPP_LAUNCH(B, kPrReceipt, k_receipt_part<<<g, kThreads, 0, s>>>(B->d_insts, t0, n0));
  }
  FPP_LAUNCH(B, kPrReceipt, k_receipt_finish<<<B->multi.n + B->single.n, kThreads, 0, s>>>(B->d_insts,
                                                                                           il(B, B->multi)));
}

void destroy_graphs(fluid_pp_batch* B) {
  for (cudaGraphExec_t* x : {&B->x_setup, &B->x_loop, &B->x_finish})
    if (*x) {
      cudaGraphExecDestroy(*x);
      *x = nullptr;
    }
  for (cudaGraph_t* g : {&B->g_setup, &B->g_loop, &B->g_finish})
    if (*g) {
      cudaGraphDestroy(*g);
      *g = nullptr;
    }
  B->graphs_valid = false;
}

bool same_opts(const fluid_pp_solve_opts& a, const fluid_pp_solve_opts& b) {
  return a.rel_tol == b.rel_tol && a.abs_tol == b.abs_tol && a.max_iters == b.max_iters &&
         a.pre_sweeps == b.pre_sweeps && a.post_sweeps == b.post_sweeps &&
         a.true_residual_every == b.true_residual_every && a.warm_start == b.warm_start &&
         a.rel_tol_inf == b.rel_tol_inf && a.cycle == b.cycle;
}

// Captures the solve into three graphs: setup, a conditional WHILE node whose
// body is one CG iteration (V-cycle, dots, SpMV, update, true residual, loop
// condition), and the gradient subtract.  The loop ends on the device when every
// instance is done or after max_iters + 2 iterations.
template <class T>
int ensure_graphs(fluid_pp_batch* B, const fluid_pp_solve_opts& o) {
  if (B->graphs_valid && same_opts(B->graph_key, o)) return FLUID_PP_OK;
  destroy_graphs(B);
  cudaStream_t cs = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    B->err = std::string("graph stream: ") + cudaGetErrorString(e);
    return FLUID_PP_CUDA;
  }
  cudaStream_t saved = B->stream;
  const bool prof = B->profiling;
  B->stream = cs;
  B->profiling = false;
  const unsigned long long before = g_launches.load();
  const int n = int(B->h.size());
  // setup
  e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    const unsigned long long c0 = g_launches.load();
    setup_launch<T>(B, o);
    B->n_setup = g_launches.load() - c0;
    e = cudaStreamEndCapture(cs, &B->g_setup);
    if (e == cudaSuccess) e = take_launch_error(B);
  }
  // loop
  cudaGraphConditionalHandle handle{};
  if (e == cudaSuccess) e = cudaGraphCreate(&B->g_loop, 0);
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&handle, B->g_loop, 1, cudaGraphCondAssignDefault);
  cudaGraph_t body = nullptr;
  if (e == cudaSuccess) {
    cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};
    p.conditional.handle = handle;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, B->g_loop, nullptr, 0, &p);
    if (e == cudaSuccess) body = p.conditional.phGraph_out[0];
  }
  if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    const unsigned long long c0 = g_launches.load();
    iter_launch<T>(B, o);
    const unsigned cap = unsigned(o.max_iters + 2);
    k_loop_cond<<<1, 256, 0, cs>>>(B->d_insts, n, B->d_loop, cap, handle);
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess && B->launch_err == cudaSuccess) B->launch_err = le;
    B->n_body = g_launches.load() - c0 + 1;
    e = cudaStreamEndCapture(cs, &body);
    if (e == cudaSuccess) e = take_launch_error(B);
  }
  // finish
  if (e == cudaSuccess) e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    const unsigned long long c0 = g_launches.load();
    finish_launch_any(B);
    B->n_finish = g_launches.load() - c0;
    e = cudaStreamEndCapture(cs, &B->g_finish);
    if (e == cudaSuccess) e = take_launch_error(B);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&B->x_setup, B->g_setup, 0);
  if (e == cudaSuccess) e = cudaGraphInstantiate(&B->x_loop, B->g_loop, 0);
  if (e == cudaSuccess) e = cudaGraphInstantiate(&B->x_finish, B->g_finish, 0);
  // captured launches did not execute
  g_launches.store(before);
  take_launch_error(B);
  B->stream = saved;
  B->profiling = prof;
  cudaStreamDestroy(cs);
  if (e != cudaSuccess) {
    destroy_graphs(B);
    B->err = std::string("graph build: ") + cudaGetErrorString(e);
    return FLUID_PP_CUDA;
  }
  B->graph_key = o;
  B->graphs_valid = true;
  return FLUID_PP_OK;
}

}  // namespace

namespace fpp {
void set_global_error(const std::string& message) { g_err = message; }
}  // namespace fpp

// ==================================================================== batch
// Dynamic shared memory limits are a property of the kernel function, shared by
// every handle in the process: they are set once per device to the most any
// instance can ask for (the largest tile shapes over every stride pattern, the
// largest dense coarsest level, the coarse-block budget), never lowered.
template <class T>
static cudaError_t configure_kernels_t(size_t factor, size_t block, size_t down, size_t up) {
  auto set = [](const void* f, size_t bytes) {
    return bytes > 48 * 1024 ? cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes))
                             : cudaSuccess;
  };
  cudaError_t e = set((const void*)k_coarse_factor<T>, factor);
  if (e == cudaSuccess) e = set((const void*)k_coarse_block<T>, block);
  if (e == cudaSuccess) e = set((const void*)k_down<float, float, T, T>, down);
  if (e == cudaSuccess) e = set((const void*)k_down<T, T, T, T>, down);
  if (e == cudaSuccess) e = set((const void*)k_up<float, float, T, T>, up);
  if (e == cudaSuccess) e = set((const void*)k_up<T, T, T, T>, up);
  // column kernels (level 0: float32 inputs and diagonal; coarser levels: the storage type)
  auto force = [](const void* f, int bytes) {
    return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  };
  if (e == cudaSuccess) e = force((const void*)k_cdown<float, float, float, T>, cdown_smem());
  if (e == cudaSuccess) e = force((const void*)k_cdown<T, T, T, T>, cdown_smem());
  if (e == cudaSuccess) e = force((const void*)k_cup<float, float, float, T, true>, cup_smem());
  if (e == cudaSuccess) e = force((const void*)k_cup<float, float, float, T>, cup_smem());
  if (e == cudaSuccess) e = force((const void*)k_cup<T, T, T, T>, cup_smem());
  return e;
}

static std::mutex g_cfg_mutex;
static bool g_cfg_done[64] = {};

static cudaError_t configure_kernels() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_cfg_mutex);
  if (dev >= 0 && dev < 64 && g_cfg_done[dev]) return cudaSuccess;
  size_t down = 0, up = 0;
  for (int m = 0; m < 8; ++m) {
    const int sx = (m & 1) ? 2 : 1, sy = (m & 2) ? 2 : 1, sz = (m & 4) ? 2 : 1;
    down = std::max(down, size_t(down_smem_bytes(16, 4, 4, sx, sy, sz)));
    up = std::max(up, size_t(up_smem_bytes(kTX, kTY, kMaxDepth, sx, sy, sz)));
  }
  const size_t factor = size_t(kMaxCoarse) * kMaxCoarse * sizeof(double);
  const size_t block = kCoarseBlockSmem;
  e = configure_kernels_t<float>(factor, block, down, up);
  if (e == cudaSuccess) e = configure_kernels_t<__half>(factor, block, down, up);
  if (e == cudaSuccess) e = configure_kernels_t<__nv_bfloat16>(factor, block, down, up);
  if (e == cudaSuccess && dev >= 0 && dev < 64) g_cfg_done[dev] = true;
  return e;
}

static int batch_build(fluid_pp* const* handles, int count, const fluid_pp_batch_tuning& tu, fluid_pp_batch** out,
                       std::string& err) {
  if (!handles || count <= 0 || !out) {
    err = "batch needs at least one handle";
    return FLUID_PP_INVALID_ARG;
  }
  auto B = std::make_unique<fluid_pp_batch>();
  B->device = handles[0]->cfg.device;
  B->precision = handles[0]->cfg.precision;
  B->stream = handles[0]->stream;
  for (int k = 0; k < count; ++k) {
    fluid_pp* h = handles[k];
    if (!h) {
      err = "null handle in batch";
      return FLUID_PP_INVALID_ARG;
    }
    if (h->cfg.device != B->device || h->cfg.precision != B->precision) {
      err = "batched handles must share device and precision";
      return FLUID_PP_INVALID_ARG;
    }
    // A batch orders its work on one stream; a handle's own uploads, downloads
    // and release use the handle's stream, so every handle must be on that one.
    if (h->stream != B->stream) {
      err = "batched handles must share one stream (fluid_pp_set_stream)";
      return FLUID_PP_INVALID_ARG;
    }
    // a batch runs one kind of kernels: the fused ones without embedded solids,
    // the face-weighted per-pass ones with them
    if (k > 0 && (h->inst.solids != 0) != B->solids) {
      err = "batched handles must all have embedded solids or none";
      return FLUID_PP_INVALID_ARG;
    }
    B->solids = h->inst.solids != 0;
    B->h.push_back(h);
    B->maxL = std::max(B->maxL, h->plan.levels);
  }
  B->dev_dt.assign(count, std::nanf(""));
  B->dev_pscale.assign(count, std::nanf(""));
  cudaSetDevice(B->device);
  // The batch's own copies of the instance descriptors.  Fused-kernel tile
  // shapes are chosen over the whole batch: the largest shape whose tiles,
  // summed over every instance with that grid level, still reach the fill count.
  // (Results do not depend on the shape: halo cells repeat their owner's
  // arithmetic.)
  std::vector<InstDev> insts(count);
  for (int k = 0; k < count; ++k) insts[k] = B->h[k]->inst;
  for (int l = 0; l + 1 < B->maxL; ++l) {
    auto grid = [l](const InstDev& I) { return l < I.first_block && l < I.nlev - 1; };
    for (int pick = 0; pick < 5; ++pick) {
      long long total = 0;
      for (const InstDev& I : insts)
        if (grid(I)) total += shape_tiles(I.lv[l + 1].nx, I.lv[l + 1].ny, I.lv[l + 1].nz, kDownShapes[pick]);
      if (tu.box_shape >= 0 ? pick == std::min(tu.box_shape, 4) : (total >= tu.fill_tiles || pick == 4)) {
        for (InstDev& I : insts)
          if (grid(I)) {
            LevelDev& L = I.lv[l];
            L.dcx = kDownShapes[pick][0];
            L.dcy = kDownShapes[pick][1];
            L.dcz = kDownShapes[pick][2];
            L.dtiles = shape_tiles(I.lv[l + 1].nx, I.lv[l + 1].ny, I.lv[l + 1].nz, kDownShapes[pick]);
          }
        break;
      }
    }
    if (l == 0) continue;   // level 0 keeps the 32 x 8 x 8 up tiles
    for (int pick = 0; pick < 5; ++pick) {
      long long total = 0;
      for (const InstDev& I : insts)
        if (grid(I)) total += shape_tiles(I.lv[l].nx, I.lv[l].ny, I.lv[l].nz, kUpShapes[pick]);
      if (tu.box_shape >= 0 ? pick == std::min(tu.box_shape, 4) : (total >= tu.fill_tiles || pick == 4)) {
        for (InstDev& I : insts)
          if (grid(I)) {
            LevelDev& L = I.lv[l];
            L.utx = kUpShapes[pick][0];
            L.uty = kUpShapes[pick][1];
            L.utz = kUpShapes[pick][2];
            L.utiles = shape_tiles(L.nx, L.ny, L.nz, kUpShapes[pick]);
          }
        break;
      }
    }
  }
  // tile lists
  std::vector<Tile> tiles;
  std::vector<int> ilist;
  std::vector<char> col0(count, 0);   // level-0 up step is the column kernel (it forms the gamma partials)
  // restriction tiles (coarse tiles of kRX x kRY x kRZ) when `restrict_tiles`
  auto add_level = [&](List& L, auto pred, int level_of_tiles, bool restrict_tiles = false) {
    L.off = int(tiles.size());
    for (int k = 0; k < count; ++k) {
      const InstDev& I = B->h[k]->inst;
      if (!pred(I)) continue;
      const LevelDev& Lv = I.lv[level_of_tiles];
      const int nt = restrict_tiles ? rtiles_of(Lv.nx, Lv.ny, Lv.nz) : Lv.ntiles;
      for (int t = 0; t < nt; ++t) tiles.push_back(Tile{k, level_of_tiles, t, 0});
    }
    L.n = int(tiles.size()) - L.off;
  };
  // z-chunk of a column tile: the longest candidate whose tiles over the batch
  // reach the fill count (or the forced chunk); results do not depend on it
  auto pick_chunk = [&](const int* cands, int ncand, int forced, auto tiles_at) {
    if (forced > 0) return forced;
    for (int i = 0; i < ncand; ++i)
      if (tiles_at(cands[i]) >= tu.fill_tiles) return cands[i];
    return cands[ncand - 1];
  };
  add_level(B->l0, [](const InstDev&) { return true; }, 0);
  // grid-kernel levels of an instance are 0 .. first_block-1; the rest run in the coarse block
  for (int l = 0; l < B->maxL; ++l) {
    add_level(B->lvl[l], [l](const InstDev& I) { return l < I.first_block && l < I.nlev - 1; }, l);
    if (l + 1 < B->maxL)
      add_level(B->rst[l], [l](const InstDev& I) { return l < I.first_block && l < I.nlev - 1; }, l + 1, true);
    if (l >= 1) add_level(B->crs[l], [l](const InstDev& I) { return l < I.nlev; }, l);
    auto grid_level = [l](const InstDev& I) { return l < I.first_block && l < I.nlev - 1; };
    // a level whose next coarser level halves every axis runs the column
    // kernels, every other grid level the box kernels: a property of the
    // lattice alone, never of the batch
    auto column = [l, &grid_level](const InstDev& I) {
      const LevelDev& C = I.lv[l + 1];
      return grid_level(I) && C.sx == 2 && C.sy == 2 && C.sz == 2;
    };
    static const int kDownChunks[] = {16, 8, 4, 2, 1};
    static const int kUpChunks0[] = {32, 16, 8};
    static const int kUpChunks[] = {32, 16, 8, 4, 2};
    const int forced_up = tu.chunk_planes > 0 ? std::max(l == 0 ? 8 : 2, tu.chunk_planes >> l) : 0;
    const int forced_dn = tu.chunk_planes > 0 ? std::max(1, tu.chunk_planes >> (l + 1)) : 0;
    const int cdz = pick_chunk(kDownChunks, 5, forced_dn, [&](int cz) {
      long long n = 0;
      for (int k = 0; k < count; ++k)
        if (column(insts[k])) n += cdown_tiles(insts[k].lv[l + 1].nx, insts[k].lv[l + 1].ny, insts[k].lv[l + 1].nz, cz);
      return n;
    });
    const int cuz = l == 0 ? pick_chunk(kUpChunks0, 3, forced_up, [&](int cz) {
      long long n = 0;
      for (int k = 0; k < count; ++k)
        if (column(insts[k])) n += cup_tiles(insts[k].lv[0].nx, insts[k].lv[0].ny, insts[k].lv[0].nz, cz);
      return n;
    }) : pick_chunk(kUpChunks, 5, forced_up, [&](int cz) {
      long long n = 0;
      for (int k = 0; k < count; ++k)
        if (column(insts[k])) n += cup_tiles(insts[k].lv[l].nx, insts[k].lv[l].ny, insts[k].lv[l].nz, cz);
      return n;
    });
    for (int k = 0; k < count; ++k)
      if (column(insts[k])) {
        insts[k].lv[l].cdz = cdz;
        insts[k].lv[l].cuz = cuz;
      }
    B->dn[l].off = int(tiles.size());
    for (int k = 0; k < count; ++k)
      if (grid_level(insts[k]) && !column(insts[k]))
        for (int t = 0; t < insts[k].lv[l].dtiles; ++t) tiles.push_back(Tile{k, l, t, 0});
    B->dn[l].n = int(tiles.size()) - B->dn[l].off;
    B->cdn[l].off = int(tiles.size());
    for (int k = 0; k < count; ++k)
      if (column(insts[k])) {
        const LevelDev& C = insts[k].lv[l + 1];
        const int nt = cdown_tiles(C.nx, C.ny, C.nz, cdz);
        for (int t = 0; t < nt; ++t) tiles.push_back(Tile{k, l, t, 0});
      }
    B->cdn[l].n = int(tiles.size()) - B->cdn[l].off;
    B->up[l].off = int(tiles.size());
    for (int k = 0; k < count; ++k)
      if (grid_level(insts[k]) && !column(insts[k]))
        for (int t = 0; t < insts[k].lv[l].utiles; ++t) tiles.push_back(Tile{k, l, t, 0});
    B->up[l].n = int(tiles.size()) - B->up[l].off;
    B->cup[l].off = int(tiles.size());
    for (int k = 0; k < count; ++k)
      if (column(insts[k])) {
        const LevelDev& Lv = insts[k].lv[l];
        const int nt = cup_tiles(Lv.nx, Lv.ny, Lv.nz, cuz);
        for (int t = 0; t < nt; ++t) tiles.push_back(Tile{k, l, t, 0});
        if (l == 0) col0[k] = 1;
      }
    B->cup[l].n = int(tiles.size()) - B->cup[l].off;
  }
  B->dot0.off = int(tiles.size());
  for (int k = 0; k < count; ++k)
    if (!col0[k])
      for (int t = 0; t < insts[k].lv[0].ntiles; ++t) tiles.push_back(Tile{k, 0, t, 0});
  B->dot0.n = int(tiles.size()) - B->dot0.off;
  add_level(B->l0single, [](const InstDev& I) { return I.nlev == 1; }, 0);
  {
    static const int kSpmvChunks[] = {32, 16, 8};
    const int forced = tu.chunk_planes > 0 ? std::max(8, tu.chunk_planes) : 0;
    const int cqz = pick_chunk(kSpmvChunks, 3, forced, [&](int cz) {
      long long n = 0;
      for (int k = 0; k < count; ++k) n += cspmv_tiles(insts[k].lv[0].nx, insts[k].lv[0].ny, insts[k].lv[0].nz, cz);
      return n;
    });
    B->cq.off = int(tiles.size());
    for (int k = 0; k < count; ++k) {
      insts[k].lv[0].cqz = cqz;
      const LevelDev& L0 = insts[k].lv[0];
      const int nt = cspmv_tiles(L0.nx, L0.ny, L0.nz, cqz);
      for (int t = 0; t < nt; ++t) tiles.push_back(Tile{k, 0, t, 0});
    }
    B->cq.n = int(tiles.size()) - B->cq.off;
  }
  B->bake.off = int(tiles.size());
  for (int k = 0; k < count; ++k) {
    const InstDev& I = B->h[k]->inst;
    for (int l = 0; l < I.nlev; ++l)
      for (int t = 0; t < I.lv[l].ntiles; ++t) tiles.push_back(Tile{k, l, t, 0});
  }
  B->bake.n = int(tiles.size()) - B->bake.off;
  B->multi.off = int(ilist.size());
  for (int k = 0; k < count; ++k)
    if (B->h[k]->inst.nlev > 1) ilist.push_back(k);
  B->multi.n = int(ilist.size()) - B->multi.off;
  B->single.off = int(ilist.size());
  for (int k = 0; k < count; ++k)
    if (B->h[k]->inst.nlev == 1) ilist.push_back(k);
  B->single.n = int(ilist.size()) - B->single.off;
  for (int l = 0; l < B->maxL; ++l) {
    B->fcb[l].off = int(ilist.size());
    for (int k = 0; k < count; ++k) {
      const InstDev& I = B->h[k]->inst;
      if (I.nlev > 1 && l < I.first_block) ilist.push_back(k);
    }
    B->fcb[l].n = int(ilist.size()) - B->fcb[l].off;
  }
  int mmax = 0;
  for (int k = 0; k < count; ++k) {
    mmax = std::max(mmax, B->h[k]->inst.coarse_m);
    const InstDev& I = insts[k];
    if (I.nlev > 1) B->smem_block = std::max(B->smem_block, size_t(I.block_smem));
    for (int l = 0; l < I.first_block && l + 1 < I.nlev; ++l) {
      const LevelDev &L = I.lv[l], &C = I.lv[l + 1];
      B->smem_down = std::max(B->smem_down, size_t(down_smem_bytes(L.dcx, L.dcy, L.dcz, C.sx, C.sy, C.sz)));
      B->smem_up = std::max(B->smem_up, size_t(up_smem_bytes(L.utx, L.uty, L.utz, C.sx, C.sy, C.sz)));
    }
  }
  B->smem_factor = size_t(mmax) * mmax * sizeof(double);

  cudaError_t e = dev_alloc(reinterpret_cast<void**>(&B->d_ctrl), sizeof(Ctrl) * count);
  if (e == cudaSuccess) e = cudaMemset(B->d_ctrl, 0, sizeof(Ctrl) * count);
  for (int k = 0; k < count; ++k) insts[k].ctrl = B->d_ctrl + k;
  if (e == cudaSuccess) e = dev_alloc(reinterpret_cast<void**>(&B->d_insts), sizeof(InstDev) * count);
  if (e == cudaSuccess) e = cudaMemcpy(B->d_insts, insts.data(), sizeof(InstDev) * count, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = dev_alloc(reinterpret_cast<void**>(&B->d_tiles), sizeof(Tile) * std::max<size_t>(1, tiles.size()));
  if (e == cudaSuccess && !tiles.empty())
    e = cudaMemcpy(B->d_tiles, tiles.data(), sizeof(Tile) * tiles.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = dev_alloc(reinterpret_cast<void**>(&B->d_ilist), sizeof(int) * std::max<size_t>(1, ilist.size()));
  if (e == cudaSuccess && !ilist.empty())
    e = cudaMemcpy(B->d_ilist, ilist.data(), sizeof(int) * ilist.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = host_alloc(reinterpret_cast<void**>(&B->h_ctrl), sizeof(Ctrl) * count);
  if (e == cudaSuccess) e = dev_alloc(reinterpret_cast<void**>(&B->d_loop), sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(B->d_loop, 0, sizeof(unsigned));
  if (e == cudaSuccess) e = host_alloc(reinterpret_cast<void**>(&B->h_loop), sizeof(unsigned));
  if (e == cudaSuccess) e = configure_kernels();
  if (e != cudaSuccess) {
    err = std::string("batch setup: ") + cudaGetErrorString(e);
    fluid_pp_batch_destroy(B.release());
    return e == cudaErrorMemoryAllocation ? FLUID_PP_OOM : FLUID_PP_CUDA;
  }
  const int np = std::min(tu.parts, count);
  if (np > 1) {
    // handles to parts by cells, largest first onto the lightest part; each
    // part keeps the batch's order and needs 1/np of the tiles to fill the GPU
    std::vector<int> order(count);
    for (int k = 0; k < count; ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
      return B->h[a]->plan_cells() > B->h[b]->plan_cells();
    });
    std::vector<long long> load(np, 0);
    std::vector<int> part_of(count, 0);
    for (int k : order) {
      const int j = int(std::min_element(load.begin(), load.end()) - load.begin());
      part_of[k] = j;
      load[j] += B->h[k]->plan_cells();
    }
    fluid_pp_batch_tuning sub = tu;
    sub.parts = 1;
    sub.fill_tiles = std::max(1, tu.fill_tiles / np);
    B->part_idx.assign(np, {});
    for (int k = 0; k < count; ++k) B->part_idx[part_of[k]].push_back(k);
    e = cudaEventCreateWithFlags(&B->part_start, cudaEventDisableTiming);
    for (int j = 0; j < np && e == cudaSuccess; ++j) {
      std::vector<fluid_pp*> hs;
      for (int k : B->part_idx[j]) hs.push_back(B->h[k]);
      fluid_pp_batch* P = nullptr;
      std::string perr;
      const int rc = batch_build(hs.data(), int(hs.size()), sub, &P, perr);
      if (rc != FLUID_PP_OK) {
        err = "batch part: " + perr;
        fluid_pp_batch_destroy(B.release());
        return rc;
      }
      B->parts.push_back(P);
      cudaStream_t st = nullptr;
      cudaEvent_t done = nullptr;
      e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&done, cudaEventDisableTiming);
      B->part_streams.push_back(st);
      B->part_done.push_back(done);
      P->stream = st;
    }
    if (e != cudaSuccess) {
      err = std::string("batch parts: ") + cudaGetErrorString(e);
      fluid_pp_batch_destroy(B.release());
      return FLUID_PP_CUDA;
    }
  }
  *out = B.release();
  return FLUID_PP_OK;
}

static void fill_receipt(const fluid_pp* h, const Ctrl& c, fluid_pp_receipt* r) {
  std::memset(r, 0, sizeof(*r));
  r->status = c.status;
  r->iterations = c.iter;
  r->liquid_cells = c.liquid;
  r->levels = h->plan.levels;
  const double hh = h->cfg.h;
  r->b_norm = std::sqrt(std::max(0.0, c.bb));
  r->rel_residual = c.bb > 0 ? std::sqrt(std::max(0.0, c.rr) / c.bb) : 0.0;
  r->true_rel_residual = c.bb > 0 ? std::sqrt(std::max(0.0, c.rr_true) / c.bb) : 0.0;
  r->max_div_after = c.red[0] / hh;
  r->l2_div_after = std::sqrt(std::max(0.0, c.red[1]) * hh);
  r->max_div_before = c.red[2] / hh;
  r->l2_div_before = std::sqrt(std::max(0.0, c.red[3]) * hh);
}

static fluid_pp_solve_opts default_opts() {
  fluid_pp_solve_opts o{};
  o.rel_tol = 1e-6;
  o.abs_tol = 0.0;
  o.max_iters = 200;
  o.pre_sweeps = 1;
  o.post_sweeps = 1;
  o.true_residual_every = 4;   // the recursive float32 residual drifts on smooth right-hand sides
  o.warm_start = 0;
  return o;
}

// Per-instance dt and pressure scale into the batch's descriptor table.
static void push_dts(fluid_pp_batch* B, const float* dts) {
  const int n = int(B->h.size());
  for (int k = 0; k < n; ++k) {
    fluid_pp* h = B->h[k];
    const float dt = dts ? dts[k] : h->last_dt;
    h->last_dt = dt;
    h->inst.dt = dt;
    h->inst.pscale = h->cfg.rho * h->cfg.h / dt;
    // only changed values cross: a copy from pageable memory may wait for the
    // stream, which would stall a caller that keeps two batches in flight
    if (!(B->dev_dt[k] == h->inst.dt)) {
      cudaMemcpyAsync(reinterpret_cast<char*>(B->d_insts + k) + offsetof(InstDev, dt), &h->inst.dt, sizeof(float),
                      cudaMemcpyHostToDevice, B->stream);
      B->dev_dt[k] = h->inst.dt;
    }
    if (!(B->dev_pscale[k] == h->inst.pscale)) {
      cudaMemcpyAsync(reinterpret_cast<char*>(B->d_insts + k) + offsetof(InstDev, pscale), &h->inst.pscale,
                      sizeof(float), cudaMemcpyHostToDevice, B->stream);
      B->dev_pscale[k] = h->inst.pscale;
    }
  }
}

template <class T>
static int batch_project_t(fluid_pp_batch* B, const float* dts, const fluid_pp_solve_opts& o, bool sync_receipts,
                           fluid_pp_receipt* receipts) {
  const int n = int(B->h.size());
  push_dts(B, dts);
  bool graphed = false;
  if (!B->profiling && B->use_graphs) {
    const int rc = ensure_graphs<T>(B, o);
    if (rc != FLUID_PP_OK) return rc;
    cudaError_t e = cudaGraphLaunch(B->x_setup, B->stream);
    if (e == cudaSuccess) e = cudaGraphLaunch(B->x_loop, B->stream);
    if (e == cudaSuccess) e = cudaGraphLaunch(B->x_finish, B->stream);
    if (e != cudaSuccess) {
      B->err = std::string("graph launch: ") + cudaGetErrorString(e);
      return FLUID_PP_CUDA;
    }
    g_launches.fetch_add(B->n_setup + B->n_finish, std::memory_order_relaxed);
    graphed = true;
  } else {
    // direct launches (per-stage events need individual launches); the host
    // polls the done flags every few iterations
    setup_launch<T>(B, o);
    const int check = 4;
    int it = 0;
    const int cap = o.max_iters + 2;
    while (it < cap) {
      const int burst = std::min(check, cap - it);
      for (int b = 0; b < burst; ++b) iter_launch<T>(B, o);
      it += burst;
      cudaMemcpyAsync(B->h_ctrl, B->d_ctrl, sizeof(Ctrl) * n, cudaMemcpyDeviceToHost, B->stream);
      cudaError_t e = take_launch_error(B);
      if (e == cudaSuccess) e = cudaStreamSynchronize(B->stream);
      if (e != cudaSuccess) {
        B->err = std::string("solve: ") + cudaGetErrorString(e);
        return FLUID_PP_CUDA;
      }
      bool all = true;
      for (int k = 0; k < n; ++k) all &= B->h_ctrl[k].done != 0;
      if (all) break;
    }
    finish_launch_any(B);
    const cudaError_t e = take_launch_error(B);
    if (e != cudaSuccess) {
      B->err = std::string("launch: ") + cudaGetErrorString(e);
      return FLUID_PP_CUDA;
    }
  }
  cudaMemcpyAsync(B->h_ctrl, B->d_ctrl, sizeof(Ctrl) * n, cudaMemcpyDeviceToHost, B->stream);
  if (graphed) cudaMemcpyAsync(B->h_loop, B->d_loop, sizeof(unsigned), cudaMemcpyDeviceToHost, B->stream);
  B->pending_graph_count = graphed;
  if (sync_receipts) {
    cudaError_t e = cudaStreamSynchronize(B->stream);
    if (e != cudaSuccess) {
      B->err = std::string("project: ") + cudaGetErrorString(e);
      return FLUID_PP_CUDA;
    }
    if (graphed) g_launches.fetch_add((unsigned long long)(*B->h_loop) * B->n_body, std::memory_order_relaxed);
    B->pending_graph_count = false;
    int worst = FLUID_PP_OK;
    for (int k = 0; k < n; ++k) {
      if (receipts) fill_receipt(B->h[k], B->h_ctrl[k], receipts + k);
      B->h[k]->has_pressure = true;
      if (B->h_ctrl[k].status != FLUID_PP_OK && worst == FLUID_PP_OK) worst = B->h_ctrl[k].status;
    }
    prof_collect(B);
    return worst;
  }
  return FLUID_PP_OK;
}

static int batch_project(fluid_pp_batch* B, const float* dts, const fluid_pp_solve_opts* opts, bool sync,
                         fluid_pp_receipt* receipts);

// ------------------------------------------------------------ CM11a LCP solve
// Grid passes of the projected multigrid (one instance: the handle's own batch,
// every level below the coarsest a grid level).
template <class T>
void restrict_pass(fluid_pp_batch* B, int l) {
  const List& Lr = B->rst[l];
  if (l == 0)
    FPP_LAUNCH(B, kPrRestrict0, k_residual_restrict<float, float, T, T><<<launch_grid(Lr.n), kThreads, 0, B->stream>>>(
                                    B->d_insts, tl(B, Lr), Lr.n, l));
  else
    FPP_LAUNCH(B, kPrRestrictC, k_residual_restrict<T, T, T, T><<<launch_grid(Lr.n), kThreads, 0, B->stream>>>(
                                    B->d_insts, tl(B, Lr), Lr.n, l));
}

template <class T>
void prolong_pass(fluid_pp_batch* B, int l) {
  const List& Ls = B->lvl[l];
  const int g = launch_grid(Ls.n);
  if (l == 0)
    FPP_LAUNCH(B, kPrProlong0, k_prolong<float, T><<<g, kThreads, 0, B->stream>>>(B->d_insts, tl(B, Ls), Ls.n, l));
  else
    FPP_LAUNCH(B, kPrProlongC, k_prolong<T, T><<<g, kThreads, 0, B->stream>>>(B->d_insts, tl(B, Ls), Ls.n, l));
}

// The bound of level l + 1 from level l (mode: k_lcp_bound_down).
template <class T>
void bound_pass(fluid_pp_batch* B, int l, int mode) {
  const List& Lc = B->crs[l + 1];
  if (l == 0)
    FPP_LAUNCH(B, kPrRestrict0, k_lcp_bound_down<float><<<launch_grid(Lc.n), kThreads, 0, B->stream>>>(
                                    B->d_insts, tl(B, Lc), Lc.n, l, mode));
  else
    FPP_LAUNCH(B, kPrRestrictC, k_lcp_bound_down<T><<<launch_grid(Lc.n), kThreads, 0, B->stream>>>(
                                    B->d_insts, tl(B, Lc), Lc.n, l, mode));
}

template <class T>
void lcp_coarse_pass(fluid_pp_batch* B, const fluid_pp_lcp_opts& o) {
  if (B->multi.n)
    FPP_LAUNCH(B, kPrCoarse, k_lcp_coarse<T><<<B->multi.n, kMaxCoarse, 0, B->stream>>>(
                                 B->d_insts, il(B, B->multi), o.coarse_sweeps, o.coarse_tol));
  if (B->single.n)   // a one-level hierarchy: the coarsest is level 0 (float vectors)
    FPP_LAUNCH(B, kPrCoarse, k_lcp_coarse<float><<<B->single.n, kMaxCoarse, 0, B->stream>>>(
                                 B->d_insts, il(B, B->single), o.coarse_sweeps, o.coarse_tol));
}

// vCycle (mg.ts:524-538) from level l with the projected smoother; level l
// keeps its z, each coarser level starts its correction at zero with the bound
// of mgDownsampleSubtract on the first constraint_levels levels.
template <class T>
void lcp_vcycle_from(fluid_pp_batch* B, int l, const fluid_pp_lcp_opts& o) {
  const int last = B->maxL - 1;
  if (l == last) {
    lcp_coarse_pass<T>(B, o);
    return;
  }
  for (int sw = 0; sw < o.pre_sweeps; ++sw) {
    smooth_pass<T>(B, l, 0, 0, 1);
    smooth_pass<T>(B, l, 1, 0, 1);
  }
  restrict_pass<T>(B, l);
  if (l + 1 < last) smooth_pass<T>(B, l + 1, 2, 1);   // the coarse correction starts at zero
  bound_pass<T>(B, l, l < o.constraint_levels ? 0 : 2);
  lcp_vcycle_from<T>(B, l + 1, o);
  prolong_pass<T>(B, l);
  for (int sw = 0; sw < o.post_sweeps; ++sw) {
    smooth_pass<T>(B, l, 1, 0, 1);
    smooth_pass<T>(B, l, 0, 0, 1);
  }
}

// fullCycle (mg.ts:539-563): the correction e of p with bound p_min - p; the
// residual and the bound restricted down every level, the coarsest solved,
// then per level from the coarsest up the prolongated e starts a V-cycle there.
template <class T>
void lcp_fcycle(fluid_pp_batch* B, const fluid_pp_lcp_opts& o) {
  const Tile* t0 = tl(B, B->l0);
  const int n0 = B->l0.n, g0 = launch_grid(n0);
  FPP_LAUNCH(B, kPrInit, k_lcp_fc_begin<<<g0, kThreads, 0, B->stream>>>(B->d_insts, t0, n0));
  const int last = B->maxL - 1;
  for (int l = 0; l < last; ++l) {
    smooth_pass<T>(B, l, 2, 1);   // e = 0 on level l
    restrict_pass<T>(B, l);
    bound_pass<T>(B, l, l < o.constraint_levels ? 1 : 2);
  }
  lcp_coarse_pass<T>(B, o);
  for (int l = last - 1; l >= 0; --l) {
    prolong_pass<T>(B, l);
    lcp_vcycle_from<T>(B, l, o);
  }
  FPP_LAUNCH(B, kPrInit, k_lcp_fc_end<<<g0, kThreads, 0, B->stream>>>(B->d_insts, t0, n0));
}

template <class T>
static int lcp_project_t(fluid_pp* pp, float dt, const fluid_pp_lcp_opts& o, fluid_pp_receipt* receipt) {
  fluid_pp_batch* B = pp->self;
  push_dts(B, &dt);
  fluid_pp_solve_opts so = default_opts();
  so.warm_start = o.warm_start;
  setup_launch<T>(B, so);
  const Tile* t0 = tl(B, B->l0);
  const int n0 = B->l0.n, g0 = launch_grid(n0);
  FPP_LAUNCH(B, kPrInit, k_lcp_init<<<g0, kThreads, 0, B->stream>>>(B->d_insts, t0, n0, o.warm_start));
  for (int c = 0; c < o.full_cycles; ++c) lcp_fcycle<T>(B, o);
  for (int c = 0; c < o.v_cycles; ++c) lcp_vcycle_from<T>(B, 0, o);
  FPP_LAUNCH(B, kPrTrue, k_lcp_measure<<<g0, kThreads, 0, B->stream>>>(B->d_insts, t0, n0,
                                                                      o.full_cycles + o.v_cycles));
  finish_launch_any(B);
  cudaMemcpyAsync(B->h_ctrl, B->d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, B->stream);
  cudaError_t e = take_launch_error(B);
  if (e == cudaSuccess) e = cudaStreamSynchronize(B->stream);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, std::string("lcp: ") + cudaGetErrorString(e));
  if (receipt) fill_receipt(pp, B->h_ctrl[0], receipt);
  pp->has_pressure = true;
  prof_collect(B);
  return B->h_ctrl[0].status;
}

// Receipts of a solve that ran in the batch's parts (waits for the batch's stream).
static int parts_receipts(fluid_pp_batch* B, fluid_pp_receipt* receipts) {
  const cudaError_t e = cudaStreamSynchronize(B->stream);
  if (e != cudaSuccess) {
    B->err = std::string("project: ") + cudaGetErrorString(e);
    return FLUID_PP_CUDA;
  }
  int worst = FLUID_PP_OK;
  for (size_t j = 0; j < B->parts.size(); ++j) {
    fluid_pp_batch* P = B->parts[j];
    if (P->pending_graph_count) {
      g_launches.fetch_add((unsigned long long)(*P->h_loop) * P->n_body, std::memory_order_relaxed);
      P->pending_graph_count = false;
    }
    for (size_t i = 0; i < B->part_idx[j].size(); ++i) {
      const int k = B->part_idx[j][i];
      if (receipts) fill_receipt(B->h[k], P->h_ctrl[i], receipts + k);
      B->h[k]->has_pressure = true;
      if (P->h_ctrl[i].status != FLUID_PP_OK && worst == FLUID_PP_OK) worst = P->h_ctrl[i].status;
    }
  }
  B->parts_pending = false;
  return worst;
}

// Every part's graph-mode solve, started together after this batch's stream
// reaches the launch point and joined back to it.
static int parts_project(fluid_pp_batch* B, const float* dts, const fluid_pp_solve_opts* opts) {
  cudaError_t e = cudaEventRecord(B->part_start, B->stream);
  std::vector<float> dp;
  for (size_t j = 0; j < B->parts.size() && e == cudaSuccess; ++j) {
    fluid_pp_batch* P = B->parts[j];
    e = cudaStreamWaitEvent(P->stream, B->part_start, 0);
    if (e != cudaSuccess) break;
    dp.clear();
    if (dts)
      for (int k : B->part_idx[j]) dp.push_back(dts[k]);
    const int rc = batch_project(P, dts ? dp.data() : nullptr, opts, false, nullptr);
    if (rc != FLUID_PP_OK) {
      B->err = P->err;
      return rc;
    }
    e = cudaEventRecord(B->part_done[j], P->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(B->stream, B->part_done[j], 0);
  }
  if (e != cudaSuccess) {
    B->err = std::string("parts: ") + cudaGetErrorString(e);
    return FLUID_PP_CUDA;
  }
  B->parts_pending = true;
  return FLUID_PP_OK;
}

static int batch_project(fluid_pp_batch* B, const float* dts, const fluid_pp_solve_opts* opts, bool sync,
                         fluid_pp_receipt* receipts) {
  const fluid_pp_solve_opts o = opts ? *opts : default_opts();
  if (!(o.rel_tol >= 0) || !(o.abs_tol >= 0) || o.max_iters < 1 || o.pre_sweeps < 0 || o.post_sweeps < 0 ||
      o.cycle < 0 || o.cycle > 1) {
    B->err = "invalid solve options";
    return FLUID_PP_INVALID_ARG;
  }
  for (fluid_pp* h : B->h)
    if (!h->has_state) {
      B->err = "state not uploaded";
      return FLUID_PP_INVALID_ARG;
    }
  cudaSetDevice(B->device);
  B->parts_pending = false;
  if (!B->parts.empty() && B->use_graphs && !B->profiling) {
    const int rc = parts_project(B, dts, &o);
    if (rc != FLUID_PP_OK || !sync) return rc;
    return parts_receipts(B, receipts);
  }
  switch (B->precision) {
    case FLUID_PP_FP16: return batch_project_t<__half>(B, dts, o, sync, receipts);
    case FLUID_PP_BF16: return batch_project_t<__nv_bfloat16>(B, dts, o, sync, receipts);
    default: return batch_project_t<float>(B, dts, o, sync, receipts);
  }
}

// ==================================================================== C ABI
extern "C" {

int fluid_pp_plan_hierarchy(int nx, int ny, int nz, int* level_count, int* level_dims, int* coarsest_cells,
                            int* semi_coarsened, int* extended) {
  HierarchyPlan p = plan_hierarchy(nx, ny, nz);
  if (level_count) *level_count = p.levels;
  if (coarsest_cells) *coarsest_cells = p.coarsest_haloed;
  if (semi_coarsened) *semi_coarsened = p.semi ? 1 : 0;
  if (extended) *extended = p.extended ? 1 : 0;
  if (!p.ok) {
    g_err = p.rejection ? p.rejection : "rejected";
    return FLUID_PP_INVALID_ARG;
  }
  if (level_dims)
    for (int l = 0; l < p.levels; ++l)
      for (int a = 0; a < 3; ++a) level_dims[3 * l + a] = p.dims[l][a];
  return FLUID_PP_OK;
}

// Device bytes of one handle's arena (every level, the resident state, the CG
// vectors, reduction partials, the dense coarsest inverse, the control block).
static size_t arena_size(const fluid_pp_config& cfg, const HierarchyPlan& plan) {
  const size_t sT = storage_bytes(cfg.precision);
  const int nx = cfg.nx, ny = cfg.ny, nz = cfg.nz;
  const long long N = (long long)nx * ny * nz;
  size_t bytes = 0;
  auto acc = [&](size_t b) { bytes = align_up(bytes + b, 256); };
  for (int l = 0; l < plan.levels; ++l) {
    const long long n = (long long)plan.dims[l][0] * plan.dims[l][1] * plan.dims[l][2];
    acc(n);                        // label
    acc(4 * n);                    // phi
    acc(4 * n);                    // diag
    acc(sT * n);                   // diagT
    acc((l == 0 ? 4 : sT) * n);    // z
    acc((l == 0 ? 4 : sT) * n);    // rhs / r
    acc((l == 0 ? 4 : sT) * n);    // res (z type)
  }
  const long long nu = (long long)(nx + 1) * ny * nz, nv = (long long)nx * (ny + 1) * nz,
                  nw = (long long)nx * ny * (nz + 1);
  acc(4 * N);                      // vof
  acc(4 * nu);
  acc(4 * nv);
  acc(4 * nw);
  for (int k = 0; k < 7; ++k) acc(4 * N);   // b x xlo d d2 q p_si
  const long long ncoarse =
      (long long)plan.dims[plan.levels - 1][0] * plan.dims[plan.levels - 1][1] * plan.dims[plan.levels - 1][2];
  acc(sizeof(double) * kSlots * tiles_of(nx, ny, nz, kMaxDepth));
  acc(sizeof(double) * ncoarse * ncoarse);
  acc(sizeof(Ctrl));
  // slack: the column kernels copy 2-byte level arrays in aligned 4-byte words,
  // which may reach up to 6 bytes past an array's last element
  acc(256);
  return bytes;
}

int fluid_pp_create(const fluid_pp_config* cfg, fluid_pp** out) {
  g_err.clear();
  if (!cfg || !out) return FLUID_PP_INVALID_ARG;
  *out = nullptr;
  HierarchyPlan plan = plan_hierarchy(cfg->nx, cfg->ny, cfg->nz);
  if (!plan.ok) {
    g_err = plan.rejection ? plan.rejection : "no hierarchy";
    return FLUID_PP_INVALID_ARG;
  }
  if (!(cfg->h > 0) || !std::isfinite(cfg->h) || !(cfg->rho > 0) || !std::isfinite(cfg->rho)) {
    g_err = "CM11a grid spacing must be positive and finite";
    return FLUID_PP_INVALID_ARG;
  }
  if (cfg->precision < 0 || cfg->precision > 2) {
    g_err = "unknown precision";
    return FLUID_PP_INVALID_ARG;
  }
  const long long ncoarse =
      (long long)plan.dims[plan.levels - 1][0] * plan.dims[plan.levels - 1][1] * plan.dims[plan.levels - 1][2];
  if (ncoarse > kMaxCoarse) {
    g_err = "coarsest level exceeds the dense solve limit";
    return FLUID_PP_INVALID_ARG;
  }
  if (cudaSetDevice(cfg->device) != cudaSuccess) {
    g_err = "cannot select CUDA device";
    return FLUID_PP_CUDA;
  }
  auto h = std::make_unique<fluid_pp>();
  h->cfg = *cfg;
  h->plan = plan;
  const size_t sT = storage_bytes(cfg->precision);
  const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz;
  const long long N = (long long)nx * ny * nz;
  if (N > (1LL << 30)) {
    g_err = "lattice exceeds 2^30 cells";
    return FLUID_PP_INVALID_ARG;
  }
  // Cells per thread along z: keep at least ~2 waves of fully occupied SMs
  // (148 x 2048 threads) in flight; small levels get one cell per thread.
  auto depth_of = [](long long n) { return n >= 4LL * 600000 ? 4 : n >= 2LL * 600000 ? 2 : 1; };
  const int nt0 = tiles_of(nx, ny, nz, kMaxDepth);   // level 0: 32 x 8 x 8 tiles
  const size_t bytes = arena_size(*cfg, plan);
  const long long nu = (long long)(nx + 1) * ny * nz, nv = (long long)nx * (ny + 1) * nz,
                  nw = (long long)nx * ny * (nz + 1);
  cudaError_t e = dev_alloc(reinterpret_cast<void**>(&h->arena), bytes);
  if (e != cudaSuccess) {
    g_err = std::string("arena allocation: ") + cudaGetErrorString(e);
    return FLUID_PP_OOM;
  }
  h->arena_bytes = bytes;
  cudaMemset(h->arena, 0, bytes);
  Arena a{h->arena, 0, bytes};
  InstDev& I = h->inst;
  std::memset(&I, 0, sizeof(I));
  I.nlev = plan.levels;
  I.nx = nx;
  I.ny = ny;
  I.nz = nz;
  I.open_top = cfg->open_top ? 1 : 0;
  I.h = cfg->h;
  I.rho = cfg->rho;
  I.dt = 1.0f;
  I.ntiles0 = nt0;
  I.coarse_m = int(ncoarse);
  float wmax_prev = 1.0f;
  for (int l = 0; l < plan.levels; ++l) {
    LevelDev& L = I.lv[l];
    L.nx = plan.dims[l][0];
    L.ny = plan.dims[l][1];
    L.nz = plan.dims[l][2];
    L.sx = plan.stride[l][0];
    L.sy = plan.stride[l][1];
    L.sz = plan.stride[l][2];
    L.n = (long long)L.nx * L.ny * L.nz;
    L.depth = l == 0 ? kMaxDepth : depth_of(L.n);
    L.ntiles = tiles_of(L.nx, L.ny, L.nz, L.depth);
    // spacing ratio h_l / h_0 per axis (webgpu-uniform-pressure-multigrid.ts:588-589)
    const double rx = double(nx) / L.nx, ry = double(ny) / L.ny, rz = double(nz) / L.nz;
    const double wx = 1.0 / (rx * rx), wy = 1.0 / (ry * ry), wz = 1.0 / (rz * rz);
    const double wmax = std::max(wx, std::max(wy, wz));
    L.wmax = float(wmax);
    L.wx = float(wx / wmax);
    L.wy = float(wy / wmax);
    L.wz = float(wz / wmax);
    L.ext_phi = float(0.5 * ry);
    if (l > 0) I.lv[l - 1].to_coarse = wmax_prev / float(wmax);
    wmax_prev = float(wmax);
    const long long n = L.n;
    L.label = static_cast<uint8_t*>(a.take(n));
    L.phi = static_cast<float*>(a.take(4 * n));
    L.diag = static_cast<float*>(a.take(4 * n));
    L.diagT = a.take(sT * n);
    L.z = a.take((l == 0 ? 4 : sT) * n);
    L.rhs = a.take((l == 0 ? 4 : sT) * n);
    L.res = a.take((l == 0 ? 4 : sT) * n);
  }
  I.lv[plan.levels - 1].to_coarse = 1.0f;
  // Fused-kernel tile shapes per grid level for a solve on its own: the largest
  // shape that still gives every SM a tile (a batch re-chooses them over all
  // its instances, batch_build).
  for (int l = 0; l + 1 < plan.levels; ++l) {
    LevelDev& L = I.lv[l];
    const LevelDev& Cl = I.lv[l + 1];
    for (const auto& t : kDownShapes) {
      L.dcx = t[0];
      L.dcy = t[1];
      L.dcz = t[2];
      L.dtiles = shape_tiles(Cl.nx, Cl.ny, Cl.nz, t);
      if (L.dtiles >= kFillTiles) break;
    }
    for (const auto& t : kUpShapes) {
      L.utx = t[0];
      L.uty = t[1];
      L.utz = t[2];
      L.utiles = shape_tiles(L.nx, L.ny, L.nz, t);
      if (l == 0 || L.utiles >= kFillTiles) break;
    }
  }
  // The single-CTA coarse block takes every level from the first one (>= 1) that
  // fits kCoarseBlockCells and whose tail of levels fits the shared-memory budget.
  I.first_block = plan.levels;
  I.block_smem = 0;
  if (plan.levels > 1) {
    for (int l = 1; l < plan.levels; ++l) {
      long long bytes = 0;
      for (int j = l; j < plan.levels; ++j) bytes += block_level_bytes(I.lv[j].n);
      if (I.lv[l].n <= kCoarseBlockCells && bytes <= kCoarseBlockSmem) {
        I.first_block = l;
        I.block_smem = int(bytes);
        break;
      }
    }
  }
  I.vof = static_cast<float*>(a.take(4 * N));
  I.u = static_cast<float*>(a.take(4 * nu));
  I.v = static_cast<float*>(a.take(4 * nv));
  I.w = static_cast<float*>(a.take(4 * nw));
  I.b = static_cast<float*>(a.take(4 * N));
  I.x = static_cast<float*>(a.take(4 * N));
  I.xlo = static_cast<float*>(a.take(4 * N));
  I.d = static_cast<float*>(a.take(4 * N));
  I.d2 = static_cast<float*>(a.take(4 * N));
  I.q = static_cast<float*>(a.take(4 * N));
  I.p_si = static_cast<float*>(a.take(4 * N));
  I.partial = static_cast<double*>(a.take(sizeof(double) * kSlots * nt0));
  I.coarse_inv = static_cast<double*>(a.take(sizeof(double) * ncoarse * ncoarse));
  I.ctrl = static_cast<Ctrl*>(a.take(sizeof(Ctrl)));
  fluid_pp* raw = h.get();
  std::string err;
  fluid_pp_batch_tuning tu;
  fluid_pp_batch_tuning_default(&tu);
  int rc = batch_build(&raw, 1, tu, &h->self, err);
  if (rc != FLUID_PP_OK) {
    g_err = err;
    dev_release(h->arena, h->stream);
    return rc;
  }
  *out = h.release();
  return FLUID_PP_OK;
}

int fluid_pp_required_bytes(const fluid_pp_config* cfg, unsigned long long* bytes) {
  if (!cfg || !bytes) return FLUID_PP_INVALID_ARG;
  HierarchyPlan plan = plan_hierarchy(cfg->nx, cfg->ny, cfg->nz);
  if (!plan.ok) {
    g_err = plan.rejection ? plan.rejection : "no hierarchy";
    return FLUID_PP_INVALID_ARG;
  }
  // the arena plus the handle's own batch tables (tile lists, descriptors)
  const long long N = (long long)cfg->nx * cfg->ny * cfg->nz;
  *bytes = arena_size(*cfg, plan) + sizeof(InstDev) + sizeof(Ctrl) + size_t(N / 64 + 4096) * sizeof(Tile);
  return FLUID_PP_OK;
}

void fluid_pp_destroy(fluid_pp* pp) {
  if (!pp) return;
  cudaSetDevice(pp->cfg.device);
  if (pp->self) fluid_pp_batch_destroy(pp->self);
  dev_release(pp->solid_mem, pp->stream);
  dev_release(pp->ext_mem, pp->stream);
  dev_release(pp->tr_mem, pp->stream);
  dev_release(pp->arena, pp->stream);
  delete pp;
}

int fluid_pp_set_stream(fluid_pp* pp, void* stream) {
  if (!pp) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(pp->cfg.device);
  const cudaStream_t next = static_cast<cudaStream_t>(stream);
  const cudaError_t e = order_streams(pp->stream, next);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, cudaGetErrorString(e));
  pp->stream = next;
  if (pp->self) pp->self->stream = pp->stream;
  return FLUID_PP_OK;
}

static int upload(fluid_pp* pp, const float* vof, const float* u, const float* v, const float* w,
                  cudaMemcpyKind kind) {
  if (!pp || !vof || !u || !v || !w) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(pp->cfg.device);
  const long long nx = pp->cfg.nx, ny = pp->cfg.ny, nz = pp->cfg.nz;
  const InstDev& I = pp->inst;
  cudaError_t e = cudaMemcpyAsync((void*)I.vof, vof, 4 * nx * ny * nz, kind, pp->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(I.u, u, 4 * (nx + 1) * ny * nz, kind, pp->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(I.v, v, 4 * nx * (ny + 1) * nz, kind, pp->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(I.w, w, 4 * nx * ny * (nz + 1), kind, pp->stream);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, std::string("upload: ") + cudaGetErrorString(e));
  pp->has_state = true;
  return FLUID_PP_OK;
}

int fluid_pp_upload_state(fluid_pp* pp, const float* vof, const float* u, const float* v, const float* w) {
  return upload(pp, vof, u, v, w, cudaMemcpyHostToDevice);
}

int fluid_pp_upload_state_device(fluid_pp* pp, const float* vof, const float* u, const float* v, const float* w) {
  return upload(pp, vof, u, v, w, cudaMemcpyDeviceToDevice);
}

int fluid_pp_project(fluid_pp* pp, float dt, const fluid_pp_solve_opts* opts, fluid_pp_receipt* receipt) {
  if (!pp) return FLUID_PP_INVALID_ARG;
  if (!(dt > 0) || !std::isfinite(dt)) return pp->set_error(FLUID_PP_INVALID_ARG, "dt must be positive and finite");
  const int rc = batch_project(pp->self, &dt, opts, true, receipt);
  if (rc != FLUID_PP_OK) pp->err = pp->self->err;
  return rc;
}

int fluid_pp_project_async(fluid_pp* pp, float dt, const fluid_pp_solve_opts* opts) {
  if (!pp) return FLUID_PP_INVALID_ARG;
  if (!(dt > 0) || !std::isfinite(dt)) return pp->set_error(FLUID_PP_INVALID_ARG, "dt must be positive and finite");
  const int rc = batch_project(pp->self, &dt, opts, false, nullptr);
  if (rc != FLUID_PP_OK) pp->err = pp->self->err;
  return rc;
}

int fluid_pp_receipt_read(fluid_pp* pp, fluid_pp_receipt* receipt) {
  if (!pp || !receipt) return FLUID_PP_INVALID_ARG;
  fluid_pp_batch* B = pp->self;
  cudaError_t e = cudaStreamSynchronize(B->stream);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, cudaGetErrorString(e));
  if (B->pending_graph_count) {
    g_launches.fetch_add((unsigned long long)(*B->h_loop) * B->n_body, std::memory_order_relaxed);
    B->pending_graph_count = false;
  }
  fill_receipt(pp, B->h_ctrl[0], receipt);
  pp->has_pressure = true;
  return receipt->status;
}

int fluid_pp_download(fluid_pp* pp, float* p, float* u, float* v, float* w) {
  const int rc = fluid_pp_download_async(pp, p, u, v, w);
  return rc == FLUID_PP_OK ? fluid_pp_synchronize(pp) : rc;
}

int fluid_pp_download_async(fluid_pp* pp, float* p, float* u, float* v, float* w) {
  if (!pp) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(pp->cfg.device);
  const long long nx = pp->cfg.nx, ny = pp->cfg.ny, nz = pp->cfg.nz;
  const InstDev& I = pp->inst;
  cudaError_t e = cudaSuccess;
  if (p) e = cudaMemcpyAsync(p, I.p_si, 4 * nx * ny * nz, cudaMemcpyDeviceToHost, pp->stream);
  if (u && e == cudaSuccess) e = cudaMemcpyAsync(u, I.u, 4 * (nx + 1) * ny * nz, cudaMemcpyDeviceToHost, pp->stream);
  if (v && e == cudaSuccess) e = cudaMemcpyAsync(v, I.v, 4 * nx * (ny + 1) * nz, cudaMemcpyDeviceToHost, pp->stream);
  if (w && e == cudaSuccess) e = cudaMemcpyAsync(w, I.w, 4 * nx * ny * (nz + 1), cudaMemcpyDeviceToHost, pp->stream);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, std::string("download: ") + cudaGetErrorString(e));
  return FLUID_PP_OK;
}

int fluid_pp_synchronize(fluid_pp* pp) {
  if (!pp) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(pp->cfg.device);
  const cudaError_t e = cudaStreamSynchronize(pp->stream);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, std::string("synchronize: ") + cudaGetErrorString(e));
  return FLUID_PP_OK;
}

int fluid_pp_device_arrays(fluid_pp* pp, float** p, float** u, float** v, float** w, float** vof) {
  if (!pp) return FLUID_PP_INVALID_ARG;
  if (p) *p = pp->inst.p_si;
  if (u) *u = pp->inst.u;
  if (v) *v = pp->inst.v;
  if (w) *w = pp->inst.w;
  if (vof) *vof = const_cast<float*>(pp->inst.vof);
  return FLUID_PP_OK;
}

const char* fluid_pp_last_error(const fluid_pp* pp) { return pp ? pp->err.c_str() : g_err.c_str(); }

// ------------------------------------------------------------ parity hooks
int fluid_pp_prepare(fluid_pp* pp, float dt) {
  if (!pp || !pp->has_state) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(pp->cfg.device);
  fluid_pp_batch* B = pp->self;
  pp->inst.dt = dt;
  pp->inst.pscale = pp->cfg.rho * pp->cfg.h / dt;
  pp->last_dt = dt;
  cudaMemcpyAsync(reinterpret_cast<char*>(B->d_insts) + offsetof(InstDev, dt), &pp->inst.dt, sizeof(float),
                  cudaMemcpyHostToDevice, B->stream);
  B->dev_dt[0] = pp->inst.dt;
  const fluid_pp_solve_opts o = default_opts();
  switch (B->precision) {
    case FLUID_PP_FP16: setup_launch<__half>(B, o); break;
    case FLUID_PP_BF16: setup_launch<__nv_bfloat16>(B, o); break;
    default: setup_launch<float>(B, o);
  }
  cudaError_t e = cudaStreamSynchronize(B->stream);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, std::string("prepare: ") + cudaGetErrorString(e));
  return FLUID_PP_OK;
}

int fluid_pp_level_dims(fluid_pp* pp, int level, int* dims3) {
  if (!pp || level < 0 || level >= pp->plan.levels || !dims3) return FLUID_PP_INVALID_ARG;
  for (int a = 0; a < 3; ++a) dims3[a] = pp->plan.dims[level][a];
  return FLUID_PP_OK;
}

int fluid_pp_get_level(fluid_pp* pp, int level, unsigned char* label, float* phi, float* diag) {
  if (!pp || level < 0 || level >= pp->plan.levels) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(pp->cfg.device);
  const LevelDev& L = pp->inst.lv[level];
  cudaError_t e = cudaSuccess;
  if (label) e = cudaMemcpy(label, L.label, L.n, cudaMemcpyDeviceToHost);
  if (phi && e == cudaSuccess) e = cudaMemcpy(phi, L.phi, 4 * L.n, cudaMemcpyDeviceToHost);
  if (diag && e == cudaSuccess) e = cudaMemcpy(diag, L.diag, 4 * L.n, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, cudaGetErrorString(e));
  return FLUID_PP_OK;
}

int fluid_pp_get_rhs(fluid_pp* pp, float* b) {
  if (!pp || !b) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(pp->cfg.device);
  cudaError_t e = cudaMemcpy(b, pp->inst.b, 4 * pp->inst.lv[0].n, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, cudaGetErrorString(e));
  return FLUID_PP_OK;
}

int fluid_pp_get_pressure_cells(fluid_pp* pp, float* x) {
  if (!pp || !x) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(pp->cfg.device);
  const long long n = pp->inst.lv[0].n;
  std::vector<float> lo(n);
  cudaError_t e = cudaMemcpy(x, pp->inst.x, 4 * n, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(lo.data(), pp->inst.xlo, 4 * n, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, cudaGetErrorString(e));
  for (long long i = 0; i < n; ++i) x[i] = float(double(x[i]) + double(lo[i]));
  return FLUID_PP_OK;
}

int fluid_pp_upload_solids(fluid_pp* pp, const float* open, const float* fx, const float* fy, const float* fz,
                           const float* usx, const float* usy, const float* usz) {
  if (!pp || !open || !fx || !fy || !fz) return FLUID_PP_INVALID_ARG;
  if ((usx != nullptr) != (usy != nullptr) || (usx != nullptr) != (usz != nullptr))
    return pp->set_error(FLUID_PP_INVALID_ARG, "solid velocities: all three face arrays or none");
  cudaSetDevice(pp->cfg.device);
  InstDev& I = pp->inst;
  const long long N = I.lv[0].n, nx = I.nx, ny = I.ny, nz = I.nz;
  const long long nf[3] = {(nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1)};
  long long floats = N + 2 * (nf[0] + nf[1] + nf[2]);
  for (int l = 0; l < I.nlev; ++l) floats += 4 * I.lv[l].n;   // face fractions and the LCP bound
  cudaStream_t s = pp->stream;
  if (!pp->solid_mem) {
    cudaError_t e = dev_alloc(reinterpret_cast<void**>(&pp->solid_mem), size_t(floats) * 4);
    if (e != cudaSuccess) return pp->set_error(FLUID_PP_OOM, std::string("solids: ") + cudaGetErrorString(e));
  }
  float* p = reinterpret_cast<float*>(pp->solid_mem);
  I.open = p;
  p += N;
  for (int a = 0; a < 3; ++a) {
    I.fv[a] = p;
    p += nf[a];
  }
  for (int a = 0; a < 3; ++a) {
    I.us[a] = p;
    p += nf[a];
  }
  for (int l = 0; l < I.nlev; ++l) {
    I.lv[l].ff = p;
    p += 3 * I.lv[l].n;
    I.lv[l].pmin = p;
    p += I.lv[l].n;
  }
  const float* src[3] = {fx, fy, fz};
  const float* vel[3] = {usx, usy, usz};
  cudaError_t e = cudaMemcpyAsync(const_cast<float*>(I.open), open, 4 * N, cudaMemcpyHostToDevice, s);
  for (int a = 0; a < 3 && e == cudaSuccess; ++a) {
    e = cudaMemcpyAsync(const_cast<float*>(I.fv[a]), src[a], 4 * nf[a], cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = vel[a] ? cudaMemcpyAsync(const_cast<float*>(I.us[a]), vel[a], 4 * nf[a], cudaMemcpyHostToDevice, s)
                 : cudaMemsetAsync(const_cast<float*>(I.us[a]), 0, 4 * nf[a], s);
  }
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, std::string("solids: ") + cudaGetErrorString(e));
  // every level below the coarsest runs the face-weighted grid kernels; the
  // coarse block only applies the dense coarsest inverse
  I.solids = 1;
  if (I.nlev > 1) {
    I.first_block = I.nlev - 1;
    I.block_smem = int(block_level_bytes(I.lv[I.nlev - 1].n));
  }
  if (pp->self) {
    fluid_pp_batch_destroy(pp->self);
    pp->self = nullptr;
  }
  fluid_pp* raw = pp;
  std::string err;
  fluid_pp_batch_tuning tu;
  fluid_pp_batch_tuning_default(&tu);
  int rc = batch_build(&raw, 1, tu, &pp->self, err);
  if (rc != FLUID_PP_OK) return pp->set_error(rc, err);
  fluid_pp_batch* B = pp->self;
  k_solid_faces<<<launch_grid(int(std::min<long long>((N + kThreads - 1) / kThreads, kMaxGrid))), kThreads, 0, s>>>(
      B->d_insts);
  for (int l = 1; l < I.nlev; ++l)
    k_coarsen_faces<<<launch_grid(int(std::min<long long>((I.lv[l].n + kThreads - 1) / kThreads, kMaxGrid))),
                      kThreads, 0, s>>>(B->d_insts, l);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, std::string("solids: ") + cudaGetErrorString(e));
  return FLUID_PP_OK;
}

int fluid_pp_extrapolate_velocity(fluid_pp* pp, long long* filled_faces) {
  if (!pp) return FLUID_PP_INVALID_ARG;
  if (!pp->has_state) return pp->set_error(FLUID_PP_INVALID_ARG, "state not uploaded");
  cudaSetDevice(pp->cfg.device);
  const InstDev& I = pp->inst;
  const int nx = I.nx, ny = I.ny, nz = I.nz;
  const long long n = (long long)nx * ny * nz;
  // the hierarchy: ceil-halved lattices until the shortest axis is one cell
  std::vector<std::array<int, 3>> dims;
  std::array<int, 3> d{nx, ny, nz};
  while (std::min({d[0], d[1], d[2]}) > 1) {
    d = {(d[0] + 1) / 2, (d[1] + 1) / 2, (d[2] + 1) / 2};
    dims.push_back(d);
  }
  long long cells = 4 * n;
  for (const auto& l : dims) cells += 2LL * l[0] * l[1] * l[2];
  // float4 states, the counters, two band mark arrays and the band list
  const size_t bytes = size_t(cells) * sizeof(float4) + 16 + 2 * size_t(n) + 4 * size_t(n) + 16;
  cudaStream_t s = pp->stream;
  if (!pp->ext_mem) {
    const cudaError_t e = dev_alloc(reinterpret_cast<void**>(&pp->ext_mem), bytes);
    if (e != cudaSuccess) return pp->set_error(FLUID_PP_OOM, std::string("extrapolation: ") + cudaGetErrorString(e));
  }
  float4* p = reinterpret_cast<float4*>(pp->ext_mem);
  ExtDev E{};
  E.nx = nx;
  E.ny = ny;
  E.nz = nz;
  E.h = I.h;   // cubic cells of edge h (the band is 2 h)
  E.open_top = I.open_top;
  E.solids = I.solids;
  E.vof = I.vof;
  E.open = I.open;
  for (int c = 0; c < 3; ++c) E.fv[c] = I.fv[c];
  E.vel[0] = I.u;
  E.vel[1] = I.v;
  E.vel[2] = I.w;
  for (int k = 0; k < 2; ++k) {
    E.val[k] = p;
    p += n;
    E.dist[k] = p;
    p += n;
  }
  std::vector<float4*> down, up;
  for (const auto& l : dims) {
    const long long m = 1LL * l[0] * l[1] * l[2];
    down.push_back(p);
    p += m;
    up.push_back(p);
    p += m;
  }
  E.count = reinterpret_cast<unsigned*>(p);
  E.mark[0] = reinterpret_cast<uint8_t*>(p + 1);
  E.mark[1] = E.mark[0] + n;
  E.band = reinterpret_cast<unsigned*>((reinterpret_cast<uintptr_t>(E.mark[1] + n) + 15) & ~uintptr_t(15));
  auto grid = [](long long cnt) { return int(std::max(1LL, std::min<long long>((cnt + kThreads - 1) / kThreads, kMaxGrid))); };
  cudaMemsetAsync(E.count, 0, 16, s);
  if (E.solids) k_ext_seed<true><<<grid(n), kThreads, 0, s>>>(E);
  else k_ext_seed<false><<<grid(n), kThreads, 0, s>>>(E);
  k_ext_dilate<<<grid(n), kThreads, 0, s>>>(E, 0, E.mark[0], E.mark[1]);
  k_ext_dilate<<<grid(n), kThreads, 0, s>>>(E, 1, E.mark[1], E.mark[0]);
  k_ext_dilate<<<grid(n), kThreads, 0, s>>>(E, 2, E.mark[0], E.mark[1]);
  k_ext_band_list<<<grid(n), kThreads, 0, s>>>(E, E.mark[1]);
  const int passes = std::min(std::max({nx, ny, nz}), 16);
  for (int k = 0; k < passes; ++k) {
    const int src = k & 1;
    k_ext_reset<<<1, 1, 0, s>>>(E.count, 1 - src);
    if (E.solids) k_ext_update<true><<<grid(n), kThreads, 0, s>>>(E, src);
    else k_ext_update<false><<<grid(n), kThreads, 0, s>>>(E, src);
  }
  const int last = passes & 1;
  const float4* result = E.val[last];
  if (!dims.empty()) {
    const float4* finer = E.val[last];
    std::array<int, 3> fd{nx, ny, nz};
    for (size_t l = 0; l < dims.size(); ++l) {
      ExtLevel L{dims[l][0], dims[l][1], dims[l][2], finer, fd[0], fd[1], fd[2], nullptr, down[l]};
      k_ext_restrict<<<grid(1LL * dims[l][0] * dims[l][1] * dims[l][2]), kThreads, 0, s>>>(L);
      finer = down[l];
      fd = dims[l];
    }
    const float4* coarser = down.back();
    std::array<int, 3> cd = dims.back();
    float4* finest = E.val[1 - last];   // free after the band solve
    for (int l = int(dims.size()) - 2; l >= -1; --l) {
      const std::array<int, 3> td = l >= 0 ? dims[l] : std::array<int, 3>{nx, ny, nz};
      const float4* keep = l >= 0 ? down[l] : E.val[last];
      float4* out = l >= 0 ? up[l] : finest;
      ExtLevel L{td[0], td[1], td[2], coarser, cd[0], cd[1], cd[2], keep, out};
      k_ext_prolong<<<grid(1LL * td[0] * td[1] * td[2]), kThreads, 0, s>>>(L);
      coarser = out;
      cd = td;
    }
    result = finest;
  }
  k_ext_pack<<<grid(n), kThreads, 0, s>>>(E, result, E.count + 2);
  unsigned got = 0;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&got, E.count + 2, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, std::string("extrapolation: ") + cudaGetErrorString(e));
  if (filled_faces) *filled_faces = got;
  return FLUID_PP_OK;
}

// Density transport scratch, allocated on first use: five fields of n floats
// (gamma, the second gamma, two density fields, the sharpening delta), 3 n
// fixed-point deposits, 3 n floats of backward trace offsets, the three
// velocity transport shells and the mass partials.  Gamma starts at 1
// everywhere.
struct TrMem {
  float *gam, *gam2, *r1, *r2, *delta, *trace;
  float* sh[3];
  int* dep;
  double* part;   // 3 kTrMassGrid partials, 6 receipt values, the sharpening list counter
};

long long tr_floats(const fluid_pp* pp) {
  const int nx = pp->cfg.nx, ny = pp->cfg.ny, nz = pp->cfg.nz;
  long long f = 11LL * nx * ny * nz;
  for (int c = 0; c < 3; ++c) f += tr_shell_size(nx, ny, nz, c);
  return f;
}

TrMem tr_layout(fluid_pp* pp) {
  const long long n = pp->plan_cells();
  TrMem M;
  float* f = reinterpret_cast<float*>(pp->tr_mem);
  M.gam = f;
  M.gam2 = f + n;
  M.r1 = f + 2 * n;
  M.r2 = f + 3 * n;
  M.delta = f + 4 * n;
  M.dep = reinterpret_cast<int*>(f + 5 * n);
  M.trace = f + 8 * n;
  float* q = f + 11 * n;
  for (int c = 0; c < 3; ++c) {
    M.sh[c] = q;
    q += tr_shell_size(pp->cfg.nx, pp->cfg.ny, pp->cfg.nz, c);
  }
  const size_t off = (size_t(tr_floats(pp)) * 4 + 15) & ~size_t(15);
  M.part = reinterpret_cast<double*>(pp->tr_mem + off);
  return M;
}

int ensure_transport(fluid_pp* pp) {
  if (pp->tr_mem) return FLUID_PP_OK;
  const long long n = pp->plan_cells();
  const size_t bytes = ((size_t(tr_floats(pp)) * 4 + 15) & ~size_t(15)) + sizeof(double) * (3 * kTrMassGrid + 8);
  const cudaError_t e = dev_alloc(reinterpret_cast<void**>(&pp->tr_mem), bytes);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_OOM, std::string("density transport: ") + cudaGetErrorString(e));
  const TrMem M = tr_layout(pp);
  k_tr_fill<<<int(std::min<long long>((n + kThreads - 1) / kThreads, kMaxGrid)), kThreads, 0, pp->stream>>>(M.gam, n, 1.0f);
  return FLUID_PP_OK;
}

void fluid_pp_transport_opts_default(fluid_pp_transport_opts* o) {
  if (!o) return;
  o->gamma_diffusion_iterations = 1;
  o->sharpening = 1;
  o->sharpening_mass_return = 1;
  o->sharpening_strength = 1.0f;
  o->sharpening_distance = 2.1f;
}

int fluid_pp_transport_density(fluid_pp* pp, float dt, const fluid_pp_transport_opts* opts,
                               fluid_pp_transport_receipt* receipt) {
  if (!pp) return FLUID_PP_INVALID_ARG;
  if (!(dt > 0.0f) || !std::isfinite(dt)) return pp->set_error(FLUID_PP_INVALID_ARG, "dt must be positive and finite");
  if (!pp->has_state) return pp->set_error(FLUID_PP_INVALID_ARG, "state not uploaded");
  if (pp->inst.solids)
    return pp->set_error(FLUID_PP_UNSUPPORTED, "density transport: handles with embedded solids are not supported");
  fluid_pp_transport_opts o;
  fluid_pp_transport_opts_default(&o);
  if (opts) o = *opts;
  if (!std::isfinite(o.sharpening_strength) || !std::isfinite(o.sharpening_distance))
    return pp->set_error(FLUID_PP_INVALID_ARG, "sharpening strength and distance must be finite");
  // the reference's clamps (webgpu-uniform-reference.ts:374-377)
  const int iters = std::min(7, std::max(0, o.gamma_diffusion_iterations));
  const float strength = std::min(2.0f, std::max(0.25f, o.sharpening_strength));
  const float dist = std::min(3.1f, std::max(0.1f, o.sharpening_distance));
  cudaSetDevice(pp->cfg.device);
  int rc = ensure_transport(pp);
  if (rc != FLUID_PP_OK) return rc;
  const InstDev& I = pp->inst;
  const long long n = pp->plan_cells();
  const TrMem M = tr_layout(pp);
  TrDev T{I.nx, I.ny, I.nz, I.open_top, I.h, dt, I.u, I.v, I.w, {M.sh[0], M.sh[1], M.sh[2]}};
  cudaStream_t s = pp->stream;
  const int g = int(std::min<long long>((n + kThreads - 1) / kThreads, kMaxGrid));
  k_tr_shells<<<g, kThreads, 0, s>>>(T, M.sh[0], M.sh[1], M.sh[2]);
  float* vof = const_cast<float*>(I.vof);
  k_tr_mass_part<<<kTrMassGrid, 256, 0, s>>>(vof, n, M.part);
  k_tr_mass_fold<<<1, 256, 0, s>>>(M.part, kTrMassGrid, M.part + 3 * kTrMassGrid);
  cudaMemsetAsync(M.dep, 0, sizeof(int) * 3 * size_t(n), s);
  int* beta = M.dep;
  k_tr_trace_beta<<<g, kThreads, 0, s>>>(T, M.gam, M.gam2, beta, M.trace);
  k_tr_deficit<<<g, kThreads, 0, s>>>(T, vof, M.gam, beta, M.dep + n, M.dep + 2 * n);
  k_tr_gather<<<g, kThreads, 0, s>>>(T, vof, M.gam2, beta, M.dep + n, M.dep + 2 * n, M.trace, M.r1, M.gam);
  float *cr = M.r1, *cg = M.gam, *nr = M.r2, *ng = M.gam2;
  for (int it = 0; it < iters; ++it)
    for (int a = 0; a < 3; ++a) {
      k_tr_diffuse<<<g, kThreads, 0, s>>>(T, a, cr, cg, nr, ng);
      std::swap(cr, nr);
      std::swap(cg, ng);
    }
  if (cg != M.gam) cudaMemcpyAsync(M.gam, cg, sizeof(float) * size_t(n), cudaMemcpyDeviceToDevice, s);
  if (o.sharpening) {
    if (o.sharpening_mass_return) {
      cudaMemsetAsync(M.dep, 0, sizeof(int) * size_t(n), s);
      // the trace offsets are spent: their buffer holds the list of cells losing density
      unsigned* lost = reinterpret_cast<unsigned*>(M.trace);
      unsigned* nlost = reinterpret_cast<unsigned*>(M.part + 3 * kTrMassGrid + 6);
      cudaMemsetAsync(nlost, 0, sizeof(unsigned), s);
      k_tr_sharpen<<<g, kThreads, 0, s>>>(T, cr, strength, nr, M.delta, lost, nlost);
      k_tr_sharpen_scatter<<<g, kThreads, 0, s>>>(T, M.delta, nr, dist, lost, nlost, M.dep);
      k_tr_sharpen_resolve<<<g, kThreads, 0, s>>>(T, nr, M.dep, vof);
    } else {
      k_tr_sharpen<<<g, kThreads, 0, s>>>(T, cr, strength, vof, M.delta, nullptr, nullptr);
    }
  } else {
    cudaMemcpyAsync(vof, cr, sizeof(float) * size_t(n), cudaMemcpyDeviceToDevice, s);
  }
  k_tr_mass_part<<<kTrMassGrid, 256, 0, s>>>(vof, n, M.part);
  k_tr_mass_fold<<<1, 256, 0, s>>>(M.part, kTrMassGrid, M.part + 3 * kTrMassGrid + 3);
  double out[6] = {};
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, M.part + 3 * kTrMassGrid, sizeof(out), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, std::string("density transport: ") + cudaGetErrorString(e));
  pp->has_pressure = false;
  if (receipt) {
    receipt->mass_before = out[0];
    receipt->mass_after = out[3];
    receipt->rho_min = float(out[4]);
    receipt->rho_max = float(out[5]);
  }
  return FLUID_PP_OK;
}

int fluid_pp_get_vof(fluid_pp* pp, float* vof) {
  if (!pp || !vof) return FLUID_PP_INVALID_ARG;
  if (!pp->has_state) return pp->set_error(FLUID_PP_INVALID_ARG, "state not uploaded");
  cudaSetDevice(pp->cfg.device);
  cudaError_t e = cudaMemcpyAsync(vof, pp->inst.vof, sizeof(float) * size_t(pp->plan_cells()), cudaMemcpyDeviceToHost,
                                  pp->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(pp->stream);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, std::string("get vof: ") + cudaGetErrorString(e));
  return FLUID_PP_OK;
}

int fluid_pp_set_gamma(fluid_pp* pp, const float* gamma) {
  if (!pp) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(pp->cfg.device);
  int rc = ensure_transport(pp);
  if (rc != FLUID_PP_OK) return rc;
  const long long n = pp->plan_cells();
  const TrMem M = tr_layout(pp);
  cudaError_t e = cudaSuccess;
  if (gamma) {
    e = cudaMemcpyAsync(M.gam, gamma, sizeof(float) * size_t(n), cudaMemcpyHostToDevice, pp->stream);
  } else {
    k_tr_fill<<<int(std::min<long long>((n + kThreads - 1) / kThreads, kMaxGrid)), kThreads, 0, pp->stream>>>(M.gam, n, 1.0f);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(pp->stream);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, std::string("set gamma: ") + cudaGetErrorString(e));
  return FLUID_PP_OK;
}

int fluid_pp_get_gamma(fluid_pp* pp, float* gamma) {
  if (!pp || !gamma) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(pp->cfg.device);
  int rc = ensure_transport(pp);
  if (rc != FLUID_PP_OK) return rc;
  const TrMem M = tr_layout(pp);
  cudaError_t e = cudaMemcpyAsync(gamma, M.gam, sizeof(float) * size_t(pp->plan_cells()), cudaMemcpyDeviceToHost, pp->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(pp->stream);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, std::string("get gamma: ") + cudaGetErrorString(e));
  return FLUID_PP_OK;
}

void fluid_pp_lcp_opts_default(fluid_pp_lcp_opts* o) {
  if (!o) return;
  o->full_cycles = 3;
  o->v_cycles = 4;
  o->pre_sweeps = 1;
  o->post_sweeps = 1;
  o->constraint_levels = 3;
  o->coarse_sweeps = 4096;
  o->coarse_tol = 1e-6;
  o->warm_start = 0;
}

int fluid_pp_project_lcp(fluid_pp* pp, float dt, const fluid_pp_lcp_opts* opts, fluid_pp_receipt* receipt) {
  if (!pp) return FLUID_PP_INVALID_ARG;
  if (!(dt > 0) || !std::isfinite(dt)) return pp->set_error(FLUID_PP_INVALID_ARG, "dt must be positive and finite");
  if (!pp->has_state) return pp->set_error(FLUID_PP_INVALID_ARG, "state not uploaded");
  if (!pp->inst.solids)
    return pp->set_error(FLUID_PP_INVALID_ARG,
                         "the LCP solve bounds solid cells: upload embedded solids first (fluid_pp_upload_solids)");
  fluid_pp_lcp_opts o;
  fluid_pp_lcp_opts_default(&o);
  if (opts) o = *opts;
  if (o.full_cycles < 0 || o.v_cycles < 0 || o.full_cycles + o.v_cycles < 1 || o.pre_sweeps < 0 ||
      o.post_sweeps < 0 || o.constraint_levels < 0 || o.coarse_sweeps < 1 || !(o.coarse_tol >= 0))
    return pp->set_error(FLUID_PP_INVALID_ARG, "invalid LCP options");
  cudaSetDevice(pp->cfg.device);
  switch (pp->cfg.precision) {
    case FLUID_PP_FP16: return lcp_project_t<__half>(pp, dt, o, receipt);
    case FLUID_PP_BF16: return lcp_project_t<__nv_bfloat16>(pp, dt, o, receipt);
    default: return lcp_project_t<float>(pp, dt, o, receipt);
  }
}

int fluid_pp_get_level_faces(fluid_pp* pp, int level, float* ff) {
  if (!pp || !ff || level < 0 || level >= pp->inst.nlev) return FLUID_PP_INVALID_ARG;
  if (!pp->inst.solids) return pp->set_error(FLUID_PP_INVALID_ARG, "no embedded solids uploaded");
  cudaSetDevice(pp->cfg.device);
  const LevelDev& L = pp->inst.lv[level];
  cudaError_t e = cudaMemcpy(ff, L.ff, 12 * size_t(L.n), cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? FLUID_PP_OK : pp->set_error(FLUID_PP_CUDA, cudaGetErrorString(e));
}

int fluid_pp_apply_operator(fluid_pp* pp, const float* p, float* out) {
  if (!pp || !p || !out) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(pp->cfg.device);
  fluid_pp_batch* B = pp->self;
  const long long N = pp->inst.lv[0].n;
  cudaMemcpyAsync(pp->inst.d, p, 4 * N, cudaMemcpyHostToDevice, B->stream);
  k_hook_ctrl<<<1, 1, 0, B->stream>>>(B->d_insts, 1.0);
  k_spmv<<<launch_grid(B->l0.n), kThreads, 0, B->stream>>>(B->d_insts, tl(B, B->l0), B->l0.n);
  cudaMemcpyAsync(out, pp->inst.q, 4 * N, cudaMemcpyDeviceToHost, B->stream);
  cudaError_t e = cudaStreamSynchronize(B->stream);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, cudaGetErrorString(e));
  return FLUID_PP_OK;
}

// The preconditioner input scale the solve would use for residual r: one over
// the rms of its nonzero entries (keeps half-precision levels in range).
static double hook_sigma(const float* r, long long N) {
  double ss = 0;
  long long cnt = 0;
  for (long long i = 0; i < N; ++i) {
    ss += double(r[i]) * r[i];
    cnt += r[i] != 0.0f;
  }
  const double per = cnt ? ss / double(cnt) : 0.0;
  return per > 1e-300 ? 1.0 / std::sqrt(per) : 1.0;
}

int fluid_pp_apply_vcycle(fluid_pp* pp, const float* r, float* z, int pre, int post) {
  if (!pp || !r || !z || pre < 0 || post < 0) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(pp->cfg.device);
  fluid_pp_batch* B = pp->self;
  const long long N = pp->inst.lv[0].n;
  cudaMemcpyAsync(pp->inst.lv[0].rhs, r, 4 * N, cudaMemcpyHostToDevice, B->stream);
  k_hook_ctrl<<<1, 1, 0, B->stream>>>(B->d_insts, hook_sigma(r, N));
  const bool fused = pre == 1 && post == 1 && !B->solids;
  switch (B->precision) {
    case FLUID_PP_FP16: fused ? vcycle_fused<__half>(B, 0) : vcycle_launch<__half>(B, pre, post); break;
    case FLUID_PP_BF16: fused ? vcycle_fused<__nv_bfloat16>(B, 0) : vcycle_launch<__nv_bfloat16>(B, pre, post); break;
    default: fused ? vcycle_fused<float>(B, 0) : vcycle_launch<float>(B, pre, post);
  }
  cudaMemcpyAsync(z, pp->inst.lv[0].z, 4 * N, cudaMemcpyDeviceToHost, B->stream);
  cudaError_t e = cudaStreamSynchronize(B->stream);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, cudaGetErrorString(e));
  return FLUID_PP_OK;
}

int fluid_pp_apply_fcycle(fluid_pp* pp, const float* r, float* z, int pre, int post, int* first_block) {
  if (!pp || !r || !z || pre < 0 || post < 0) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(pp->cfg.device);
  fluid_pp_batch* B = pp->self;
  const long long N = pp->inst.lv[0].n;
  if (first_block) *first_block = pp->inst.nlev > 1 ? pp->inst.first_block : 0;
  cudaMemcpyAsync(pp->inst.lv[0].rhs, r, 4 * N, cudaMemcpyHostToDevice, B->stream);
  k_hook_ctrl<<<1, 1, 0, B->stream>>>(B->d_insts, hook_sigma(r, N));
  switch (B->precision) {
    case FLUID_PP_FP16: fcycle_launch<__half>(B, pre, post); break;
    case FLUID_PP_BF16: fcycle_launch<__nv_bfloat16>(B, pre, post); break;
    default: fcycle_launch<float>(B, pre, post);
  }
  cudaMemcpyAsync(z, pp->inst.lv[0].z, 4 * N, cudaMemcpyDeviceToHost, B->stream);
  cudaError_t e = cudaStreamSynchronize(B->stream);
  if (e != cudaSuccess) return pp->set_error(FLUID_PP_CUDA, cudaGetErrorString(e));
  return FLUID_PP_OK;
}

// ------------------------------------------------------------------ batch API
void fluid_pp_batch_tuning_default(fluid_pp_batch_tuning* tuning) {
  if (!tuning) return;
  tuning->fill_tiles = kFillTiles;
  tuning->chunk_planes = 0;
  tuning->box_shape = -1;
  tuning->parts = 1;
}

int fluid_pp_batch_create(fluid_pp* const* handles, int count, fluid_pp_batch** out) {
  return fluid_pp_batch_create_tuned(handles, count, nullptr, out);
}

int fluid_pp_batch_create_tuned(fluid_pp* const* handles, int count, const fluid_pp_batch_tuning* tuning,
                                fluid_pp_batch** out) {
  fluid_pp_batch_tuning tu;
  fluid_pp_batch_tuning_default(&tu);
  if (tuning) {
    if (tuning->fill_tiles < 1 || tuning->chunk_planes < 0 || tuning->chunk_planes > 256 ||
        tuning->chunk_planes % 8 != 0 || tuning->box_shape < -1 || tuning->box_shape > 4 || tuning->parts < 1 ||
        tuning->parts > 16) {
      g_err = "batch tuning: fill_tiles >= 1, chunk_planes a multiple of 8 in 0..256, box_shape in -1..4, "
              "parts in 1..16";
      return FLUID_PP_INVALID_ARG;
    }
    tu = *tuning;
  }
  std::string err;
  const int rc = batch_build(handles, count, tu, out, err);
  g_err = err;
  return rc;
}

void fluid_pp_batch_destroy(fluid_pp_batch* B) {
  if (!B) return;
  cudaSetDevice(B->device);
  for (fluid_pp_batch* P : B->parts) fluid_pp_batch_destroy(P);
  for (cudaStream_t st : B->part_streams)
    if (st) cudaStreamDestroy(st);
  for (cudaEvent_t ev : B->part_done)
    if (ev) cudaEventDestroy(ev);
  if (B->part_start) cudaEventDestroy(B->part_start);
  destroy_graphs(B);
  dev_release(B->d_insts, B->stream);
  dev_release(B->d_ctrl, B->stream);
  dev_release(B->d_tiles, B->stream);
  dev_release(B->d_ilist, B->stream);
  host_release(B->h_ctrl, B->stream);
  dev_release(B->d_loop, B->stream);
  host_release(B->h_loop, B->stream);
  for (cudaEvent_t e : B->ev_pool) cudaEventDestroy(e);
  delete B;
}

unsigned long long fluid_pp_kernel_launches(void) { return g_launches.load(); }

int fluid_pp_batch_set_graphs(fluid_pp_batch* B, int on) {
  if (!B) return FLUID_PP_INVALID_ARG;
  B->use_graphs = on != 0;
  return FLUID_PP_OK;
}

int fluid_pp_batch_set_profiling(fluid_pp_batch* B, int on) {
  if (!B) return FLUID_PP_INVALID_ARG;
  B->profiling = on != 0;
  return FLUID_PP_OK;
}

int fluid_pp_batch_profile_read(fluid_pp_batch* B, double* ms, long long* launches, int reset) {
  if (!B) return FLUID_PP_INVALID_ARG;
  prof_collect(B);
  for (int s = 0; s < FLUID_PP_PROFILE_STAGES; ++s) {
    if (ms) ms[s] = B->prof_ms[s];
    if (launches) launches[s] = B->prof_count[s];
    if (reset) {
      B->prof_ms[s] = 0;
      B->prof_count[s] = 0;
    }
  }
  return FLUID_PP_OK;
}

int fluid_pp_set_profiling(fluid_pp* pp, int on) {
  return pp ? fluid_pp_batch_set_profiling(pp->self, on) : FLUID_PP_INVALID_ARG;
}

int fluid_pp_profile_read(fluid_pp* pp, double* ms, long long* launches, int reset) {
  return pp ? fluid_pp_batch_profile_read(pp->self, ms, launches, reset) : FLUID_PP_INVALID_ARG;
}

// Every handle of a batch must still be on the batch's stream: fluid_pp_set_stream
// on a member after fluid_pp_batch_create would let that handle's uploads,
// downloads and release race the batched solve.
static int batch_streams_ok(fluid_pp_batch* B) {
  for (fluid_pp* h : B->h)
    if (h->stream != B->stream) {
      B->err = "a batched handle's stream no longer matches the batch's stream (fluid_pp_set_stream after "
               "fluid_pp_batch_create)";
      g_err = B->err;
      return FLUID_PP_INVALID_ARG;
    }
  return FLUID_PP_OK;
}

int fluid_pp_batch_project(fluid_pp_batch* B, const float* dts, const fluid_pp_solve_opts* opts,
                           fluid_pp_receipt* receipts) {
  if (!B) return FLUID_PP_INVALID_ARG;
  if (batch_streams_ok(B) != FLUID_PP_OK) return FLUID_PP_INVALID_ARG;
  if (dts)
    for (size_t k = 0; k < B->h.size(); ++k)
      if (!(dts[k] > 0) || !std::isfinite(dts[k])) {
        B->err = "dt must be positive and finite";
        return FLUID_PP_INVALID_ARG;
      }
  const int rc = batch_project(B, dts, opts, true, receipts);
  if (rc != FLUID_PP_OK && rc != FLUID_PP_NONCONVERGENCE && rc != FLUID_PP_NONFINITE) g_err = B->err;
  return rc;
}

int fluid_pp_batch_project_async(fluid_pp_batch* B, const float* dts, const fluid_pp_solve_opts* opts) {
  if (!B) return FLUID_PP_INVALID_ARG;
  if (batch_streams_ok(B) != FLUID_PP_OK) return FLUID_PP_INVALID_ARG;
  if (dts)
    for (size_t k = 0; k < B->h.size(); ++k)
      if (!(dts[k] > 0) || !std::isfinite(dts[k])) {
        B->err = "dt must be positive and finite";
        g_err = B->err;
        return FLUID_PP_INVALID_ARG;
      }
  const int rc = batch_project(B, dts, opts, false, nullptr);
  if (rc != FLUID_PP_OK) g_err = B->err;
  return rc;
}

int fluid_pp_batch_upload_state(fluid_pp_batch* B, const float* const* vof, const float* const* u,
                                const float* const* v, const float* const* w) {
  if (!B || !vof || !u || !v || !w) return FLUID_PP_INVALID_ARG;
  if (batch_streams_ok(B) != FLUID_PP_OK) return FLUID_PP_INVALID_ARG;
  for (size_t k = 0; k < B->h.size(); ++k) {
    const int rc = upload(B->h[k], vof[k], u[k], v[k], w[k], cudaMemcpyHostToDevice);
    if (rc != FLUID_PP_OK) {
      B->err = B->h[k]->err;
      g_err = B->err;
      return rc;
    }
  }
  return FLUID_PP_OK;
}

int fluid_pp_batch_download_async(fluid_pp_batch* B, float* const* p, float* const* u, float* const* v,
                                  float* const* w) {
  if (!B) return FLUID_PP_INVALID_ARG;
  if (batch_streams_ok(B) != FLUID_PP_OK) return FLUID_PP_INVALID_ARG;
  for (size_t k = 0; k < B->h.size(); ++k) {
    const int rc = fluid_pp_download_async(B->h[k], p ? p[k] : nullptr, u ? u[k] : nullptr, v ? v[k] : nullptr,
                                           w ? w[k] : nullptr);
    if (rc != FLUID_PP_OK) {
      B->err = B->h[k]->err;
      g_err = B->err;
      return rc;
    }
  }
  return FLUID_PP_OK;
}

int fluid_pp_batch_receipts_read(fluid_pp_batch* B, fluid_pp_receipt* receipts) {
  if (!B) return FLUID_PP_INVALID_ARG;
  cudaSetDevice(B->device);
  if (B->parts_pending) {
    const int rc = parts_receipts(B, receipts);
    if (rc == FLUID_PP_CUDA) g_err = B->err;
    return rc;
  }
  const cudaError_t e = cudaStreamSynchronize(B->stream);
  if (e != cudaSuccess) {
    B->err = std::string("project: ") + cudaGetErrorString(e);
    g_err = B->err;
    return FLUID_PP_CUDA;
  }
  if (B->pending_graph_count) {
    g_launches.fetch_add((unsigned long long)(*B->h_loop) * B->n_body, std::memory_order_relaxed);
    B->pending_graph_count = false;
  }
  int worst = FLUID_PP_OK;
  for (size_t k = 0; k < B->h.size(); ++k) {
    if (receipts) fill_receipt(B->h[k], B->h_ctrl[k], receipts + k);
    B->h[k]->has_pressure = true;
    if (B->h_ctrl[k].status != FLUID_PP_OK && worst == FLUID_PP_OK) worst = B->h_ctrl[k].status;
  }
  prof_collect(B);
  return worst;
}

}  // extern "C"
