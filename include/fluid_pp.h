/*
 * fluid_pp.h -- C ABI of the B200 free-surface pressure projection.
 *
 * One handle owns one dense uniform MAC grid resident in device memory: the
 * VOF field, the face velocities, the multigrid hierarchy and the pressure.
 * A projection runs: cell labelling -> divergence -> ghost-fluid theta
 * assembly -> multigrid-preconditioned CG -> gradient subtract, entirely on
 * the device, and returns a receipt.  Every entry point returns an int status
 * (FLUID_PP_OK on success); no exception crosses the boundary.  Host pointers
 * are borrowed for the duration of the call only.  One handle per host thread;
 * the batch entry points are the only calls that touch several handles.
 *
 * Array layouts (float32, x fastest, cubic cells of size h):
 *   vof [nz][ny][nx]      liquid volume fraction
 *   u   [nz][ny][nx+1]    x-face velocity, face x sits between cells x-1 and x
 *   v   [nz][ny+1][nx]    y-face velocity
 *   w   [nz+1][ny][nx]    z-face velocity
 *   p   [nz][ny][nx]      pressure in Pa (zero outside the liquid)
 *
 * Each declaration names the reference interface it replaces (paths inside
 * the peter-suggate/fluid tree).
 */
#ifndef FLUID_PP_H
#define FLUID_PP_H

#ifdef __cplusplus
extern "C" {
#endif

#define FLUID_PP_OK 0
#define FLUID_PP_INVALID_ARG 1   /* host precondition failed (RangeError in the reference) */
#define FLUID_PP_OOM 2
#define FLUID_PP_NONFINITE 3     /* non-finite input; the previous pressure is kept */
#define FLUID_PP_NONCONVERGENCE 4/* iteration cap or lost curvature; iterate published, status set */
#define FLUID_PP_TIMEOUT 5
#define FLUID_PP_CUDA 6          /* CUDA runtime error; see fluid_pp_last_error */
#define FLUID_PP_UNSUPPORTED 7

#define FLUID_PP_MAX_LEVELS 24

enum fluid_pp_precision {
  FLUID_PP_FP32 = 0, /* multigrid levels stored in float32 */
  FLUID_PP_FP16 = 1, /* multigrid levels stored in float16, float32 arithmetic */
  FLUID_PP_BF16 = 2  /* multigrid levels stored in bfloat16, float32 arithmetic */
};

/* Kernel stages reported by the profiling entry points. */
enum fluid_pp_stage {
  FLUID_PP_STAGE_RESET = 0, FLUID_PP_STAGE_LABEL, FLUID_PP_STAGE_COARSEN, FLUID_PP_STAGE_BAKE,
  FLUID_PP_STAGE_FACTOR, FLUID_PP_STAGE_INIT, FLUID_PP_STAGE_SMOOTH0, FLUID_PP_STAGE_SMOOTHC,
  FLUID_PP_STAGE_RESIDUAL0, FLUID_PP_STAGE_RESIDUALC, FLUID_PP_STAGE_RESTRICT0, FLUID_PP_STAGE_RESTRICTC,
  FLUID_PP_STAGE_COARSE, FLUID_PP_STAGE_PROLONG0, FLUID_PP_STAGE_PROLONGC, FLUID_PP_STAGE_DOT,
  FLUID_PP_STAGE_DIR, FLUID_PP_STAGE_SPMV, FLUID_PP_STAGE_UPDATE, FLUID_PP_STAGE_TRUE, FLUID_PP_STAGE_GRAD,
  FLUID_PP_STAGE_RECEIPT, FLUID_PP_STAGE_DOWN0, FLUID_PP_STAGE_DOWNC, FLUID_PP_STAGE_UP0, FLUID_PP_STAGE_UPC,
  FLUID_PP_STAGE_DIRSPMV
};
#define FLUID_PP_PROFILE_STAGES 27

typedef struct fluid_pp fluid_pp;
typedef struct fluid_pp_batch fluid_pp_batch;

typedef struct fluid_pp_config {
  int nx, ny, nz;   /* physical lattice, cells */
  float h;          /* cell size, m */
  float rho;        /* liquid density, kg/m^3 */
  int open_top;     /* 1: the +y domain face is atmospheric air, else a closed wall */
  int precision;    /* enum fluid_pp_precision: storage of the V-cycle levels */
  int device;       /* CUDA device ordinal */
} fluid_pp_config;

typedef struct fluid_pp_solve_opts {
  double rel_tol;          /* stop when ||b - A p||_2 <= max(abs_tol, rel_tol * ||b||_2) */
  double abs_tol;
  int max_iters;           /* CG iteration cap */
  int pre_sweeps;          /* red-black Gauss-Seidel sweeps before restriction */
  int post_sweeps;         /* ... after prolongation (equal to pre_sweeps keeps M symmetric) */
  int true_residual_every; /* replace r by b - A p, recomputed in float64, every k iterations (0: only when the
                              recursive residual meets the tolerance).  Opts NULL: 4.  Without it the float32
                              recursive residual drifts on smooth right-hand sides (e.g. a step whose input is
                              the previous step's projected velocity plus gravity) and CG stalls above 1e-6. */
  int warm_start;          /* 1: start from the previous pressure of this handle */
  double rel_tol_inf;      /* >0: also require max|b - A p| <= rel_tol_inf * max|b| (divergence in max norm) */
  int cycle;               /* preconditioner: 0 (opts NULL) one V-cycle under PCG; 1 one full (F) cycle under
                              flexible CG, beta = r_k+1 . (z_k+1 - z_k) / r_k . z_k (Polak-Ribiere), the
                              schedule of the reference's fullCycle (webgpu-uniform-pressure-multigrid.ts:539-563).
                              Uniform grid only; the tall grid rejects 1. */
} fluid_pp_solve_opts;

typedef struct fluid_pp_receipt {
  int status;               /* FLUID_PP_* of this solve */
  int iterations;           /* CG iterations */
  int liquid_cells;
  int levels;               /* multigrid levels */
  double b_norm;            /* ||b||_2, finest-cell units */
  double rel_residual;      /* recursive ||r||/||b|| at exit */
  double true_rel_residual; /* ||b - A p||/||b|| recomputed in float64 */
  double max_div_before;    /* max |div u - div_target| over liquid cells, 1/s */
  double max_div_after;
  double l2_div_before;     /* sqrt(sum (div)^2 h^3) over liquid cells */
  double l2_div_after;
} fluid_pp_receipt;

/* Hierarchy planner, host only (no GPU needed).
 * Replaces planUniformCM11aHierarchy
 * (lib/methods/uniform/webgpu-uniform-pressure-multigrid.ts:149-169).  Lattices
 * the reference rejects are planned by ceil-halving (extended = 1).
 * level_dims receives level_count * 3 ints, finest first. */
int fluid_pp_plan_hierarchy(int nx, int ny, int nz, int* level_count, int* level_dims, int* coarsest_cells,
                            int* semi_coarsened, int* extended);

/* Replaces `new WebGPUUniformPressureMultigrid(device, dims, spacing, schedule)`
 * (webgpu-uniform-pressure-multigrid.ts:246-301) plus its initialize()
 * (:311-324): allocates every level and the resident state. */
int fluid_pp_create(const fluid_pp_config* config, fluid_pp** out);

/* Device bytes a handle for this configuration allocates (its arena and tables);
 * host only.  The serving loop's admission by HBM budget reads it. */
int fluid_pp_required_bytes(const fluid_pp_config* config, unsigned long long* bytes);

/* Replaces WebGPUUniformPressureMultigrid.destroy() (webgpu-uniform-pressure-multigrid.ts:595-604). */
void fluid_pp_destroy(fluid_pp* pp);

/* Launch every kernel of this handle on `stream` (a cudaStream_t; NULL = legacy default). */
int fluid_pp_set_stream(fluid_pp* pp, void* stream);

/* Copies the step's VOF and face velocities from host memory into the handle.
 * Replaces the texture uploads of WebGPUUniformReferenceSolver
 * (lib/methods/uniform/webgpu-uniform-reference.ts:836-894 initial state,
 * velocity/volume textures bound at :405-413). */
int fluid_pp_upload_state(fluid_pp* pp, const float* vof, const float* u, const float* v, const float* w);

/* Device-pointer variant of upload: copies from device buffers (same layouts). */
int fluid_pp_upload_state_device(fluid_pp* pp, const float* vof, const float* u, const float* v, const float* w);

/* Embedded solids (cut cells), host arrays, kept for every later projection of
 * the handle.  Replaces the solid topology the reference bakes on the finest
 * level (mgBuildFinestTopology, webgpu-uniform-pressure-multigrid.wgsl.ts:
 * 136-150: cellOpenFraction and pressureFaceVolumeFraction,
 * webgpu-uniform-reference.wgsl.ts:208-233, 530-556) and the solid face
 * velocities of its divergence and projection (:1005-1024, :1052-1099).
 *   open  [nz][ny][nx]    open (non-solid) volume fraction of each cell, in [0, 1]
 *   fx, fy, fz            open fraction of each MAC face's dual cell, layouts of u, v, w
 *   usx, usy, usz         the solids' normal velocity on each face (all NULL: static solids)
 * Fractions are clamped to [0, 1]; a face at or below 1e-6 is closed.  The
 * operator's face weights become the face fractions (coarse levels: the mean of
 * the eight children's), rho' = vof / open with the open neighbours' maximum
 * continued into solid cells (open <= 1e-5), and every level below the coarsest
 * runs the face-weighted grid kernels.  Allocates about (4 + 24 + 14) bytes per
 * cell beside the arena, once.  Upload solids before creating a batch of the
 * handle; a batch holds handles that all have solids or none. */
int fluid_pp_upload_solids(fluid_pp* pp, const float* open, const float* fx, const float* fy, const float* fz,
                           const float* usx, const float* usy, const float* usz);

/* The CM11a LCP variant (the reference's uniform GPU method,
 * webgpu-uniform-pressure-multigrid.ts:419-576, .wgsl.ts:155-166, 267-344,
 * 404-471): a standalone projected multigrid solve of A p = b with p >= 0 on
 * solid cells that are pressure unknowns (a separating boundary; a domain wall
 * that should separate is a layer of solid cells, the reference's halo) and
 * p unbounded elsewhere.  full_cycles full cycles, then v_cycles V-cycles, each
 * level smoothed by projected red-black Gauss-Seidel; a coarse correction is
 * bounded by max over the children of (p_min - p) on the first
 * constraint_levels coarse levels (mgDownsampleSubtract) and unbounded below
 * them; the coarsest runs projected sweeps until its projected residual is at
 * most coarse_tol x max|rhs| or coarse_sweeps sweeps.  Needs embedded solids
 * (fluid_pp_upload_solids).  The receipt's true_rel_residual is the fine
 * level's projected fixed-point residual over ||b|| (mgMeasureFineResidual),
 * iterations the number of cycles; the velocities are projected like
 * fluid_pp_project's. */
/* Velocity extrapolation into the air (CM12 Sec. 3.3 / CM11b Secs. 3.3-3.3.1),
 * replacing WebGPUUniformVelocityExtrapolator.encode
 * (lib/methods/uniform/webgpu-uniform-velocity-extrapolation.ts:328-395), in
 * place on the handle's u, v, w (e.g. after fluid_pp_project, before the host's
 * advection reads them back with fluid_pp_download).  Source faces (open faces
 * with a liquid side, rho' > 0.5) keep their values; the other open faces take
 * the Fast Iterative Method's upwind extension within two cells of the liquid
 * and, farther out, the known-value hierarchy's fill (0 where none reaches);
 * closed faces (walls, closed solid faces) are left as they are.
 * *filled_faces (may be NULL) receives the open faces holding a value. */
int fluid_pp_extrapolate_velocity(fluid_pp* pp, long long* filled_faces);

/* CM12 conservative surface-density transport (Secs. 3.4-3.5), replacing the
 * dense uniform method's density passes (lib/methods/uniform/
 * webgpu-uniform-reference.ts:1150-1215; .wgsl.ts:640-858, 1187-1255): the
 * handle's VOF (surface density rho) and its persistent gamma advance by dt
 * along the handle's face velocities (extrapolate them first), then gamma
 * diffuses and the density is sharpened with its local mass return.  The new
 * rho replaces the handle's VOF, ready for fluid_pp_project.  Options outside
 * the reference's ranges are clamped as it clamps them.  Handles with
 * embedded solids: FLUID_PP_UNSUPPORTED. */
typedef struct fluid_pp_transport_opts {
  int gamma_diffusion_iterations;   /* 1 (0 .. 7), x -> y -> z Jacobi repetitions */
  int sharpening;                   /* 1 */
  int sharpening_mass_return;       /* 1: removed mass carried to the 0.5 contour */
  float sharpening_strength;        /* 1 (0.25 .. 2) */
  float sharpening_distance;        /* 2.1 cells (0.1 .. 3.1) */
} fluid_pp_transport_opts;
void fluid_pp_transport_opts_default(fluid_pp_transport_opts* opts);

typedef struct fluid_pp_transport_receipt {
  double mass_before;   /* sum of rho over the cells before the step (float64) */
  double mass_after;
  float rho_min, rho_max;   /* after the step */
} fluid_pp_transport_receipt;
int fluid_pp_transport_density(fluid_pp* pp, float dt, const fluid_pp_transport_opts* opts,
                               fluid_pp_transport_receipt* receipt);
/* The persistent gamma, [nz][ny][nx] host floats (1 everywhere until set;
 * NULL resets it to 1). */
int fluid_pp_set_gamma(fluid_pp* pp, const float* gamma);
/* The handle's VOF (rho), [nz][ny][nx] host floats. */
int fluid_pp_get_vof(fluid_pp* pp, float* vof);
int fluid_pp_get_gamma(fluid_pp* pp, float* gamma);

typedef struct fluid_pp_lcp_opts {
  int full_cycles;        /* 3 (UNIFORM_CM11A_FULL_CYCLES) */
  int v_cycles;           /* 4 (UNIFORM_CM11A_V_CYCLES) */
  int pre_sweeps;         /* 1 */
  int post_sweeps;        /* 1 */
  int constraint_levels;  /* 3 (UNIFORM_CM11A_CONSTRAINT_LEVELS) */
  int coarse_sweeps;      /* 4096 (UNIFORM_CM11A_COARSE_SWEEP_CAP) */
  double coarse_tol;      /* 1e-6 */
  int warm_start;         /* 1: start from the handle's previous pressure */
} fluid_pp_lcp_opts;
void fluid_pp_lcp_opts_default(fluid_pp_lcp_opts* opts);
int fluid_pp_project_lcp(fluid_pp* pp, float dt, const fluid_pp_lcp_opts* opts, fluid_pp_receipt* receipt);

/* Label -> divergence -> assemble -> MGPCG -> gradient subtract, on the device.
 * Replaces WebGPUUniformPressureMultigrid.encode (webgpu-uniform-pressure-multigrid.ts:327-364)
 * followed by the `project` dispatch (webgpu-uniform-reference.ts:1280-1282);
 * the receipt replaces the diagnostics words read by readStats
 * (webgpu-uniform-reference.ts:1358-1420).  dt in seconds; opts may be NULL
 * (rel 1e-6, 200 iterations, 1+1 sweeps, true residual every 4).  The receipt is written after the
 * stream synchronises. */
int fluid_pp_project(fluid_pp* pp, float dt, const fluid_pp_solve_opts* opts, fluid_pp_receipt* receipt);

/* Asynchronous form: enqueues the projection on the handle's stream and returns
 * without synchronising; fluid_pp_receipt_read() synchronises and fills it. */
int fluid_pp_project_async(fluid_pp* pp, float dt, const fluid_pp_solve_opts* opts);
int fluid_pp_receipt_read(fluid_pp* pp, fluid_pp_receipt* receipt);

/* Copies pressure (Pa) and projected velocities to host memory; any pointer may be NULL.
 * Replaces the pressureTexture / velocity readback (webgpu-uniform-pressure-multigrid.ts:303). */
int fluid_pp_download(fluid_pp* pp, float* p, float* u, float* v, float* w);

/* fluid_pp_download without the wait: enqueues the copies on the handle's
 * stream and returns.  The host buffers must stay valid, and hold the results
 * only after fluid_pp_synchronize (or any later wait on that stream); pinned
 * buffers let the copies overlap work on other streams. */
int fluid_pp_download_async(fluid_pp* pp, float* p, float* u, float* v, float* w);
/* Waits for everything enqueued on the handle's stream. */
int fluid_pp_synchronize(fluid_pp* pp);

/* Device pointers of the resident arrays (for zero-copy consumers); any may be NULL. */
int fluid_pp_device_arrays(fluid_pp* pp, float** p, float** u, float** v, float** w, float** vof);

/* Last error message of this handle (empty string when none). */
const char* fluid_pp_last_error(const fluid_pp* pp);

/* Parity hooks (host arrays).  Level data after the last project/prepare:
 * label (1 liquid, 0 air), phi (finest-cell units), diag (float32, finest-cell units). */
int fluid_pp_prepare(fluid_pp* pp, float dt);   /* label + divergence + hierarchy only */
int fluid_pp_level_dims(fluid_pp* pp, int level, int* dims3);
int fluid_pp_get_level(fluid_pp* pp, int level, unsigned char* label, float* phi, float* diag);
int fluid_pp_get_rhs(fluid_pp* pp, float* b);
int fluid_pp_apply_operator(fluid_pp* pp, const float* p, float* out);  /* finest A, host in/out */
int fluid_pp_apply_vcycle(fluid_pp* pp, const float* r, float* z, int pre, int post);
/* One full (F) cycle z = F(r) with zero initial guess, the preconditioner of
 * solve option cycle = 1: r restricted down every grid level, the levels from
 * *first_block on (at most 4096 cells each, one CTA) solved by one V-cycle,
 * then for each grid level from the coarsest up the prolongated correction is
 * the initial guess of a V-cycle started at that level.  *first_block (may be
 * NULL) receives that first block level (0 for a single-level hierarchy). */
int fluid_pp_apply_fcycle(fluid_pp* pp, const float* r, float* z, int pre, int post, int* first_block);
int fluid_pp_get_pressure_cells(fluid_pp* pp, float* x);             /* solution, finest-cell units */
/* Embedded solids: a level's face open fractions, planar [3][n] (+x, +y, +z face of each cell). */
int fluid_pp_get_level_faces(fluid_pp* pp, int level, float* ff);

/* Batched projection of several handles in one set of launches per stage.
 * Replaces nothing in the reference (which runs one solver per device); the
 * per-solve semantics are those of fluid_pp_project.  Every handle must be on
 * one stream (fluid_pp_set_stream before fluid_pp_batch_create): the batch
 * orders its work on that stream, and a handle's own uploads, downloads and
 * release use the handle's stream.  Handles on different streams, or a member
 * moved to another stream later, give FLUID_PP_INVALID_ARG. */
int fluid_pp_batch_create(fluid_pp* const* handles, int count, fluid_pp_batch** out);
void fluid_pp_batch_destroy(fluid_pp_batch* batch);
int fluid_pp_batch_project(fluid_pp_batch* batch, const float* dts, const fluid_pp_solve_opts* opts,
                           fluid_pp_receipt* receipts);

/* Asynchronous batch form: enqueues the projection on the batch's stream (its
 * first handle's stream) and returns.  fluid_pp_batch_receipts_read waits for
 * that stream, fills `receipts` (one per handle; may be NULL) and returns what
 * fluid_pp_batch_project would have.  The batch only orders work on its own
 * stream: uploads and downloads of its handles belong on that stream too.  With
 * graphs on (the default) nothing waits on the host between the two calls, so a
 * caller can keep two batches on two streams in flight, the copies of one
 * overlapping the solve of the other. */
int fluid_pp_batch_project_async(fluid_pp_batch* batch, const float* dts, const fluid_pp_solve_opts* opts);
int fluid_pp_batch_receipts_read(fluid_pp_batch* batch, fluid_pp_receipt* receipts);
/* fluid_pp_upload_state and fluid_pp_download_async for every handle of the
 * batch in one call: element k of each pointer array belongs to handle k (any
 * of the download arrays may be NULL, and so may an element). */
int fluid_pp_batch_upload_state(fluid_pp_batch* batch, const float* const* vof, const float* const* u,
                                const float* const* v, const float* const* w);
int fluid_pp_batch_download_async(fluid_pp_batch* batch, float* const* p, float* const* u, float* const* v,
                                  float* const* w);

/* How a batch lays out its work (no reference counterpart: the reference
 * solves one grid per device).  A launch of a V-cycle step needs enough tiles
 * to fill the GPU; fill_tiles is that count (default 148, one per SM).  Levels
 * whose next coarser level halves every axis run the column-block kernels,
 * whose tiles are fixed in x / y and split along z into chunks: chunk_planes
 * is the chunk length in level-0 fine planes (a multiple of 8 up to 256,
 * halved on each coarser level), 0 (default) takes the longest chunk whose
 * tiles over the batch reach fill_tiles.  The other levels run box kernels,
 * which take the largest tile shape whose tiles over the batch reach
 * fill_tiles; box_shape 0..4 forces one (largest first), -1 (default) leaves
 * it to fill_tiles.  parts (1..16, default 1) splits the handles into that many
 * sub-batches of about equal cells, each solved on a stream of its own, all
 * started together and joined back to the batch's stream (graph-mode solves;
 * direct launches run the whole batch), so that one part's small launches and
 * last iterations overlap another's work.  Every layout applies the same
 * arithmetic per cell and folds every scalar over the same fixed tiles of one
 * instance, so a batch's results do not depend on its tuning, bit for bit;
 * only its speed does (fluid_b200.autotune measures the candidates). */
typedef struct fluid_pp_batch_tuning {
  int fill_tiles;
  int chunk_planes;
  int box_shape;
  int parts;
} fluid_pp_batch_tuning;
void fluid_pp_batch_tuning_default(fluid_pp_batch_tuning* tuning);
int fluid_pp_batch_create_tuned(fluid_pp* const* handles, int count, const fluid_pp_batch_tuning* tuning,
                                fluid_pp_batch** out);

/* Solve a batch through CUDA graphs (on = 1, the default: the solve is captured
 * once per option set and replayed) or with direct launches (on = 0: for a batch
 * that lives for a few solves, e.g. a serving tick, capture would cost more
 * than it saves).  Results are identical either way. */
int fluid_pp_batch_set_graphs(fluid_pp_batch* batch, int on);

/* Diagnostics (no reference counterpart; the reference times passes with
 * GPUPassTimestampRecorder, lib/core/performance-trace.ts:1183).
 * Kernel launches issued by this library in this process: */
unsigned long long fluid_pp_kernel_launches(void);
/* Per-stage kernel timing with CUDA events on the launching stream (on = 1).
 * read: ms[FLUID_PP_PROFILE_STAGES] and launches[FLUID_PP_PROFILE_STAGES]
 * accumulated since the last reset; reset = 1 clears after reading. */
int fluid_pp_set_profiling(fluid_pp* pp, int on);
int fluid_pp_profile_read(fluid_pp* pp, double* ms, long long* launches, int reset);
int fluid_pp_batch_set_profiling(fluid_pp_batch* batch, int on);
int fluid_pp_batch_profile_read(fluid_pp_batch* batch, double* ms, long long* launches, int reset);

/* Allocation-free finest-level operator apply.  This entry point has no
 * counterpart in the reference.  It is for host applications that cannot let a
 * plug-in allocate device memory (an engine or renderer that has reserved the
 * GPU's memory for its own pool, or a framework whose caching allocator holds
 * the free memory): it allocates nothing and calls no allocating routine.
 * All buffers are caller-owned device memory, x fastest, nx*ny*nz cells:
 * label (1 liquid / 0 air) and diag as returned by fluid_pp_get_level(level 0)
 * for the same state, p the vector to apply.  Writes out = A p (the operator of
 * fluid_pp_apply_operator, with air entries of p treated as zero) and
 * *p_dot_ap = p . A p, accumulated in float64 in a fixed order, asynchronously
 * on `stream` (a cudaStream_t, NULL = legacy default stream).
 * Reduction scratch is one fixed device array inside the library (about 128 KB
 * per GPU, held until the process exits), enough for lattices of up to 16384
 * work tiles of 32x8x4 cells (e.g. 256^3); larger lattices return
 * FLUID_PP_INVALID_ARG with the reason in fluid_pp_last_error(NULL).
 * out and p_dot_ap must not overlap label, diag, p or each other
 * (FLUID_PP_INVALID_ARG otherwise).  Every call looks the scratch address up
 * for the current device (no allocation); the first call on a device may load
 * the library's device code, so make it before any stream capture.  Calls on
 * one device share the scratch, so calls whose GPU work overlaps race. */
int fluid_pp_apply_operator_noalloc(int nx, int ny, int nz, const unsigned char* label, const float* diag,
                                    const float* p, float* out, double* p_dot_ap, void* stream);

/* Allocation cache for servers that create and destroy handles continuously
 * (no reference counterpart: the reference allocates one GPU solver per
 * simulation, lib/core/method-contract.ts:355).  cudaFree waits for the whole
 * device; with the cache on, destroying a handle or batch waits only for its
 * own stream and keeps its device blocks (and pinned control blocks, device
 * -1) on a free list of at most max_cached_bytes, from which later handles of
 * similar sizes are carved without any CUDA allocation call.  0 (the default)
 * turns caching off and frees the list.  Cached bytes stay allocated on the
 * device until trimmed this way.  With the cache on, the work of a handle or
 * batch must have been issued on its own stream (fluid_pp_set_stream, the
 * batch's first handle's stream) or have finished before it is destroyed. */
int fluid_pp_set_allocation_cache(int device, unsigned long long max_cached_bytes);
/* Reserves `bytes` of device memory for the cache in one cudaMalloc, so that
 * later handles are carved from memory already mapped (a first-time cudaMalloc
 * of a large arena can take tens of ms).  While the cache is on, handles take
 * slab ranges by best fit and released ranges coalesce.  The slabs are freed
 * when the cache is turned off with none of their ranges in use. */
int fluid_pp_reserve_allocation(int device, unsigned long long bytes);
/* Bytes the cache holds free on `device` (block list plus free slab ranges). */
int fluid_pp_allocation_cache_bytes(int device, unsigned long long* cached_bytes);

/* ------------------------------------------------------------------------
 * Restricted tall-cell grid (lib/core/tall-cell-grid.ts).  An nx x nz grid of
 * columns over fine_ny world rows: each column has one tall cell over rows
 * [0, base) and a cubic band of `band` rows above it.  Every per-cell array is
 * packed per column in P = band + 2 samples, float32 [nz][P][nx]: sample 0 is
 * the tall cell's bottom subcell (row 0), sample 1 its top subcell
 * (row base - 1), sample j >= 2 the band row base + j - 2 (tall-cell-grid.ts:
 * 171-190, 398-409).  Face velocities are packed the same way: each sample
 * owns the +x, +y and +z faces of its cell.
 * ---------------------------------------------------------------------- */
typedef struct fluid_pp_tall fluid_pp_tall;

typedef struct fluid_pp_tall_config {
  int nx, nz;      /* columns */
  int fine_ny;     /* world rows */
  int band;        /* cubic rows per column (B_y) */
  float h;         /* cell size, m */
  float rho;       /* liquid density, kg/m^3 */
  int precision;   /* FLUID_PP_FP32 */
  int device;
} fluid_pp_tall_config;

/* chooseTallCellBase (lib/core/tall-cell-grid.ts:61-82), host only. */
int fluid_pp_tall_choose_base(int lowest_surface, int highest_surface, int fine_ny, int regular_layers,
                              int liquid_halo, int air_halo);

/* limitNeighboringTallCellBases (tall-cell-grid.ts:84-106), host only; bases
 * (x + nx * z) are limited in place. */
int fluid_pp_tall_limit_bases(float* bases, int nx, int nz, int max_delta, int passes);

/* Tall multigrid hierarchy, host only: level_shapes receives level_count * 4
 * ints (nx, fine_ny, nz, band), finest first. */
int fluid_pp_tall_plan(int nx, int nz, int fine_ny, int band, const int* bases, int* level_count, int* level_shapes);

/* Replaces the restricted backend's pressure setup (createTallCellLayout,
 * tall-cell-grid.ts:309-436, plus the tall-cell multigrid of
 * docs/papers/tallCells.txt Alg. 2): allocates the hierarchy for the given
 * bases (every base >= 2, band inside the domain).  Errors: fluid_pp_last_error(NULL). */
int fluid_pp_tall_create(const fluid_pp_tall_config* config, const int* bases, fluid_pp_tall** out);
void fluid_pp_tall_destroy(fluid_pp_tall* tall);
int fluid_pp_tall_set_stream(fluid_pp_tall* tall, void* stream);
/* CUDA graphs of the tall CG iteration (on by default; off: one launch per
 * kernel, e.g. for profilers, which do not see kernels inside conditional graphs). */
int fluid_pp_tall_set_graphs(fluid_pp_tall* T, int on);
/* Packed VOF and owned face velocities from host (or device) memory. */
int fluid_pp_tall_upload_state(fluid_pp_tall* tall, const float* vof, const float* u, const float* v, const float* w);
int fluid_pp_tall_upload_state_device(fluid_pp_tall* tall, const float* vof, const float* u, const float* v,
                                      const float* w);
/* Labels, assembly, MGPCG to the tolerance, gradient subtract on the packed
 * faces, receipt (divergence receipts over liquid band cells).  pre_sweeps /
 * post_sweeps (1 to 4; opts NULL: 2 and 2) count the block Gauss-Seidel sweeps
 * of the grid levels; the levels held in one CTA sweep once. */
int fluid_pp_tall_project(fluid_pp_tall* tall, float dt, const fluid_pp_solve_opts* opts, fluid_pp_receipt* receipt);
/* The same projection in slices (no reference counterpart: a serving loop
 * interleaves other simulations' steps between the slices of a long solve).
 * begin enqueues labels, assembly, right-hand side and the CG start on the
 * handle's stream; continue runs at most max_iterations more CG iterations
 * (<= 0: until done) and sets *finished once the solve converged or hit its
 * iteration cap; end enqueues the gradient subtract, synchronises and fills
 * the receipt.  fluid_pp_tall_project is begin + continue(0) + end. */
int fluid_pp_tall_project_begin(fluid_pp_tall* tall, float dt, const fluid_pp_solve_opts* opts);
int fluid_pp_tall_project_continue(fluid_pp_tall* tall, int max_iterations, int* finished);
int fluid_pp_tall_project_end(fluid_pp_tall* tall, fluid_pp_receipt* receipt);
/* Pressure in Pa and the projected faces, packed. */
int fluid_pp_tall_download(fluid_pp_tall* tall, float* p, float* u, float* v, float* w);
/* Diagnostics for parity tests: prepare runs labels, hierarchy and assembly
 * for dt; then the finest-level rhs, labels per level, A p, the solved pressure
 * (finest-cell units, double-single rounded once). */
int fluid_pp_tall_prepare(fluid_pp_tall* tall, float dt);
int fluid_pp_tall_get_rhs(fluid_pp_tall* tall, float* b);
int fluid_pp_tall_get_labels(fluid_pp_tall* tall, int level, unsigned char* label);
int fluid_pp_tall_apply_operator(fluid_pp_tall* tall, const float* p, float* out);
int fluid_pp_tall_get_pressure(fluid_pp_tall* tall, float* p);
/* Parity hook: solve the assembled finest system A x = b for a caller-given b
 * (host, finest-cell units, packed; air entries ignored) with the projection's
 * MGPCG, after labels, hierarchy and operator are built from the uploaded state
 * and dt.  x (host, packed) receives the solution in finest-cell units.  Lets a
 * test refine a float64 solution of an independently assembled system with the
 * device solver.  Returns the solve status. */
int fluid_pp_tall_solve_rhs(fluid_pp_tall* tall, float dt, const float* b, const fluid_pp_solve_opts* opts,
                            float* x, fluid_pp_receipt* receipt);
const char* fluid_pp_tall_last_error(fluid_pp_tall* tall);
/* Device bytes a tall handle for this layout allocates; host only. */
int fluid_pp_tall_required_bytes(const fluid_pp_tall_config* config, const int* bases, unsigned long long* bytes);

/* ------------------------------------------------------------------------
 * Sparse brick atlas: the default adaptive method's pressure projection
 * (lib/methods/adaptive-mass/webgpu-sparse-cm12-resident.ts; its CPU
 * statement projectSparseAtlasVelocity, sparse-atlas-composite-projection.ts:
 * 978-1566) for atlases whose bricks all carry the finest resolution.  Only
 * the present bricks of 8^3 cells are stored.  Faces between present bricks,
 * faces to absent bricks inside the domain (air, phi 0.5) and faces inside a
 * brick are the system's rows; domain faces are walls.  A cell is liquid iff
 * rho >= 0.5; liquid with no face to air is a pure Neumann problem whose mean
 * pressure is removed, as the reference removes it.
 * ---------------------------------------------------------------------- */
typedef struct fluid_pp_atlas fluid_pp_atlas;

typedef struct fluid_pp_atlas_config {
  int nx, ny, nz;   /* domain in finest cells, multiples of 8 */
  float h;          /* cell size, m */
  float rho;        /* liquid density, kg/m^3 */
  int device;
} fluid_pp_atlas_config;

/* Host only: the block hierarchy's level count and cells per level (at most
 * 16 levels), and (with density) the liquid components without a face to air
 * and their cells. */
int fluid_pp_atlas_plan(int nx, int ny, int nz, int nbricks, const int* coords, const float* density,
                        int* level_count, long long* level_cells, int* components, int* component_cells);
int fluid_pp_atlas_create(const fluid_pp_atlas_config* config, fluid_pp_atlas** out);
void fluid_pp_atlas_destroy(fluid_pp_atlas* atlas);
int fluid_pp_atlas_set_stream(fluid_pp_atlas* atlas, void* stream);
/* The PCG iteration as a CUDA graph (default on); off: one launch per kernel (profilers). */
int fluid_pp_atlas_set_graphs(fluid_pp_atlas* atlas, int on);
/* nbricks bricks: coords (bx, by, bz) per brick (each in [0, n / 8)), density
 * nbricks x 512 floats [brick][z][y][x], faces nbricks x 3 x 576 floats: per
 * brick its u [8][8][9], v [8][9][8], w [9][8][8] (face f of an axis between
 * local cells f - 1 and f).  A face between two present bricks is read from
 * the lower brick's copy.  Builds the rows' weights and the block hierarchy. */
int fluid_pp_atlas_upload(fluid_pp_atlas* atlas, int nbricks, const int* coords, const float* density,
                          const float* faces);
/* PCG to ||b - A p|| <= max(abs_tol, rel_tol ||b||) (opts NULL: 1e-6, 200
 * iterations).  opts->cycle 0: one V-cycle on the brick hierarchy per
 * iteration (pre_sweeps / post_sweeps red-black sweeps on every level, 1 to
 * 4; opts NULL: 2 and 2); 2: Jacobi (the reference's own preconditioner);
 * others FLUID_PP_UNSUPPORTED.  Faces of rows with a liquid side take
 * u - (dt / rho) grad p / theta, faces of rows without one become 0, domain
 * walls keep their values.  Divergence receipts are over liquid cells. */
int fluid_pp_atlas_project(fluid_pp_atlas* atlas, float dt, const fluid_pp_solve_opts* opts, fluid_pp_receipt* receipt);
/* pressure: nbricks x 512 floats in Pa (0 off the liquid); faces: as uploaded.  Either may be NULL. */
int fluid_pp_atlas_download(fluid_pp_atlas* atlas, float* pressure, float* faces);
const char* fluid_pp_atlas_last_error(fluid_pp_atlas* atlas);

#ifdef __cplusplus
}
#endif
#endif /* FLUID_PP_H */
