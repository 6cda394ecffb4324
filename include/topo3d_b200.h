/*
 * topo3d_b200 — C ABI of the B200 (sm_100a) SIMP hot path.
 *
 * Every entry point takes plain device pointers and sizes plus a `void*`
 * CUDA stream (NULL = legacy default stream) and returns an int status:
 *   0  ok,  >0 not converged / iteration cap,  <0 bad argument or CUDA error.
 * `tp3d_last_error()` returns a thread-local message for the last failure.
 *
 * Array conventions (all follow PyTopo3D):
 *   element arrays: length nelx*nely*nelz, Fortran order of the (nely, nelx,
 *     nelz) design array, e = y + nely*(x + nelx*z)   (pytopo3d/utils/filter.py:85-87)
 *   node / DOF vectors: DOF = 3*(iy + (nely+1)*(ix + (nelx+1)*iz)) + c
 *     (pytopo3d/utils/assembly.py:121-129, 375-401)
 *   masks: uint8, nonzero = true.
 * The caller owns every buffer passed in.  Solver handles own their scratch
 * and multigrid hierarchy; a handle belongs to one stream and one thread.
 */
#ifndef TOPO3D_B200_H
#define TOPO3D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TP3D_OK 0
#define TP3D_NOT_CONVERGED 1
#define TP3D_ERR_ARG (-1)
#define TP3D_ERR_CUDA (-2)
#define TP3D_ERR_TIMEOUT (-3)   /* a bounded device-side wait expired */
#define TP3D_ERR_NONFINITE (-4) /* NaN / Inf met in a reduction */

#define TP3D_PRECISION_FP64 0  /* FP64 everywhere */
#define TP3D_PRECISION_MIXED 1 /* FP32 inner PCG + BF16 density, FP64 refinement */

const char* tp3d_last_error(void);
int tp3d_abi_version(void);

/* Kernel launches issued by this library since load (CUDA-graph replays add
 * their kernel-node count).  Instrumentation; no reference counterpart. */
long long tp3d_launch_count(void);

/* ---------------------------------------------------------------------------
 * Density filter and Heaviside projection
 * ------------------------------------------------------------------------- */

/* Row sums Hs of the cone filter, zero sums replaced by 1.
 * Replaces build_filter's Hs (pytopo3d/utils/filter.py:122-228); the matrix H
 * itself is never formed: every filter entry point applies the same cone
 * weights rmin - |d| > 1e-9 as a stencil. */
int tp3d_filter_rowsum(int nelx, int nely, int nelz, double rmin, double* Hs, void* stream);

/* rho_filtered = (H x) / Hs, projected and clamped on protected regions.
 * Replaces build_physical_density (pytopo3d/utils/filter.py:63-100) and
 * heaviside_projection (filter.py:26-60).  rho_filtered and dproj may be NULL;
 * solid / void_ may be NULL (no protected elements). */
int tp3d_filter_project(int nelx, int nely, int nelz, double rmin, const double* x,
                        const double* Hs, double beta, double eta, const uint8_t* solid,
                        const uint8_t* void_, double* rho_filtered, double* rho_physical,
                        double* dproj, void* stream);

/* out = H^T (g * dproj / Hs).  Replaces apply_density_filter_chain_rule
 * (pytopo3d/utils/filter.py:103-119).  dproj may be NULL (treated as 1). */
int tp3d_filter_transpose(int nelx, int nely, int nelz, double rmin, const double* g,
                          const double* dproj, const double* Hs, double* out, void* stream);

/* Elementwise tanh projection and its derivative, n values.
 * Replaces heaviside_projection (pytopo3d/utils/filter.py:26-60). */
int tp3d_heaviside(const double* rho_filtered, long long n, double beta, double eta, double* out,
                   double* derivative, void* stream);

/* ---------------------------------------------------------------------------
 * Element energy and sensitivities
 * ------------------------------------------------------------------------- */

/* ce[e] = u_e^T KE u_e.  KE is 24x24 row-major on the HOST.
 * Replaces element_compliance (pytopo3d/core/compliance.py:18-75). */
int tp3d_element_compliance(int nelx, int nely, int nelz, const double* U, const double* KE_host,
                            double* ce, void* stream);

/* Fused loop-body sensitivities (pytopo3d/core/optimizer.py:596-625):
 *   ce, compliance = sum (Emin + (1-Emin) rho^p) ce  (written to *compliance, device),
 *   dc_dx = H^T(dc dproj / Hs) with dc = -p (1-Emin) rho^(p-1) ce,
 *   dv_dx = H^T(free dproj / Hs).
 * ce may be NULL.  `scratch` holds >= tp3d_sensitivity_scratch_bytes() bytes of
 * device memory. */
size_t tp3d_sensitivity_scratch_bytes(int nelx, int nely, int nelz);
int tp3d_sensitivity(int nelx, int nely, int nelz, double rmin, const double* U,
                     const double* KE_host, const double* rho_physical, const double* dproj,
                     const double* Hs, const uint8_t* free_mask, double penal, double* ce,
                     double* dc_dx, double* dv_dx, double* compliance, void* scratch,
                     void* stream);

/* ---------------------------------------------------------------------------
 * Optimality-criteria update with projected-volume bisection
 * ------------------------------------------------------------------------- */

/* Replaces optimality_criteria_update_projected (pytopo3d/utils/oc_update.py:25-124).
 * The whole lambda bisection runs in one cooperative launch; each step
 * re-filters and re-projects the candidate on the device.
 * stats (device, 8 doubles): [lambda_best, volume_best, steps, change,
 *   ratio_scale, lambda_lo, lambda_hi, best_error].
 * change = max |x_new - x| over free elements (optimizer.py:642).
 * `scratch` holds >= tp3d_oc_scratch_bytes() bytes of device memory. */
size_t tp3d_oc_scratch_bytes(int nelx, int nely, int nelz, double rmin);
int tp3d_oc_update(int nelx, int nely, int nelz, double rmin, const double* x,
                   const double* dc_dx, const double* dv_dx, const double* Hs,
                   const uint8_t* solid, const uint8_t* void_, double move,
                   double target_free_volume, double beta, double eta, int max_bisection,
                   double bisection_tol, double* x_new, double* rho_new, double* stats,
                   void* scratch, void* stream);

/* The same OC update without any device allocation, for callers that must
 * not allocate device memory per call (an application whose device memory
 * is reserved up front by its own allocator, or code that cannot accept the
 * implicit device synchronisation of cudaMalloc / cudaFree).  No counterpart
 * in the reference: it is an addition of this library.
 * Scratch is one file-scope __device__ array (about 2.2 MB) that every GPU
 * loading this library holds until exit; grids above
 * tp3d_oc_noalloc_max_elements() (262144) elements are rejected with
 * TP3D_ERR_ARG.  The first call on a device looks up the array's address
 * (cudaGetSymbolAddress) and should come before any stream capture.  Each
 * call queues only device work on `stream` (the filter column table is built
 * in the array by a small kernel, the barrier words and stats are cleared by
 * memsets): no host buffer is read after the call returns.  All calls share
 * the array, so calls that overlap on the GPU race; issue them on one stream.
 * Arguments and results are those of tp3d_oc_update. */
long long tp3d_oc_noalloc_max_elements(void);
int tp3d_oc_update_noalloc(int nelx, int nely, int nelz, double rmin, const double* x,
                           const double* dc_dx, const double* dv_dx, const double* Hs,
                           const uint8_t* solid, const uint8_t* void_, double move,
                           double target_free_volume, double beta, double eta, int max_bisection,
                           double bisection_tol, double* x_new, double* rho_new, double* stats,
                           void* stream);

/* Wait-expiry test hook: from the next OC launch on, every grid-barrier wait
 * of the OC kernel gives up after `spin_limit` polls (0 = the normal limit of
 * about a second) and waits for `phantom_blocks` extra blocks that never
 * arrive (0 = none), so with phantom_blocks > 0 every wait runs out and the
 * launch ends with its stats left NaN, which the Python layer reports as
 * Topo3dError.  Process-wide; tests only (it checks that an expired bounded
 * wait reaches the host as an error and leaves the context usable).  No
 * reference counterpart. */
int tp3d_debug_expire_oc_waits(long long spin_limit, int phantom_blocks);

/* ---------------------------------------------------------------------------
 * Obstacle masks
 * ------------------------------------------------------------------------- */

#define TP3D_OBSTACLE_CUBE 0
#define TP3D_OBSTACLE_SPHERE 1
#define TP3D_OBSTACLE_CYLINDER 2

/* One obstacle primitive in element indices (x, y, z order), as the reference
 * computes them from fractions with int() truncation:
 *   cube:     lo <= (x, y, z) < hi                    (obstacles.py:12-61)
 *   sphere:   |(x, y, z) - center|^2 <= r2            (obstacles.py:63-108)
 *   cylinder: squared distance to center in the two axes other than `axis`
 *             <= r2, and lo[axis] <= coordinate along axis < hi[axis]
 *                                                     (obstacles.py:110-193) */
typedef struct tp3d_obstacle {
  int kind;
  int axis;
  int center[3];
  int lo[3];
  int hi[3];
  long long r2;
} tp3d_obstacle;

/* mask[e] = 1 where any of the `nshapes` primitives (host array) contains
 * element e, else 0; mask is a device array of nelx*nely*nelz bytes in the
 * element order above.  Replaces the numpy mask construction of
 * create_cube/sphere/cylinder_obstacle and the OR of parse_obstacle_config_file
 * (pytopo3d/utils/obstacles.py:12-269). */
int tp3d_obstacle_mask(int nelx, int nely, int nelz, const tp3d_obstacle* shapes, int nshapes, uint8_t* mask,
                       void* stream);

/* ---------------------------------------------------------------------------
 * Matrix-free H8 elasticity solver (multigrid-preconditioned CG)
 * ------------------------------------------------------------------------- */

typedef struct tp3d_solver tp3d_solver;

typedef struct tp3d_solver_opts {
  int precision;        /* TP3D_PRECISION_FP64 or TP3D_PRECISION_MIXED */
  int max_iterations;   /* CG iterations */
  double rtol;          /* target ||f - K u|| / ||f|| (checked on the FP64 residual) */
  int pre_sweeps;       /* smoother degree before restriction (<= 8) */
  int post_sweeps;      /* smoother degree after prolongation (<= 8) */
  double omega;         /* damped-Jacobi weight when smoother == 1 */
  int coarsest_max_dofs;/* stop coarsening at or below this many DOFs */
  int max_levels;       /* cap on multigrid levels (1 = Jacobi-PCG only) */
  int smoother;         /* 0 Chebyshev(Jacobi) with power-iteration bounds, 1 damped Jacobi */
  double cheb_ratio;    /* Chebyshev interval [lambda_max / ratio, lambda_max] (default 30) */
  int power_iterations; /* power iterations per level for lambda_max(Dinv A) */
  int inner_density;    /* mixed: FP32 fine operator from 0 = FP32 moduli, 1 = BF16 densities */
  double reliable_delta;/* mixed: replace the FP32 residual by the FP64 one when it fell by this factor
                           (default 0.05; 0.01 measured 1.5% faster on the 128x64x64 step, but the
                           FP32 residual then drifts further from the FP64 one between
                           replacements, and a solve ended 2% above rtol) */
  int max_restarts;     /* FP64: restarts from the true residual when the recursive one drifted */
  int fine_operator;    /* fine-level K u: 0 the fastest of the dense-KE form and the Walsh-Hadamard
                           block form's launch shapes, tile shapes (the three with the fewest blocks
                           per node plane) and slab depths, timed on the grid at the first
                           set_density; 1 dense KE; 2 Walsh-Hadamard (fastest shape); 3 + v the
                           Walsh-Hadamard form with shape v only (FP64: v = 0..2; FP32: v = 0..2 the
                           packed two-plane kernel with paired FP32 instructions, 3..5 the scalar
                           two-barrier kernel, 6..7 the one-barrier kernel for the apply, residual,
                           CG-product and power-iteration modes; the timed choices 0 and 2 skip the
                           packed shapes, which measured slower).  The block form needs an
                           axis-aligned orthotropic KE and falls back to the dense form otherwise. */
  int fused_cycle_dofs; /* the V-cycle from the first level (>= 1) with at most this many DOFs down
                           to the coarsest runs as one cooperative launch with grid barriers;
                           0 (default) keeps one launch per smoothing step and transfer, which
                           measured faster inside the CUDA graph of a CG iteration on B200 */
  int galerkin;         /* levels >= 2: 0 (default) element-wise Galerkin products (level-2 element
                           matrices from the fine moduli, deeper ones from their 8 sub-elements,
                           then assembled to stencils); 1 stencil triple product P^T A P */
  int coarse_sweeps;    /* smoother degree (before and after) on levels >= 1; 0: pre/post_sweeps.
                           Defaults (fine degree 1, coarse degree 2, interval ratio 30) are the
                           fastest measured on the 128x64x64 cantilever in both precisions. */
  int device_loop;      /* 1: the CG loop runs on the device (one CUDA graph per solve with a
                           conditional WHILE node); 0: the host replays a one-iteration graph and
                           polls the stop flag (profilers see the loop's kernels only then) */
  int deep_sweeps;      /* smoother degree on levels >= 2; 0: as coarse_sweeps.  Default 4: the
                           deep levels are small and latency-bound, so more smoothing there costs
                           little and saves CG iterations (measured on the 128x64x64 cantilever) */
  int pdl;              /* programmatic dependent launch in the CG loop (each kernel's launch overlaps
                           the tail of the one before it), a mask: 1 the coarse levels' kernels,
                           2 the fine operator and fine-level vector kernels, 3 both, 0 plain stream
                           order.  Turned off by itself when a CUDA graph cannot be built with it. */
  int coarse_bf16;      /* mixed form: levels 1 .. coarse_bf16 (default 99: every level but the
                           dense coarsest) store their packed stencils in bf16 (symmetrized, FP32
                           arithmetic), halving the bytes each smoothing step there reads; 0 all
                           FP32.  The preconditioner only: the CG operator and the
                           FP64 residuals are unchanged, so the stopping test is too.  Used with
                           the Chebyshev smoother, whose interval is measured on the operator it
                           smooths (damped Jacobi's fixed omega has no margin for the rounding). */
  int split_dofs;       /* packed-layout coarse levels (the FP64 form, FP32 levels, bf16 levels with
                           coarse_node_major = 0) with at most this many DOFs apply their stencil with
                           four threads per DOF (more loads in flight on levels too small to fill the
                           GPU); larger levels one thread per DOF */
  int deep_cta;         /* mixed form, 1 (default): the last smoothed level and the coarsest solve run
                           as one thread block with the level's operator in shared memory (when it
                           fits), instead of one launch per smoothing step and grid transfer */
  int block_sweeps;     /* smoother degree on the level run as one block (deep_cta); 0: as the
                           other levels >= 2 (deep_sweeps) */
  int resid_restrict_dofs; /* coarse levels with at most this many DOFs compute their residual inside
                           the restriction kernel (one launch instead of two, each fine residual
                           computed by up to 8 coarse nodes).  Default 0 (off): at 128x64x64 the
                           two launches are faster (measured 0.4% per SIMP iteration mixed, 0.7%
                           FP64) */
  int spectra_streams;  /* 1 (default): each level's power iteration at set-up on its own stream, as
                           soon as the level is built; 0: all of them in order on the solver's stream */
  int cluster_cycle;    /* mixed form, 1 (default): the two last smoothed levels and the coarsest solve
                           run as one thread-block cluster of 8 (or 16) CTAs, each level's bf16
                           stencil split over the CTAs' shared memory and the halos exchanged through
                           distributed shared memory, when both levels hold bf16 stencils and the
                           cluster fits; 0: the last smoothed level as one block (deep_cta) and the
                           one before it one launch per smoothing step and transfer */
  int fine_slab_depth;  /* Walsh-Hadamard fine operator: node planes per block along z; 0 (default)
                           the fastest of the tile model's depth, half of it and twice it, timed with
                           the launch shapes; > 0 that depth only (profiling, reproducible tiles) */
  int coarse_node_major; /* mixed form, 1 (default): the bf16 coarse levels apply their stencil from a
                           node-major copy (three lanes per node, one per z-plane of neighbours,
                           16-byte coefficient loads, each neighbour's u loaded once per node);
                           0: the packed layout (split_dofs decides between one thread and four
                           lanes per DOF) */
  int ritz_start;       /* 1 (default): keep the buffers of tp3d_solver_ritz_start, and start each
                           solve of a stage graph from the Rayleigh-Ritz combination of the last two
                           solutions; 0: the linear extrapolation of tp3d_warm_start */
  double cheb_ratio_coarse; /* Chebyshev interval ratio of the coarse levels (> 1; 0, the default: the
                           fine level's cheb_ratio).  110 measured 7.43 against 7.87 ms per mixed
                           SIMP step at 128x64x64 (18.85 against 20.4 CG iterations), but an FP64
                           solve of a random design with 1e-9 voids then stopped at its residual
                           floor 1.2e-7, so it is opt-in */
} tp3d_solver_opts;

void tp3d_solver_default_opts(tp3d_solver_opts* opts);

/* Create a solver for a (nelx, nely, nelz) grid.  KE_host: 24x24 row-major
 * host array (lk_H8, pytopo3d/utils/stiffness.py:12-130).  fixed_dofs: device
 * uint8 per DOF (the complement of build_supports' freedofs,
 * pytopo3d/utils/assembly.py:224-348). */
int tp3d_solver_create(int nelx, int nely, int nelz, const double* KE_host,
                       const uint8_t* fixed_dofs, const tp3d_solver_opts* opts, void* stream,
                       tp3d_solver** out);
int tp3d_solver_destroy(tp3d_solver* s);

/* Set the SIMP moduli E = Emin + (1-Emin) rho^penal (optimizer.py:584-586) and
 * rebuild the multigrid hierarchy.  rho_physical: device, nele doubles. */
int tp3d_solver_set_density(tp3d_solver* s, const double* rho_physical, double penal);

/* Solve K(rho) U = F on the free DOFs; fixed DOFs of U are set to 0.
 * U holds the initial guess on entry.  Replaces the assembly + solver_func
 * call (optimizer.py:584-594, pytopo3d/utils/solver.py:43-73).
 * iterations / relres: host out-params (may be NULL). */
int tp3d_solver_solve(tp3d_solver* s, const double* F, double* U, int* iterations,
                      double* relres);

/* y = K u with fixed rows/cols replaced by identity (FP64 / FP32 forms). */
/* tp3d_solver_solve in two halves, so that a caller can queue work that reads U
 * (sensitivities) before the host waits for the solve.  _begin queues the solve
 * (the mixed form: its FP32 iteration and FP64 result; the FP64 form solves
 * completely here) and returns at once; U holds the result in stream order.
 * _end waits, reads the iteration count and residual, and returns the status
 * tp3d_solver_solve would have returned.  When the mixed form had to finish
 * the system with the FP64 solver, that solve runs in _end after the work the
 * caller queued since _begin, overwrites U and sets *replaced = 1: the caller
 * then repeats its work that read U.  No other solver call may come between
 * the two halves. */
int tp3d_solver_solve_begin(tp3d_solver* s, const double* F, double* U);
int tp3d_solver_solve_end(tp3d_solver* s, int* iterations, double* relres, int* replaced);

/* Initial guess of the next solve from the last two solutions of the same load
 * case, for the operator of the current density (call after set_density): U <-
 * a U + b U_prev with (a, b) minimising the energy x'Kx / 2 - F'x over span{U,
 * U_prev} (a 2x2 Galerkin system on the device: two FP64 operator applies and
 * one fused reduction), U_prev <- the old U.  With have_prev = 0 only U_prev is
 * updated.  The span holds the linear extrapolation 2 U - U_prev of
 * tp3d_warm_start, so the start is at least as close in the energy norm; on the
 * 128x64x64 workload it saves 1-3 CG iterations per solve.  Replaces the
 * reference's cold spsolve (pytopo3d/core/optimizer.py:592), which has no
 * initial guess.  F, U, U_prev: device FP64 vectors of the grid's 3 x nodes
 * DOFs (fixed DOFs of U and U_prev zero, as the solves leave them); queued on
 * the solver's stream after the caller's stream.  Needs a solver created with
 * ritz_start = 1. */
int tp3d_solver_ritz_start(tp3d_solver* s, const double* F, double* U, double* U_prev, int have_prev);
int tp3d_solver_apply_f64(tp3d_solver* s, const double* u, double* y);
int tp3d_solver_apply_f32(tp3d_solver* s, const float* u, float* y);
/* Coarse level `level` (1 .. levels - 2) of the mixed form's multigrid applied as
 * the V-cycle applies it (bf16 or FP32 stencil, packed or node-major): y = A u on
 * the level's free DOFs, y = u on its fixed DOFs; u, y: device FP32 vectors of
 * 3 x the level's nodes.  Test helper for the coarse-level kernels; the
 * reference's direct solve has no multigrid levels. */
int tp3d_solver_apply_level_f32(tp3d_solver* s, int level, const float* u, float* y);

/* Average device time (ms) of the fine-level operator kernel over `launches`
 * back-to-back launches on the solver's stream, timed with one pair of CUDA
 * events, the launches rotating over input/output vectors that together exceed
 * twice L2 so that each reads its input from HBM (fp32 != 0: the mixed form's
 * FP32 kernel).  Measurement helper for the roofline figure; no reference
 * counterpart. */
int tp3d_solver_time_apply(tp3d_solver* s, int fp32, int launches, double* ms_per_launch);

/* Autotuner of the smoothing degrees: a coordinate search from the current setting over the
 * deeper levels' Chebyshev degree (2, 4, 6), then level 1's (1, 2, 3), then the fine level's
 * (1, 2).  A candidate's cost is its solve of K U = F from the initial guess U0 (device, not
 * modified): criterion 0 (latency: one design alone on the GPU) the faster of two solves timed
 * on the host clock after a first one that captures the iteration graph; criterion 1
 * (throughput: designs sharing the GPU) the solve's algorithmic bytes, CG iterations times the
 * bytes of one iteration.  The cheapest candidate that converged (without the mixed form's FP64
 * fallback) becomes the solver's setting.  Call it on a representative design and warm start
 * (the SIMP loop does so at an iteration of the caller's choice).  The choice is cached per
 * process for the grid, precision and criterion: a later call applies it without solving.  (The
 * fine operator's launch shape and slab depth are chosen by timing at the first set_density and
 * cached the same way.)  report (host, up to 10 doubles): fine, level-1 and deeper degrees
 * chosen, best and starting-setting cost (ms for criterion 0, GB for criterion 1), candidates
 * tried, 1 when taken from the cache, the criterion, the CG iterations and bytes per iteration of
 * the last candidate solved.  No reference counterpart. */
int tp3d_solver_autotune(tp3d_solver* s, const double* F, const double* U0, int criterion, double* report,
                         int nreport);

/* Average device time (ms) of one Apply-mode launch of the level-`level` operator (0: the fine
 * operator; >= 1: the coarse packed-stencil kernel of the V-cycle; the coarsest dense level is
 * excluded), each launch timed alone with its own CUDA events after a 256 MiB write that evicts
 * L2, so it reads its operator and vectors from HBM; *bytes_per_launch receives its algorithmic
 * bytes (vectors in and out, stencil or moduli, fixed-DOF mask).  fp32 != 0: the mixed form's
 * kernels.  Measurement helper for the roofline figures; no reference counterpart. */
int tp3d_solver_time_level(tp3d_solver* s, int level, int fp32, int launches, double* ms_per_launch,
                           double* bytes_per_launch);

/* Diagnostics of the last solve, in this order: levels, CG iterations, reliable updates
 * (mixed), relres, restarts (FP64), coarsest dense size, dense-form tile (y, x, z chunk),
 * coarsest-inverse fallback flag, lambda_max(Dinv A) of the fine level, residual-floor flag,
 * FP64-fallback flag (mixed), fine form of the FP64 operator and of the FP32 operator
 * (0 dense, 1 + shape for the Walsh-Hadamard form, -1 absent), first level of the fused
 * coarse cycle (0 none), 1 when the CG loop runs on the device (one graph launch per
 * solve) rather than host-polled, the programmatic-dependent-launch mask in use (0 none),
 * the number of levels whose stencils are held in bf16, the coarsest inverse's status (0 first
 * attempt, 1-3 attempts with a raised diagonal, 4 diagonal fallback), the level run as one block
 * with the coarsest solve (0 none), the algorithmic bytes of one CG iteration (every array each
 * kernel of the iteration must read or write once, summed over the iteration's kernels; the
 * reliable-update branch excluded; 0 before the first solve), the kernels launched per CG
 * iteration, the autotuner state (0 not tuned, 1 searched, 2 from the cache), the smoothing degrees
 * of the fine level, level 1 and level 2, the fine operator's slab depth (node planes per block; 0
 * for the dense form) and threads per block of the Walsh-Hadamard form in use, the first level of
 * the cluster cycle (0 none) and its CTAs, and the Walsh-Hadamard form's interior tile (nodes along
 * y, nodes along x; 0 for the dense form).  Returns the count written. */
int tp3d_solver_stats(tp3d_solver* s, double* out, int n);

/* ---------------------------------------------------------------------------
 * A projection stage of the SIMP loop as one CUDA graph
 * ------------------------------------------------------------------------- */

/* The loop body of top3d (pytopo3d/core/optimizer.py:578-696: moduli, solves,
 * sensitivities, OC update, change, re-projection) captured once per projection
 * stage into the body of a device-side WHILE loop whose condition is decided on
 * the device: continue while change > tolx and the stage's iteration limit is
 * not reached (optimizer.py:578).  Each solve's CG loop is a nested WHILE node
 * (the FP64 form's restart loop one more).  One launch runs the stage; the host
 * reads the per-iteration record once.  Where the host path would have decided
 * differently inside a solve (the mixed form's FP64 fallback, an FP64 solve the
 * host path reports as failed) the pass raises counters[1], skips the rest of
 * the iteration and ends the loop, with each case's warm-started initial guess
 * in U_bak: the caller runs that iteration on the host path from U_bak (without
 * a new set-up) and launches the graph again.
 * All arrays are device arrays the caller owns and keeps at the same addresses
 * for the graph's life; x is updated in place (x_new is the OC output).
 * counters (5 ints, written by the caller before each launch): [0] iteration of
 * the launch (0), [1] abort flag (0), [2] CG iterations of the running
 * iteration (0), [3] iteration limit of the launch, [4] solves of the loop done
 * before the launch (the warm start's history test).  record: limit x 8
 * doubles per iteration: compliance, lambda, projected free volume, bisection
 * steps, change, CG iterations, lambda bracket (lo, hi).  The solver must have
 * run one loop body (set_density and a solve) on the host path before capture.
 * No reference counterpart beyond the loop body itself. */
typedef struct tp3d_stage tp3d_stage;
typedef struct tp3d_stage_desc {
  int ncases;                 /* load cases; F, U, U_prev, U_bak are ncases x ndof */
  double rmin, beta, eta, penal, move, target_free_volume, tolx;
  int max_bisection;
  double bisection_tol;
  const double* F;
  double *U, *U_prev, *U_bak;
  double *x, *x_new, *rho_f, *rho_p, *dproj, *rho_new;
  double *dc_dx, *dc_acc, *dv_dx, *ce;
  double* c;                  /* 2 doubles: compliance (and a case's share) */
  const double* Hs;
  const uint8_t *solid, *void_, *free_mask;
  const double* KE_host;      /* 24x24 row-major, host */
  void *sens_scratch, *oc_scratch;
  double* oc_stats;           /* 8 doubles (tp3d_oc_update's stats) */
  double* record;
  int* counters;
} tp3d_stage_desc;
int tp3d_stage_capture(tp3d_solver* s, const tp3d_stage_desc* d, void* stream, tp3d_stage** out);
/* Launch on `stream`, wait, and return the iterations completed and the abort flag. */
int tp3d_stage_run(tp3d_stage* g, void* stream, int* iterations, int* aborted);
/* Add a run's kernel launches (passes of the loop body, CG iterations) to tp3d_launch_count. */
int tp3d_stage_count_launches(tp3d_stage* g, long long passes, long long cg_iterations);
int tp3d_stage_destroy(tp3d_stage* g);

/* Many designs in one graph launch: each design's loop body, as in the stage
 * graph (its own solver, descriptor and buffers; counters and record per
 * design), in a WHILE node of its own, the n loops parallel branches of one
 * graph.  One launch advances every design by up to its counters' iteration
 * limit (tolx < 0: exactly that many unless a solve is handed back); the
 * designs share nothing but the GPU, whose scheduler overlaps their kernels as
 * the branches allow.  The reference runs designs one after another
 * (pytopo3d/runners/experiment.py); this has no counterpart there beyond the
 * loop body. */
typedef struct tp3d_batch tp3d_batch;
int tp3d_batch_capture(tp3d_solver* const* solvers, const tp3d_stage_desc* descs, int n, void* stream,
                       tp3d_batch** out);
/* Launch on `stream` and wait; the caller reads each design's counters. */
int tp3d_batch_run(tp3d_batch* b, void* stream);
/* Add a run's kernel launches (per design: passes of the loop body, CG iterations) to tp3d_launch_count. */
int tp3d_batch_count_launches(tp3d_batch* b, const long long* passes, const long long* cg_iterations);
int tp3d_batch_destroy(tp3d_batch* b);

/* Initial guess for the next solve of a load case from its last two solutions:
 * U <- 2 U - U_prev and U_prev <- (old) U; with have_prev == 0 only U_prev <- U.
 * Device arrays of n doubles.  The reference solves from scratch every
 * iteration (optimizer.py:584-594); an iterative solve converges from any
 * guess, and on the 128x64x64 cantilever this one saves about 5% of the CG
 * iterations over starting from the last solution. */
int tp3d_warm_start(double* U, double* U_prev, long long n, int have_prev, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TOPO3D_B200_H */
