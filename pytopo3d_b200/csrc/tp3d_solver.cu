// Multigrid-preconditioned CG on the matrix-free H8 operator.
//
// Replaces, per SIMP iteration, the reference's
//   K = assemble(kron(E, KE)); Kff = K[free][:, free]; Uf = solver_func(Kff, F[free])
// (pytopo3d/core/optimizer.py:584-594; pytopo3d/utils/solver.py:15-73).
//
// Two forms:
//  * FP64: CG with an FP64 V-cycle; the recursive residual is checked against
//    the true residual at the end and CG restarts from it if they drifted apart.
//  * mixed: CG whose operator, V-cycle and vectors are FP32 (fine operator from
//    FP32 moduli or BF16 densities), with FP64 "reliable updates": whenever the
//    FP32 residual has fallen by `reliable_delta`, the FP32 iterate is added to
//    the FP64 solution, the FP64 residual f - K u is recomputed and replaces the
//    FP32 one.  The search direction is kept, so the Krylov space is not
//    restarted; convergence is decided on the FP64 residual only.
//
// The V-cycle smooths with Chebyshev polynomials in Dinv A whose interval comes
// from a per-level power iteration, coarse operators are Galerkin products,
// the coarsest level is a dense inverse.  One CG iteration is captured once
// into a CUDA graph and replayed; the host polls the stop flag between replays.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "tp3d_coarse_nm.cuh"
#include "tp3d_fine.cuh"
#include "tp3d_fine_wht.cuh"
#include "tp3d_coarse.cuh"
#include "tp3d_deep.cuh"
#include "tp3d_cluster.cuh"
#include "tp3d_pcg.cuh"

namespace tp3d {

namespace {
// While a graph is being captured launches are counted into the graph's tally.
thread_local long long* t_capture_count = nullptr;
// ... and, for the CG iteration graph, each launch's algorithmic bytes (the
// arrays it must read and write once; the measure of the step-level roofline).
thread_local double* t_capture_bytes = nullptr;
}  // namespace
inline void count_launch() {
  if (t_capture_count) ++*t_capture_count;
  else add_launches(1);
}
inline void count_bytes(double b) {
  if (t_capture_bytes) *t_capture_bytes += b;
}

// Algorithmic bytes of one operator launch in mode MODE over a level with n
// DOFs and nn nodes: input and output vectors, `src` bytes of moduli or
// stencil, the fixed-DOF mask (a byte per node), and the mode's epilogue
// vectors (right-hand side, inverse diagonal, Chebyshev direction read/written).
template <typename T, int MODE>
double op_bytes(long long n, long long nn, double src) {
  const double w = (double)sizeof(T);
  double b = 2.0 * w * n + src + (double)nn;
  if (epi_reads_b<MODE>()) b += w * n;
  if (epi_reads_dinv<MODE>()) b += w * n;
  if (MODE == kModeChebStep || MODE == kModeChebStepDot) b += w * n;
  if (MODE == kModeChebFirst || MODE == kModeChebStep || MODE == kModeChebStepDot) b += w * n;
  return b;
}

constexpr int kMaxPartials = 1 << 16;
constexpr int kWhtTileCandidates = 3;  // tile shapes per Walsh-Hadamard launch shape in the timed choice
constexpr int kSpectraPartials = 4096;  // per level at set-up: two reductions of at most 2048 blocks
constexpr int kPdlCoarse = 1, kPdlFine = 2;  // tp3d_solver_opts::pdl bits

// Process-wide caches of tuning choices (fine operator form and tile; the
// smoothing degrees of the autotuner), keyed by the grid and precision.
struct FineChoiceKey {
  int nx, ny, nz, tsize, bf16, form_opt, slab_opt;
  bool operator<(const FineChoiceKey& o) const {
    return std::tie(nx, ny, nz, tsize, bf16, form_opt, slab_opt) <
           std::tie(o.nx, o.ny, o.nz, o.tsize, o.bf16, o.form_opt, o.slab_opt);
  }
};
struct FineChoice {
  bool use;
  WhtTile tile;
};
inline std::mutex& fine_choice_mu() {
  static std::mutex m;
  return m;
}
inline std::map<FineChoiceKey, FineChoice>& fine_choice_cache() {
  static std::map<FineChoiceKey, FineChoice> c;
  return c;
}
struct DegreeKey {
  int nx, ny, nz, mixed;
  bool operator<(const DegreeKey& o) const {
    return std::tie(nx, ny, nz, mixed) < std::tie(o.nx, o.ny, o.nz, o.mixed);
  }
};
struct Degrees {
  int fine, coarse, deep;
};
inline std::mutex& degree_mu() {
  static std::mutex m;
  return m;
}
inline std::map<DegreeKey, Degrees>& degree_cache() {
  static std::map<DegreeKey, Degrees> c;
  return c;
}

template <typename T>
struct LevelVec {
  T* x[2] = {nullptr, nullptr};
  T* b = nullptr;
  T* r = nullptr;
  T* d = nullptr;  // Chebyshev direction
  T* dinv = nullptr;
  T* A = nullptr;  // packed stencil for the apply kernels (levels >= 1)
};

template <typename T>
struct KrylovVec {
  T *u = nullptr, *r = nullptr, *p = nullptr, *q = nullptr;
  cudaGraphExec_t graph = nullptr;
  long long graph_kernels = 0;
  double graph_bytes = 0.0;  // algorithmic bytes of one CG iteration (reliable-update branch excluded)
  // device-side loop (conditional nodes): kernels per pass, and in the
  // reliable-update branch
  bool loop = false;
  long long branch_kernels = 0;
};

struct Tile {
  int TY = 32, TX = 8, ZC = 8, tiles_y = 1, tiles_x = 1, zchunks = 1, threads = 256, occ = 0;
};

// Launch / occupancy of the fine operator for a compile-time tile height.
template <typename T, class ESrc, bool CLS>
int fine_launch_t(const FineParams<T, ESrc>& p, int TY, dim3 grid, int threads, cudaStream_t st, bool pdl) {
  constexpr int NZT = sizeof(T) == 4 ? 2 : 1;
  switch (TY) {
#define TP3D_FINE_CASE(ty)                                                                             \
  case ty:                                                                                             \
    launch_kernel(pdl, fine_apply_kernel<T, ESrc, ty, NZT, CLS>, grid, dim3(threads),               \
                  fine_smem_bytes<T, ty, NZT>(), st, p);                                                \
    return TP3D_OK;
    TP3D_FINE_TY_LIST(TP3D_FINE_CASE)
#undef TP3D_FINE_CASE
  }
  return TP3D_ERR_ARG;
}
template <typename T, class ESrc>
int fine_launch(const FineParams<T, ESrc>& p, int TY, bool cls, dim3 grid, int threads, cudaStream_t st, bool pdl) {
  return cls ? fine_launch_t<T, ESrc, true>(p, TY, grid, threads, st, pdl)
             : fine_launch_t<T, ESrc, false>(p, TY, grid, threads, st, pdl);
}

template <typename T, class ESrc>
int fine_occupancy(int TY, int threads) {
  constexpr int NZT = sizeof(T) == 4 ? 2 : 1;
  int occ = 0;
  switch (TY) {
#define TP3D_FINE_CASE(ty)                                                                                      \
  case ty:                                                                                                      \
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fine_apply_kernel<T, ESrc, ty, NZT, true>, threads,     \
                                                  fine_smem_bytes<T, ty, NZT>());                               \
    break;
    TP3D_FINE_TY_LIST(TP3D_FINE_CASE)
#undef TP3D_FINE_CASE
  }
  return std::max(occ, 1);
}

// Class values of KE when it has the cubic-symmetry structure of kKEClassHost
// (entry = sign * class value, checked to 1e-12 of max |KE|); false otherwise.
bool ke_classes(const double* KE, double* vals) {
  double mx = 0.0;
  for (int i = 0; i < 576; ++i) mx = std::max(mx, std::fabs(KE[i]));
  bool have[kKEClasses] = {};
  for (int i = 0; i < 576; ++i) {
    const int t = kKEClassHost[i];
    if (t == 0) continue;
    const int k = std::abs(t) - 1;
    if (!have[k]) {
      vals[k] = t > 0 ? KE[i] : -KE[i];
      have[k] = true;
    }
  }
  for (int i = 0; i < 576; ++i) {
    const int t = kKEClassHost[i];
    const double rec = t == 0 ? 0.0 : (t > 0 ? vals[std::abs(t) - 1] : -vals[std::abs(t) - 1]);
    if (std::fabs(rec - KE[i]) > 1e-12 * mx) return false;
  }
  return true;
}

// Node-plane tile from the compile-time heights (TY) and a run-time width
// (TX, TY*TX <= 256) with little padding and halo waste; then the z chunk
// (a multiple of the nodes per step) that fills the resident block slots in
// whole waves at the lowest prologue cost.
template <typename T, class ESrc>
Tile choose_tile(const Grid& g, int nsm) {
  constexpr int NZT = sizeof(T) == 4 ? 2 : 1;
  const int NX = g.nx + 1, NY = g.ny + 1, NZ = g.nz + 1;
  static const int kMenu[] = {8, 13, 16, 17, 24, 32, 33, 43, 64};
  Tile best;
  double best_cost = 1e300;
  for (int TY : kMenu) {
    const int ky = (NY + TY - 1) / TY;
    for (int TX = 1; TX * TY <= 256; ++TX) {
      const int thr = ((TY * TX + 31) / 32) * 32;
      if ((TY + 2) * (TX + 2) > 2 * thr || (TY + 1) * (TX + 1) > 2 * thr) continue;
      const int kx = (NX + TX - 1) / TX;
      const double slots = (double)ky * kx * thr;
      const double halo = (double)(TY + 2) * (TX + 2) / ((double)TY * TX);
      const double cost = slots * (1.0 + 0.3 * (halo - 1.0)) * (thr < 96 ? 1.5 : 1.0);
      if (cost < best_cost) {
        best_cost = cost;
        best.TY = TY;
        best.TX = TX;
        best.tiles_y = ky;
        best.tiles_x = kx;
        best.threads = thr;
      }
    }
  }
  best.occ = fine_occupancy<T, ESrc>(best.TY, best.threads);
  const long long planes = (long long)best.tiles_y * best.tiles_x;
  // Relative throughput of an SM running L co-resident blocks (latency hiding).
  auto eff = [&](long long L) {
    const long long l = std::min<long long>(L, best.occ);
    return l <= 1 ? 1.0 : (l == 2 ? 1.5 : (l == 3 ? 1.75 : 1.9));
  };
  double best_t = 1e300;
  for (int zc = NZT; zc <= std::max(NZT, NZ + NZT); zc += NZT) {
    const long long nch = (NZ + zc - 1) / zc;
    const long long per_sm = (planes * nch + nsm - 1) / nsm;  // blocks on the busiest SM
    const double t = (double)per_sm * (zc + 2.0 * (NZT + 1)) / eff(per_sm);  // steps + synchronous prologue
    if (t < best_t - 1e-9) {
      best_t = t;
      best.ZC = zc;
      best.zchunks = (int)nch;
    }
  }
  return best;
}

}  // namespace tp3d

using namespace tp3d;

struct tp3d_solver {
  Grid g{};
  tp3d_solver_opts o{};
  cudaStream_t st = nullptr;    // the solver's own stream (graphs cannot be captured on the legacy stream)
  cudaStream_t user = nullptr;  // the caller's stream
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  int nsm = 148;
  bool mixed = false;
  KEP<double> ke64{};
  KEP<float> ke32{};
  bool ke_cls = false;              // KE has the cubic-symmetry class structure
  double kcls64[kKEClasses] = {};   // its class values
  double* KE1 = nullptr;
  double* KE2 = nullptr;       // level-2 element tables (element-wise Galerkin)
  std::vector<double*> Kel;    // element matrices of levels >= 2 (element-wise Galerkin)
  double penal = 3.0;
  bool have_density = false;

  std::vector<Grid> grids;
  std::vector<uint8_t*> fix;
  std::vector<double*> A64;   // stencils (index 0 unused)
  std::vector<double*> coef;  // Chebyshev coefficients per level (device)
  int nlev = 1;
  int cn = 0;  // coarsest dense size
  double *cdense = nullptr, *cinv64 = nullptr;
  float* cinv32 = nullptr;
  int* cstatus = nullptr;

  double* E64 = nullptr;
  float* E32 = nullptr;
  __nv_bfloat16* rho16 = nullptr;
  std::vector<double*> pv;              // per-level normalised dominant vectors (warm starts)
  bool have_spectra = false;

  std::vector<LevelVec<double>> L64;
  std::vector<LevelVec<float>> L32;
  KrylovVec<double> K64;
  KrylovVec<float> K32;
  double* u64 = nullptr;        // FP64 solution (both forms)
  double* r64 = nullptr;        // FP64 residual (mixed)
  double* F_capture = nullptr;  // the mixed graph reads F from here

  double* partials = nullptr;
  unsigned int* fin_count = nullptr;  // arrivals of the reduction in flight (last_block_finalize)
  // device-side CG loop (capture_loop)
  bool loop_ok = true, in_loop_capture = false, branch_ok = true;
  // Programmatic dependent launch (o.pdl; cleared when a graph cannot be
  // built with it).  Used only while the CG iteration is captured
  // (pdl_region), and never for the first kernel after a graph entry or a
  // conditional node (plain_next), so that every such launch follows a kernel.
  bool pdl = true, pdl_region = false, plain_next = true;
  std::vector<__nv_bfloat16*> S16;  // packed stencils in bf16 of levels 1 .. o.coarse_bf16 (mixed form), or null
  std::vector<__nv_bfloat16*> SN3;  // node-major copies of S16 (coarse_node_major levels), or null
  long long branch_count = 0;
  cudaStream_t st_branch = nullptr;   // captures the reliable-update branch
  cudaStream_t st_side = nullptr;     // the coarsest inverse, concurrent with the power iterations
  std::vector<cudaStream_t> st_pow;   // one per smoothed level: its power iteration
  std::vector<cudaEvent_t> ev_pow_in, ev_pow_out;
  cudaEvent_t ev_side_in = nullptr, ev_side_out = nullptr, ev_side_elem = nullptr;
  unsigned int* loop_passes = nullptr;
  unsigned int* loop_pass_host = nullptr;
  PcgState* state = nullptr;
  PcgState* state_host = nullptr;  // two pinned slots
  Tile tile;
  // Walsh-Hadamard form of the fine operator (used when KE allows it and the
  // timed choice at the first set_density prefers it), per precision
  bool wht_ok = false;
  WhtBlocks<double> wb64{};
  WhtBlocks<float> wb32{};
  WhtTile wt64, wt32;
  bool use_wht64 = false, use_wht32 = false;
  bool fine_chosen = false;
  // coarse end of the V-cycle as one cooperative launch from level cyc_L0
  // (0: off); grid barrier state
  int cyc_L0 = 0;
  // the last smoothed level and the coarsest solve in one block (mixed form;
  // 0 none), and that block's shared memory
  int deep_L = 0;
  size_t deep_smem = 0;
  bool deep_inv_smem = false;
  __nv_bfloat16* deep_SN = nullptr;  // its node-major bf16 stencil (bf16 levels)
  // the two last smoothed levels (clu_L and deep_L = clu_L + 1) and the
  // coarsest solve as one thread-block cluster of clu_C CTAs (mixed form; 0 none)
  int clu_L = 0, clu_C = 0;
  size_t clu_smem = 0;
  __nv_bfloat16* clu_SN = nullptr;  // level clu_L's node-major bf16 stencil
  // Rayleigh-Ritz initial guess (o.ritz_start): K U1, K U2, gate, partials, arrivals, (a, b)
  double *rz_q1 = nullptr, *rz_q2 = nullptr, *rz_part = nullptr, *rz_coef = nullptr;
  int* rz_gate = nullptr;
  unsigned int* rz_count = nullptr;
  int cyc_blocks64 = 0, cyc_blocks32 = 0;
  unsigned int* cyc_bar = nullptr;  // [barrier word, error]
  std::vector<void*> allocs;

  int last_iters = 0, last_updates = 0, last_restarts = 0;
  bool last_floor = false;
  double last_relres = 0.0;

  template <typename T>
  T* alloc(size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) p = nullptr;
    allocs.push_back(p);  // a failure is recorded too: create() checks the list
    return (T*)p;
  }
  ~tp3d_solver() {
    if (st) cudaStreamSynchronize(st);
    if (K64.graph) cudaGraphExecDestroy(K64.graph);
    if (K32.graph) cudaGraphExecDestroy(K32.graph);
    for (void* p : allocs) cudaFree(p);
    if (state_host) cudaFreeHost(state_host);
    if (loop_pass_host) cudaFreeHost(loop_pass_host);
    if (st_branch) cudaStreamDestroy(st_branch);
    if (st_loop) cudaStreamDestroy(st_loop);
    if (st_restart) cudaStreamDestroy(st_restart);
    if (st_side) cudaStreamDestroy(st_side);
    for (cudaStream_t p : st_pow) if (p) cudaStreamDestroy(p);
    for (cudaEvent_t e : ev_pow_in) if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : ev_pow_out) if (e) cudaEventDestroy(e);
    if (ev_side_in) cudaEventDestroy(ev_side_in);
    if (ev_side_out) cudaEventDestroy(ev_side_out);
    if (ev_side_elem) cudaEventDestroy(ev_side_elem);
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_out) cudaEventDestroy(ev_out);
    if (st) cudaStreamDestroy(st);
  }
  // order the solver's stream after the caller's work, and the caller's after ours
  int enter() {
    TP3D_CHECK(cudaEventRecord(ev_in, user));
    TP3D_CHECK(cudaStreamWaitEvent(st, ev_in, 0));
    return TP3D_OK;
  }
  int leave() {
    TP3D_CHECK(cudaEventRecord(ev_out, st));
    TP3D_CHECK(cudaStreamWaitEvent(user, ev_out, 0));
    return TP3D_OK;
  }

  int grid_blocks(long long n, int per = 256) const {
    return (int)std::max<long long>(1, std::min<long long>((n + per - 1) / per, (long long)nsm * 8));
  }

  template <typename T>
  std::vector<LevelVec<T>>& levels() {
    if constexpr (sizeof(T) == 8) return L64;
    else return L32;
  }

  // ---------------- operators ----------------
  // bytes per element of the fine operator's modulus source
  template <typename T>
  double fine_src_bytes() const {
    if constexpr (sizeof(T) == 8) return 8.0;
    else return rho16 ? 2.0 : 4.0;
  }
  // Rayleigh-Ritz initial guess for the next solve (ritz_gate_kernel and the
  // kernels after it): U <- a U + b U_prev minimising the energy under the
  // current operator, U_prev <- the old U.  Queued on the solver's stream, the
  // gate read on the device, so a stage graph captures the same kernels.
  int ritz_start(const double* F, double* U, double* U_prev, int have_prev, const int* ctr) {
    if (!rz_q1) return TP3D_ERR_ARG;
    const long long ndof = 3 * g.nnode();
    const int nb = grid_blocks(ndof);
    ritz_gate_kernel<<<1, 1, 0, st>>>(rz_gate, have_prev, ctr);
    count_launch();
    OpIO<double> io;
    io.u = U;
    io.out = rz_q1;
    io.gate = rz_gate;
    if (int rc = fine<double, kModeApply>(io)) return rc;
    io.u = U_prev;
    io.out = rz_q2;
    if (int rc = fine<double, kModeApply>(io)) return rc;
    ritz_dot_kernel<<<nb, 256, 0, st>>>(ndof, F, U, U_prev, rz_q1, rz_q2, rz_gate, rz_part, rz_count, rz_coef);
    ritz_combine_kernel<<<nb, 256, 0, st>>>(ndof, U, U_prev, rz_coef, rz_gate);
    count_launch();
    count_launch();
    TP3D_CHECK_LAUNCH();
    return TP3D_OK;
  }

  template <typename T, int MODE>
  int fine(const OpIO<T>& io) {
    count_bytes(op_bytes<T, MODE>(3 * g.nnode(), g.nnode(), fine_src_bytes<T>() * (double)g.nele()));
    if (use_wht<T>()) return fine_wht<T>(MODE, io);
    const dim3 grid(tile.tiles_y * tile.tiles_x, tile.zchunks);
    int rc;
    if constexpr (sizeof(T) == 8) {
      FineParams<double, EFromF64> p;
      p.ke = ke64;
      for (int k = 0; k < kKEClasses; ++k) p.kcls[k] = kcls64[k];
      p.g = g;
      p.TX = tile.TX; p.ZC = tile.ZC; p.tiles_y = tile.tiles_y; p.tiles_x = tile.tiles_x;
      p.mode = MODE;
      p.fix = fix[0];
      p.esrc = EFromF64{E64};
      p.io = io;
      rc = fine_launch(p, tile.TY, ke_cls, grid, tile.threads, st, take_pdl(kPdlFine));
    } else if (rho16) {
      FineParams<float, EFromBF16> p;
      p.ke = ke32;
      for (int k = 0; k < kKEClasses; ++k) p.kcls[k] = (float)kcls64[k];
      p.g = g;
      p.TX = tile.TX; p.ZC = tile.ZC; p.tiles_y = tile.tiles_y; p.tiles_x = tile.tiles_x;
      p.mode = MODE;
      p.fix = fix[0];
      p.esrc = EFromBF16{rho16, (float)penal};
      p.io = io;
      rc = fine_launch(p, tile.TY, ke_cls, grid, tile.threads, st, take_pdl(kPdlFine));
    } else {
      FineParams<float, EFromF32> p;
      p.ke = ke32;
      for (int k = 0; k < kKEClasses; ++k) p.kcls[k] = (float)kcls64[k];
      p.g = g;
      p.TX = tile.TX; p.ZC = tile.ZC; p.tiles_y = tile.tiles_y; p.tiles_x = tile.tiles_x;
      p.mode = MODE;
      p.fix = fix[0];
      p.esrc = EFromF32{E32};
      p.io = io;
      rc = fine_launch(p, tile.TY, ke_cls, grid, tile.threads, st, take_pdl(kPdlFine));
    }
    if (rc) return rc;
    count_launch();
    TP3D_CHECK_LAUNCH();
    return TP3D_OK;
  }
  template <typename T>
  bool use_wht() const {
    if constexpr (sizeof(T) == 8) return use_wht64;
    else return use_wht32;
  }
  template <typename T>
  const WhtTile& wtile() const {
    if constexpr (sizeof(T) == 8) return wt64;
    else return wt32;
  }
  // Whether the next loop kernel is launched with the programmatic-serialization
  // attribute; consumes plain_next.
  // cls: kPdlCoarse for kernels over a coarse level, kPdlFine for the fine
  // operator and the fine-level vector kernels (o.pdl is a mask of the two).
  bool take_pdl(int cls) {
    const bool on = (o.pdl & cls) && pdl && pdl_region && !plain_next;
    plain_next = false;
    return on;
  }
  // A loop kernel (it begins with pdl_entry()); errors surface through
  // cudaGetLastError like a <<<>>> launch.
  template <typename... P, typename... A>
  void launch(int cls, void (*k)(P...), dim3 grid, dim3 block, size_t smem, A&&... args) {
    launch_kernel(take_pdl(cls), k, grid, block, smem, st, static_cast<A&&>(args)...);
    count_launch();
  }
  template <typename T, class ESrc>
  int wht_launch_with(int mode, const OpIO<T>& io, const WhtTile& w, ESrc esrc) {
    WhtParams<T, ESrc> p;
    if constexpr (sizeof(T) == 8) p.mb = wb64;
    else p.mb = wb32;
    p.g = g;
    p.TX = w.TX; p.TY = w.TY; p.PY = w.PY; p.ZC = w.ZC;
    p.tiles_y = w.tiles_y; p.tiles_x = w.tiles_x;
    p.fix = fix[0];
    p.esrc = esrc;
    p.io = io;
    return wht_launch<T, ESrc>(p, mode, w.variant, dim3(w.tiles_y * w.tiles_x, w.zchunks), st, take_pdl(kPdlFine));
  }
  template <typename T>
  int fine_wht_tile(int mode, const OpIO<T>& io, const WhtTile& w) {
    int rc;
    if constexpr (sizeof(T) == 8) rc = wht_launch_with<double>(mode, io, w, EFromF64{E64});
    else if (rho16) rc = wht_launch_with<float>(mode, io, w, EFromBF16{rho16, (float)penal});
    else rc = wht_launch_with<float>(mode, io, w, EFromF32{E32});
    if (rc) {
      tp3d_set_last_error("fine operator launch failed");
      return rc;
    }
    count_launch();
    TP3D_CHECK_LAUNCH();
    return TP3D_OK;
  }
  template <typename T>
  int fine_wht(int mode, const OpIO<T>& io) {
    return fine_wht_tile<T>(mode, io, wtile<T>());
  }
  // Average time of `launches` back-to-back Apply-mode launches of the fine
  // operator (current form) rotating over input/output vector pairs that
  // together exceed twice L2 (at most 64 pairs), so each launch reads cold
  // inputs; one warm-up pass over all pairs first, events on the solver's
  // stream.  The vectors are allocated for the measurement and freed after it.
  template <typename T>
  int time_fine_cold(int launches, double* ms_out) {
    constexpr size_t kColdBytes = (size_t)256 << 20;
    const long long ndof = 3 * g.nnode();
    const size_t pair_bytes = (size_t)ndof * sizeof(T) * 2;
    const int npairs =
        (int)std::min<size_t>(64, std::max<size_t>(2, (kColdBytes + pair_bytes - 1) / pair_bytes));
    unsigned char* buf = nullptr;
    if (cudaMalloc(&buf, (size_t)npairs * pair_bytes) != cudaSuccess) {
      tp3d_set_last_error("timing buffers: allocation failed");
      return TP3D_ERR_CUDA;
    }
    struct Free {
      unsigned char* p;
      ~Free() { cudaFree(p); }
    } guard{buf};
    TP3D_CHECK(cudaMemsetAsync(buf, 0, (size_t)npairs * pair_bytes, st));
    auto launch = [&](int k) -> int {
      unsigned char* base = buf + (size_t)(k % npairs) * pair_bytes;
      OpIO<T> io;
      io.u = (const T*)base;
      io.out = (T*)base + ndof;
      return fine<T, kModeApply>(io);
    };
    int rc = TP3D_OK;
    for (int k = 0; k < npairs && rc == TP3D_OK; ++k) rc = launch(k);
    cudaEvent_t a, b;
    TP3D_CHECK(cudaEventCreate(&a));
    TP3D_CHECK(cudaEventCreate(&b));
    TP3D_CHECK(cudaEventRecord(a, st));
    for (int k = 0; k < launches && rc == TP3D_OK; ++k) rc = launch(k);
    TP3D_CHECK(cudaEventRecord(b, st));
    TP3D_CHECK(cudaEventSynchronize(b));
    float ms = 0.f;
    TP3D_CHECK(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ms_out = ms / launches;
    return rc;
  }

  // Average device time of `launches` Apply-mode launches of the level-L
  // operator (L >= 1: the packed-stencil kernel of the V-cycle; L = 0: the fine
  // operator), each timed alone with its own event pair after a 256 MiB memset
  // that evicts L2, so every launch reads its stencil and vectors from HBM.
  // *bytes_out: the launch's algorithmic bytes (op_bytes).
  template <typename T>
  int time_level_cold(int L, int launches, double* ms_out, double* bytes_out) {
    constexpr size_t kFlushBytes = (size_t)256 << 20;
    auto& lv = levels<T>()[L];
    if (!lv.x[0] || !lv.x[1]) return TP3D_ERR_ARG;
    const long long nn = grids[L].nnode(), n = 3 * nn;
    const double src = L == 0 ? fine_src_bytes<T>() * (double)g.nele() : 81.0 * stencil_bytes<T>(L) * (double)n;
    *bytes_out = op_bytes<T, kModeApply>(n, nn, src);
    unsigned char* flush = nullptr;
    if (cudaMalloc(&flush, kFlushBytes) != cudaSuccess) {
      tp3d_set_last_error("timing buffers: allocation failed");
      return TP3D_ERR_CUDA;
    }
    struct Free {
      unsigned char* p;
      ~Free() { cudaFree(p); }
    } guard{flush};
    cudaEvent_t a, b;
    TP3D_CHECK(cudaEventCreate(&a));
    TP3D_CHECK(cudaEventCreate(&b));
    OpIO<T> io;
    io.u = lv.x[0];
    io.out = lv.x[1];
    int rc = apply_level<T, kModeApply>(L, io);  // warm-up (instruction cache, first-launch costs)
    double total = 0.0;
    for (int k = 0; k < launches && rc == TP3D_OK; ++k) {
      if (cudaMemsetAsync(flush, k & 0xff, kFlushBytes, st) != cudaSuccess) rc = TP3D_ERR_CUDA;
      if (rc == TP3D_OK && cudaEventRecord(a, st) != cudaSuccess) rc = TP3D_ERR_CUDA;
      if (rc == TP3D_OK) rc = apply_level<T, kModeApply>(L, io);
      if (rc == TP3D_OK && cudaEventRecord(b, st) != cudaSuccess) rc = TP3D_ERR_CUDA;
      float ms = 0.f;
      if (rc == TP3D_OK && (cudaEventSynchronize(b) != cudaSuccess || cudaEventElapsedTime(&ms, a, b) != cudaSuccess))
        rc = TP3D_ERR_CUDA;
      total += ms;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ms_out = total / launches;
    return rc;
  }

  // Fine operator form for precision T: the dense-KE kernel or one of the
  // Walsh-Hadamard launch shapes, whichever runs the Apply mode fastest on this
  // grid with cold inputs (time_fine_cold, 8 launches each).  For each shape
  // (threads per block, hence the node patch and elements per block) the slab
  // depth (node planes per block along z) is searched too: the tile model's
  // choice, half of it and twice it.  fine_operator = 1 / 2 restricts the
  // choice to one form, 3..5 to one shape.  The choice is cached per process
  // for the grid, precision and modulus source, so later solvers of the same
  // grid skip the timing.
  template <typename T>
  WhtTile wht_tile_for(int v) const {
    if constexpr (sizeof(T) == 8) return wht_choose_tile<double, EFromF64>(g, nsm, v);
    else if (rho16) return wht_choose_tile<float, EFromBF16>(g, nsm, v);
    else return wht_choose_tile<float, EFromF32>(g, nsm, v);
  }
  template <typename T>
  int wht_tiles_for(int v, WhtTile* out, int max_out) const {
    if constexpr (sizeof(T) == 8) return wht_tile_candidates<double, EFromF64>(g, nsm, v, out, max_out);
    else if (rho16) return wht_tile_candidates<float, EFromBF16>(g, nsm, v, out, max_out);
    else return wht_tile_candidates<float, EFromF32>(g, nsm, v, out, max_out);
  }
  template <typename T>
  int choose_fine_form() {
    bool& use = sizeof(T) == 8 ? use_wht64 : use_wht32;
    WhtTile& wt = sizeof(T) == 8 ? wt64 : wt32;
    use = false;
    if (!wht_ok) return TP3D_OK;
    const FineChoiceKey key{g.nx, g.ny, g.nz, (int)sizeof(T), rho16 ? 1 : 0, o.fine_operator, o.fine_slab_depth};
    {
      std::lock_guard<std::mutex> lk(fine_choice_mu());
      auto it = fine_choice_cache().find(key);
      if (it != fine_choice_cache().end()) {
        use = it->second.use;
        wt = it->second.tile;
        return TP3D_OK;
      }
    }
    auto time_one = [&](double* ms) -> int { return time_fine_cold<T>(8, ms); };
    double best = 1e300;
    WhtTile best_t;
    bool best_wht = false;
    int rc = TP3D_OK;
    if (o.fine_operator == 0) rc = time_one(&best);  // dense form
    const int NZ = g.nz + 1;
    int nvar;
    if constexpr (sizeof(T) == 8) nvar = wht_variant_count<double, EFromF64>();
    else nvar = wht_variant_count<float, EFromF32>();
    for (int v = 0; v < nvar && rc == TP3D_OK; ++v) {
      if (o.fine_operator > 2 && v != o.fine_operator - 3) continue;
      // the packed FP32 shapes are taken only when asked for by name: on B200
      // they measured slower than the scalar ones (150 registers per thread, a
      // quarter of the resident warps), so the timed choice skips them
      bool timed;
      if constexpr (sizeof(T) == 8) timed = wht_variant_timed<double, EFromF64>(v);
      else timed = wht_variant_timed<float, EFromF32>(v);
      if (o.fine_operator <= 2 && !timed) continue;
      // the tile shapes with the fewest blocks per node plane (elements per
      // block), each at its modelled slab depth, half and twice it
      WhtTile tiles[kWhtTileCandidates];
      const int ntile = wht_tiles_for<T>(v, tiles, kWhtTileCandidates);
      for (int ti = 0; ti < ntile && rc == TP3D_OK; ++ti) {
        const WhtTile& base = tiles[ti];
        int zcs[3] = {base.ZC, std::max(1, base.ZC / 2), std::min(NZ, 2 * base.ZC)};
        const int nzc = o.fine_slab_depth > 0 ? 1 : 3;
        if (o.fine_slab_depth > 0) zcs[0] = std::min(NZ, o.fine_slab_depth);
        for (int k = 0; k < nzc && rc == TP3D_OK; ++k) {
          if (k > 0 && (zcs[k] == base.ZC || (k == 2 && zcs[2] == zcs[1]))) continue;
          WhtTile w = base;
          w.ZC = zcs[k];
          w.zchunks = (NZ + w.ZC - 1) / w.ZC;
          if ((long long)w.tiles_y * w.tiles_x * w.zchunks > kMaxPartials) continue;
          wt = w;
          use = true;
          double ms = 0.0;
          rc = time_one(&ms);
          use = false;
          if (rc == TP3D_OK && ms < best) {
            best = ms;
            best_t = w;
            best_wht = true;
          }
        }
      }
    }
    if (rc) return rc;
    if (best_wht) {
      wt = best_t;
      use = true;
    }
    std::lock_guard<std::mutex> lk(fine_choice_mu());
    fine_choice_cache()[key] = FineChoice{use, wt};
    return TP3D_OK;
  }

  // ---------------- autotuning of the smoothing degrees ----------------
  // Drop the CG iteration graphs: the next solve captures them again with the
  // current options (the smoothing degrees are read at capture).
  void drop_graphs() {
    for (auto* K : {&K64.graph, &K32.graph})
      if (*K) {
        cudaGraphExecDestroy(*K);
        *K = nullptr;
      }
    K64.loop = K32.loop = false;
  }
  int tuned = 0;  // 0 not tuned, 1 searched here, 2 taken from the cache

  template <typename T, int MODE>
  int apply_level(int L, const OpIO<T>& io) {
    if (L == 0) return fine<T, MODE>(io);
    const long long ndof = 3 * grids[L].nnode();
    const bool split = ndof <= o.split_dofs;  // four lanes per DOF on the small levels
    count_bytes(op_bytes<T, MODE>(ndof, grids[L].nnode(), 81.0 * stencil_bytes<T>(L) * (double)ndof));
    if constexpr (sizeof(T) == 4) {
      if (L < (int)SN3.size() && SN3[L]) {
        StencilParams<float, __nv_bfloat16> p;
        p.g = grids[L];
        p.S = SN3[L];
        p.fix = fix[L];
        p.io = io;
        const long long nn = grids[L].nnode();
        launch(kPdlCoarse, nm3_apply_kernel<float, MODE>, dim3(grid_blocks((nn + 9) / 10, 8)), dim3(256), 0, p);
        TP3D_CHECK_LAUNCH();
        return TP3D_OK;
      }
      if (L < (int)S16.size() && S16[L]) {
        StencilParams<float, __nv_bfloat16> p;
        p.g = grids[L];
        p.S = S16[L];
        p.fix = fix[L];
        p.io = io;
        if (split)
          launch(kPdlCoarse, stencil_apply4_kernel<float, MODE, __nv_bfloat16>, dim3(grid_blocks(4 * ndof)),
                 dim3(256), 0, p);
        else
          launch(kPdlCoarse, stencil_apply_kernel<float, MODE, __nv_bfloat16>, dim3(grid_blocks(ndof)), dim3(256), 0,
                 p);
        TP3D_CHECK_LAUNCH();
        return TP3D_OK;
      }
    }
    StencilParams<T> p;
    p.g = grids[L];
    p.S = levels<T>()[L].A;
    p.fix = fix[L];
    p.io = io;
    if (split) launch(kPdlCoarse, stencil_apply4_kernel<T, MODE>, dim3(grid_blocks(4 * ndof)), dim3(256), 0, p);
    else launch(kPdlCoarse, stencil_apply_kernel<T, MODE>, dim3(grid_blocks(ndof)), dim3(256), 0, p);
    TP3D_CHECK_LAUNCH();
    return TP3D_OK;
  }

  // bytes per stencil coefficient of level L >= 1 in precision T's cycle
  template <typename T>
  double stencil_bytes(int L) const {
    if constexpr (sizeof(T) == 4)
      if (L < (int)S16.size() && S16[L]) return 2.0;
    return (double)sizeof(T);
  }

  // ---------------- V-cycle ----------------
  template <typename T>
  // dot_op >= 0: the last step is a Chebyshev step that also reduces b . out
  // and applies finalize op dot_op (the caller checked it applies).
  int smooth_steps(int L, int first_step, int nsteps, int* cur, const T* b, const int* done, int dot_op = -1) {
    auto& lv = levels<T>()[L];
    int rc = TP3D_OK;
    for (int s = first_step; s < first_step + nsteps; ++s) {
      OpIO<T> io;
      io.u = lv.x[*cur];
      io.out = lv.x[1 - *cur];
      io.b = b;
      io.dinv = lv.dinv;
      io.d = lv.d;
      io.coef = coef[L];
      io.step = s;
      io.omega = (T)o.omega;
      io.done = done;
      if (dot_op >= 0 && s == first_step + nsteps - 1) {
        io.partials = partials;
        io.fin = state;
        io.fin_op = dot_op;
        io.fin_count = fin_count;
        rc |= apply_level<T, kModeChebStepDot>(L, io);
      } else if (o.smoother == 1) {
        rc |= apply_level<T, kModeJacobi>(L, io);
      } else if (s == 0) {
        rc |= apply_level<T, kModeChebFirst>(L, io);
      } else {
        rc |= apply_level<T, kModeChebStep>(L, io);
      }
      *cur = 1 - *cur;
    }
    return rc;
  }

  // Levels L .. nlev-1 of the V-cycle in one cooperative launch (rhs b on
  // level L); returns the buffer holding level L's iterate.
  template <typename T>
  T* coarse_cycle(int L, const T* b, int* rc) {
    auto& lvs = levels<T>();
    CycleParams<T> p;
    for (int k = L; k < nlev; ++k) {
      CycleLevel<T>& c = p.lv[k];
      c.g = grids[k];
      c.S = lvs[k].A;
      c.fix = fix[k];
      c.dinv = lvs[k].dinv;
      c.coef = coef[k];
      c.x[0] = lvs[k].x[0];
      c.x[1] = lvs[k].x[1];
      c.b = lvs[k].b;
      c.r = lvs[k].r;
      c.d = lvs[k].d;
    }
    p.lv[L].b = const_cast<T*>(b);
    p.L0 = L;
    p.Lc = nlev - 1;
    p.pre = pre_sweeps(L);
    p.post = post_sweeps(L);
    p.cheb = o.smoother != 1 ? 1 : 0;
    p.omega = (T)o.omega;
    p.cn = cn;
    if constexpr (sizeof(T) == 8) p.inv = cinv64;
    else p.inv = cinv32;
    p.done = &state->done;
    p.bar = cyc_bar;
    p.bar_err = (int*)(cyc_bar + 1);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(sizeof(T) == 8 ? cyc_blocks64 : cyc_blocks32));
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    for (int k = L; k < nlev; ++k) {
      const double n = 3.0 * grids[k].nnode();
      count_bytes(81.0 * stencil_bytes<T>(k) * n + 5.0 * sizeof(T) * n);
    }
    if (cudaLaunchKernelEx(&cfg, coarse_cycle_kernel<T>, p) != cudaSuccess) *rc = TP3D_ERR_CUDA;
    count_launch();
    return L == nlev - 1 ? lvs[L].x[0] : lvs[L].x[cycle_final_buffer(pre_sweeps(L), post_sweeps(L))];
  }

  // Cooperative grid for the coarse cycle from level L: enough blocks for
  // one DOF per thread on level L, at most what can be co-resident.
  template <typename T>
  int cycle_blocks(int L) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, coarse_cycle_kernel<T>, 256, 0) != cudaSuccess ||
        occ < 1)
      return 0;
    const long long need = (3 * grids[L].nnode() + 255) / 256;
    return (int)std::max<long long>(1, std::min<long long>(need, (long long)occ * nsm));
  }

  // The first smoothing step of level L from zero, for kernels that compute it
  // alongside the right-hand side (none when there is no hierarchy).
  template <typename T>
  CoarseFirstStep<T> first_step(int L) {
    CoarseFirstStep<T> fs;
    if (nlev == 1 || L >= nlev - 1) return fs;
    auto& lv = levels<T>()[L];
    const bool cheb = o.smoother != 1;
    fs.dinv = lv.dinv;
    fs.coef = cheb ? coef[L] : nullptr;
    fs.omega = (T)o.omega;
    fs.x0 = lv.x[0];
    fs.d = cheb ? lv.d : nullptr;
    return fs;
  }

  // smoothing degrees of level L (coarse_sweeps > 0 overrides both on levels >= 1)
  int pre_sweeps(int L) const {
    if (L == deep_L && deep_L > 0 && o.block_sweeps > 0) return o.block_sweeps;
    if (L > 1 && o.deep_sweeps > 0) return o.deep_sweeps;
    return (L > 0 && o.coarse_sweeps > 0) ? o.coarse_sweeps : o.pre_sweeps;
  }
  int post_sweeps(int L) const {
    if (L == deep_L && deep_L > 0 && o.block_sweeps > 0) return o.block_sweeps;
    if (L > 1 && o.deep_sweeps > 0) return o.deep_sweeps;
    return (L > 0 && o.coarse_sweeps > 0) ? o.coarse_sweeps : o.post_sweeps;
  }

  // Level L (the last smoothed level) and the coarsest solve as one block
  // (deep_cycle_kernel); the restriction that produced b took the first
  // smoothing step.  Returns the buffer holding level L's iterate.
  float* deep_cycle(int L, const float* b, const int* done, int* rc) {
    auto& lv = L32[L];
    auto fill = [&](auto& p) {
      p.g = grids[L];
      p.gc = grids[L + 1];
      p.fix = fix[L];
      p.fixc = fix[L + 1];
      p.dinv = lv.dinv;
      p.coef = coef[L];
      p.inv = cinv32;
      p.cn = cn;
      p.inv_smem = deep_inv_smem ? 1 : 0;
      p.b = b;
      p.x0 = lv.x[0];
      p.d0 = o.smoother != 1 ? lv.d : nullptr;
      p.xout = lv.x[0];
      p.pre = pre_sweeps(L);
      p.post = post_sweeps(L);
      p.cheb = o.smoother != 1;
      p.omega = (float)o.omega;
      p.done = done;
    };
    {
      const double n = 3.0 * grids[L].nnode();
      count_bytes(81.0 * stencil_bytes<float>(L) * n + 4.0 * cn * cn + 4.0 * sizeof(float) * n +
                  (double)grids[L].nnode());
    }
    if (S16[L]) {
      DeepParams<float, __nv_bfloat16> p;
      fill(p);
      p.S = deep_SN;
      launch(kPdlCoarse, deep_cycle_kernel<float, __nv_bfloat16>, dim3(1), dim3(kDeepThreads), deep_smem, p);
    } else {
      DeepParams<float, float> p;
      fill(p);
      p.S = lv.A;
      launch(kPdlCoarse, deep_cycle_kernel<float, float>, dim3(1), dim3(kDeepThreads), deep_smem, p);
    }
    if (cudaGetLastError() != cudaSuccess) *rc = TP3D_ERR_CUDA;
    return lv.x[0];
  }

  // Levels L, L + 1 and the coarsest solve as one thread-block cluster
  // (cluster_cycle_kernel); the restriction that produced b took level L's
  // first smoothing step.  Returns the buffer holding level L's iterate.
  float* cluster_cycle(int L, const float* b, const int* done, int* rc) {
    auto& la = L32[L];
    auto& lb = L32[L + 1];
    ClusterParams p;
    p.gA = grids[L];
    p.gB = grids[L + 1];
    p.gC = grids[L + 2];
    p.SA = clu_SN;
    p.SB = deep_SN;
    p.fixA = fix[L];
    p.fixB = fix[L + 1];
    p.fixC = fix[L + 2];
    p.dinvA = la.dinv;
    p.dinvB = lb.dinv;
    p.coefA = coef[L];
    p.coefB = coef[L + 1];
    p.inv = cinv32;
    p.cn = cn;
    p.b = b;
    p.x0 = la.x[0];
    p.d0 = o.smoother != 1 ? la.d : nullptr;
    p.xout = la.x[0];
    p.preA = pre_sweeps(L);
    p.postA = post_sweeps(L);
    p.preB = pre_sweeps(L + 1);
    p.postB = post_sweeps(L + 1);
    p.cheb = o.smoother != 1;
    p.omega = (float)o.omega;
    p.done = done;
    {
      const double na = 3.0 * grids[L].nnode(), nb = 3.0 * grids[L + 1].nnode();
      count_bytes(2.0 * kDeepRow / 3.0 * (na + nb) + 4.0 * cn * cn + 5.0 * sizeof(float) * na +
                  (double)(grids[L].nnode() + grids[L + 1].nnode()));
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)clu_C);
    cfg.blockDim = dim3(kClThreads);
    cfg.dynamicSmemBytes = clu_smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)clu_C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = take_pdl(kPdlCoarse) ? 2 : 1;
    if (cudaLaunchKernelEx(&cfg, cluster_cycle_kernel, p) != cudaSuccess) *rc = TP3D_ERR_CUDA;
    count_launch();
    return la.x[0];
  }

  // V-cycle on level L with right-hand side b; returns the buffer holding x.
  template <typename T>
  // zero_done: the first smoothing step from zero already ran (fused into the
  // restriction that produced b).
  // dot_op >= 0 (level 0 only): when the last post-smoothing step is a
  // Chebyshev step, it also reduces b . x and applies finalize op dot_op;
  // *dot_done tells the caller whether it did.
  T* vcycle(int L, const T* b, const int* done, int* rc, bool zero_done = false, int dot_op = -1,
            bool* dot_done = nullptr) {
    if (dot_done) *dot_done = false;
    auto& lv = levels<T>()[L];
    const Grid& gl = grids[L];
    const long long ndof = 3 * gl.nnode();
    if (nlev == 1) {  // no hierarchy: Jacobi preconditioner
      count_bytes(3.0 * sizeof(T) * ndof);
      launch(kPdlFine, smooth_zero_kernel<T>, dim3(grid_blocks(ndof)), dim3(256), 0, ndof, b, (const T*)lv.dinv, T(1),
             (const double*)nullptr, lv.x[0], (T*)nullptr, done);
      return lv.x[0];
    }
    if (L == nlev - 1) {
      const T* inv;
      if constexpr (sizeof(T) == 8) inv = cinv64;
      else inv = cinv32;
      count_bytes((double)sizeof(T) * cn * cn + 2.0 * sizeof(T) * cn);
      launch(kPdlCoarse, dense_matvec_kernel<T>, dim3(std::max(1, std::min(cn / 8 + 1, nsm))), dim3(256), 0, cn, inv,
             b, lv.x[0], done);
      return lv.x[0];
    }
    if (L == cyc_L0 && cyc_L0 > 0) return coarse_cycle<T>(L, b, rc);
    if constexpr (sizeof(T) == 4) {
      if (L == clu_L && clu_L > 0 && zero_done) return cluster_cycle(L, b, done, rc);
      if (L == deep_L && deep_L > 0 && zero_done) return deep_cycle(L, b, done, rc);
    }
    const bool cheb = o.smoother != 1;
    int cur = 0;
    if (!zero_done) {
      count_bytes((cheb ? 4.0 : 3.0) * sizeof(T) * ndof);
      launch(L == 0 ? kPdlFine : kPdlCoarse, smooth_zero_kernel<T>, dim3(grid_blocks(ndof)), dim3(256), 0, ndof, b,
             (const T*)lv.dinv, (T)o.omega, (const double*)(cheb ? coef[L] : nullptr), lv.x[cur],
             cheb ? lv.d : (T*)nullptr, done);
    }
    *rc |= smooth_steps<T>(L, 1, pre_sweeps(L) - 1, &cur, b, done);
    auto& lc = levels<T>()[L + 1];
    const Grid& gn = grids[L + 1];
    // small coarse levels: residual and restriction in one launch
    const bool resid_fused = L > 0 && ndof <= o.resid_restrict_dofs;
    if (!resid_fused) {
      OpIO<T> io;
      io.u = lv.x[cur];
      io.out = lv.r;
      io.b = b;
      io.done = done;
      *rc |= apply_level<T, kModeResid>(L, io);
    }
    // the next level's first smoothing step rides along when that level smooths
    const bool fuse_first = L + 1 < nlev - 1 && !(L + 1 == cyc_L0 && cyc_L0 > 0);
    CoarseFirstStep<T> fs;
    if (fuse_first) {
      fs.dinv = lc.dinv;
      fs.coef = cheb ? coef[L + 1] : nullptr;
      fs.omega = (T)o.omega;
      fs.x0 = lc.x[0];
      fs.d = cheb ? lc.d : nullptr;
    }
    if (resid_fused) {
      auto fill = [&](auto& p) {
        p.g = gl;
        p.fix = fix[L];
        p.io.u = lv.x[cur];
        p.io.b = b;
        p.io.done = done;
      };
      count_bytes(2.0 * sizeof(T) * ndof + 81.0 * stencil_bytes<T>(L) * ndof + (double)gl.nnode() +
                  (double)gn.nnode() + (fuse_first ? 4.0 : 1.0) * sizeof(T) * 3.0 * gn.nnode());
      const dim3 grid((unsigned)gn.nnode());
      bool done16 = false;
      if constexpr (sizeof(T) == 4) {
        if (S16[L]) {
          StencilParams<float, __nv_bfloat16> p;
          fill(p);
          p.S = S16[L];
          launch(kPdlCoarse, restrict_resid_kernel<float, __nv_bfloat16>, grid, dim3(kRestrictResidThreads), 0, p,
                 gn, (const uint8_t*)fix[L + 1], lc.b, fs);
          done16 = true;
        }
      }
      if (!done16) {
        StencilParams<T> p;
        fill(p);
        p.S = lv.A;
        launch(kPdlCoarse, restrict_resid_kernel<T, T>, grid, dim3(kRestrictResidThreads), 0, p, gn,
               (const uint8_t*)fix[L + 1], lc.b, fs);
      }
    } else {
      count_bytes((double)sizeof(T) * ndof + (double)gn.nnode() +
                  (fuse_first ? 4.0 : 1.0) * sizeof(T) * 3.0 * gn.nnode());
      launch(kPdlCoarse, restrict_kernel<T>, plane_grid((gn.nx + 1) * (gn.ny + 1), gn.nz + 1), dim3(256), 0, gl,
             gn, (const T*)lv.r, (const uint8_t*)fix[L + 1], lc.b, done, fs);
    }
    T* xc = vcycle<T>(L + 1, lc.b, done, rc, fuse_first);
    count_bytes((double)sizeof(T) * 3.0 * gn.nnode() + 2.0 * sizeof(T) * ndof + (double)gl.nnode());
    launch(L == 0 ? kPdlFine : kPdlCoarse, prolong_add_kernel<T>, plane_grid((gl.nx + 1) * (gl.ny + 1), gl.nz + 1),
           dim3(256), 0, gl, gn, (const T*)xc, (const uint8_t*)fix[L], lv.x[cur], done);
    const bool dot_here = dot_op >= 0 && o.smoother != 1 && post_sweeps(L) >= 1;
    *rc |= smooth_steps<T>(L, 0, post_sweeps(L), &cur, b, done, dot_here ? dot_op : -1);
    if (dot_here && dot_done) *dot_done = true;
    if (cudaGetLastError() != cudaSuccess) *rc = TP3D_ERR_CUDA;
    return lv.x[cur];
  }

  // ---------------- graphs ----------------
  template <typename T, class Body>
  int capture(KrylovVec<T>& K, Body body) {
    if (K.graph) return TP3D_OK;
    cudaGraph_t gr = nullptr;
    TP3D_CHECK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    long long nk = 0;
    double nbytes = 0.0;
    t_capture_count = &nk;
    t_capture_bytes = &nbytes;
    pdl_region = true;
    plain_next = true;
    const int rc = body();
    pdl_region = false;
    t_capture_count = nullptr;
    t_capture_bytes = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &gr);
    const cudaError_t e2 = (rc || e != cudaSuccess) ? cudaErrorUnknown : cudaGraphInstantiate(&K.graph, gr, 0);
    if (e == cudaSuccess && gr) cudaGraphDestroy(gr);
    if (rc || e != cudaSuccess || e2 != cudaSuccess) {
      cudaGetLastError();
      K.graph = nullptr;
      if (pdl) {  // retry in plain stream order
        pdl = false;
        return capture<T>(K, body);
      }
      tp3d_set_last_error("CG graph capture failed");
      return TP3D_ERR_CUDA;
    }
    K.graph_kernels = nk;
    K.graph_bytes = nbytes;
    return TP3D_OK;
  }

  // The CG iteration as the body of a device-side while loop (a CUDA graph
  // WHILE node whose condition set_loop_cond_kernel sets at the end of each
  // pass); a reliable-update branch inside the body becomes an IF node
  // (update_branch).  One graph launch then runs the whole solve with no host
  // round trip.  Returns false when the graph cannot be built this way; the
  // caller then captures the plain iteration and polls.
  template <typename T, class Body>
  bool capture_loop(KrylovVec<T>& K, Body body) {
    if (K.graph) return true;
    if (!loop_ok || !o.device_loop) return false;
    cudaGraph_t G = nullptr;
    bool ok = cudaGraphCreate(&G, 0) == cudaSuccess;
    cudaGraphConditionalHandle hw = 0;
    ok = ok && cudaGraphConditionalHandleCreate(&hw, G, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = hw;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wnode;
    ok = ok && cudaGraphAddNode(&wnode, G, nullptr, 0, &cp) == cudaSuccess;
    bool capturing = false;
    long long nk = 0;
    double nbytes = 0.0;
    int rc = TP3D_OK;
    if (ok) {
      cudaGraph_t B = cp.conditional.phGraph_out[0];
      capturing = cudaStreamBeginCaptureToGraph(st, B, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
                  cudaSuccess;
      ok = capturing;
    }
    if (ok) {
      t_capture_count = &nk;
      t_capture_bytes = &nbytes;
      in_loop_capture = true;
      branch_count = 0;
      pdl_region = true;
      plain_next = true;
      rc = body();
      pdl_region = false;
      set_loop_cond_kernel<<<1, 1, 0, st>>>(hw, state, loop_passes, (unsigned int)o.max_iterations + 16u);
      ++nk;
      in_loop_capture = false;
      t_capture_count = nullptr;
      t_capture_bytes = nullptr;
    }
    if (capturing) {
      cudaGraph_t out = nullptr;
      ok = cudaStreamEndCapture(st, &out) == cudaSuccess && ok;
    }
    ok = ok && rc == TP3D_OK && branch_ok && cudaGraphInstantiate(&K.graph, G, 0) == cudaSuccess;
    if (G) cudaGraphDestroy(G);
    cudaGetLastError();  // clear a failed attempt's error state
    if (!ok) {
      if (K.graph) cudaGraphExecDestroy(K.graph);
      K.graph = nullptr;
      branch_ok = true;
      if (pdl) {  // retry in plain stream order
        pdl = false;
        return capture_loop<T>(K, body);
      }
      loop_ok = false;
      return false;
    }
    K.loop = true;
    K.graph_kernels = nk;
    K.graph_bytes = nbytes;
    K.branch_kernels = branch_count;
    return true;
  }

  // Kernels of the reliable update: inside a loop capture they form the body
  // of an IF node on set_update_cond_kernel's condition; otherwise they are
  // launched directly (each gated on state->update itself).
  template <class Branch>
  int update_branch(Branch branch) {
    if (!in_loop_capture) return branch();
    cudaStreamCaptureStatus cs;
    cudaGraph_t capg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    cudaGraphConditionalHandle h = 0;
    if (cudaStreamGetCaptureInfo(st, &cs, nullptr, &capg, &deps, &nd) != cudaSuccess ||
        cudaGraphConditionalHandleCreate(&h, capg, 0, cudaGraphCondAssignDefault) != cudaSuccess) {
      branch_ok = false;
      return TP3D_ERR_CUDA;
    }
    set_update_cond_kernel<<<1, 1, 0, st>>>(h, state);
    count_launch();
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    if (cudaStreamGetCaptureInfo(st, &cs, nullptr, &capg, &deps, &nd) != cudaSuccess ||
        cudaGraphAddNode(&node, capg, deps, nd, &cp) != cudaSuccess ||
        cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess) {
      branch_ok = false;
      return TP3D_ERR_CUDA;
    }
    // the branch body, captured on the second stream
    std::swap(st, st_branch);
    int rc = TP3D_OK;
    if (cudaStreamBeginCaptureToGraph(st, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      branch_ok = false;
      rc = TP3D_ERR_CUDA;
    } else {
      long long* outer = t_capture_count;
      double* outer_bytes = t_capture_bytes;
      long long nb = 0;
      t_capture_count = &nb;
      t_capture_bytes = nullptr;  // the branch runs only on a reliable update
      plain_next = true;
      rc = branch();
      t_capture_count = outer;
      t_capture_bytes = outer_bytes;
      cudaGraph_t out = nullptr;
      if (cudaStreamEndCapture(st, &out) != cudaSuccess) {
        branch_ok = false;
        rc = TP3D_ERR_CUDA;
      }
      branch_count += nb;
    }
    std::swap(st, st_branch);
    plain_next = true;  // the next kernel follows the IF node
    return rc;
  }

  // One launch of the loop graph; the pass count and reliable updates of the
  // run feed the launch counter.
  template <typename T>
  int replay_loop(KrylovVec<T>& K) {
    TP3D_CHECK(cudaMemsetAsync(loop_passes, 0, sizeof(unsigned int), st));
    TP3D_CHECK(cudaGraphLaunch(K.graph, st));
    unsigned int passes = 0;
    TP3D_CHECK(cudaMemcpyAsync(state_host, state, sizeof(PcgState), cudaMemcpyDeviceToHost, st));
    TP3D_CHECK(cudaMemcpyAsync(loop_pass_host, loop_passes, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
    TP3D_CHECK(cudaStreamSynchronize(st));
    passes = *loop_pass_host;
    add_launches((long long)passes * K.graph_kernels + (long long)state_host[0].updates * K.branch_kernels);
    return TP3D_OK;
  }

  // Replay the iteration graph until the device stop flag is set (two-deep polling).
  template <typename T>
  int replay(KrylovVec<T>& K, int max_iters) {
    if (K.loop) return replay_loop<T>(K);
    const int chunk = 4;
    int launched = 0, which = 0, status = TP3D_OK;
    bool pending = false;
    cudaEvent_t ev[2];
    cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
    while (true) {
      for (int k = 0; k < chunk && status == TP3D_OK; ++k) {
        if (cudaGraphLaunch(K.graph, st) != cudaSuccess) status = TP3D_ERR_CUDA;
        add_launches(K.graph_kernels);
      }
      launched += chunk;
      cudaMemcpyAsync(state_host + which, state, sizeof(PcgState), cudaMemcpyDeviceToHost, st);
      cudaEventRecord(ev[which], st);
      if (pending) {
        cudaEventSynchronize(ev[1 - which]);
        if (state_host[1 - which].done) break;
      }
      pending = true;
      which = 1 - which;
      if (status || launched > max_iters + 2 * chunk) break;
    }
    cudaMemcpyAsync(state_host, state, sizeof(PcgState), cudaMemcpyDeviceToHost, st);
    const cudaError_t e = cudaStreamSynchronize(st);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    if (e != cudaSuccess) {
      tp3d_set_last_error(cudaGetErrorString(e));
      return TP3D_ERR_CUDA;
    }
    return status;
  }

  int status_of(const PcgState& s) {
    if (s.done == 1) return TP3D_OK;
    if (s.done == 5) {
      last_floor = true;
      return TP3D_OK;
    }
    if (s.done == 3 || s.done == 4) {
      tp3d_set_last_error(s.done == 3 ? "CG breakdown (p'Ap <= 0)" : "non-finite residual in CG");
      return TP3D_ERR_NONFINITE;
    }
    if (s.done == 7) {
      tp3d_set_last_error("coarse-cycle grid barrier expired");
      return TP3D_ERR_TIMEOUT;
    }
    return TP3D_NOT_CONVERGED;
  }

  // ---------------- solves inside a captured SIMP stage ----------------
  cudaStream_t st_loop = nullptr, st_restart = nullptr;
  long long stage_loop_kernels = 0;  // kernels of one CG iteration in the last loop captured this way
  double* restart_state = nullptr;   // device [previous residual, iterations, restarts] (stage graphs)

  // A WHILE node added to the graph that `st` is being captured into; its body
  // is captured by body(handle) on `other` (swapped in as `st` meanwhile) and
  // must end with a kernel that sets the handle's condition.  The node is
  // re-armed by a kernel before it (a nested loop runs once per entry).
  template <class Body>
  int while_into(cudaStream_t& other, Body body) {
    if (!other) return TP3D_ERR_ARG;  // created before the capture
    cudaStreamCaptureStatus cs;
    cudaGraph_t capg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    cudaGraphConditionalHandle hw = 0;
    TP3D_CHECK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &capg, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) {
      tp3d_set_last_error("while_into: the solver stream is not capturing");
      return TP3D_ERR_ARG;
    }
    TP3D_CHECK(cudaGraphConditionalHandleCreate(&hw, capg, 1, cudaGraphCondAssignDefault));
    arm_conditional_kernel<<<1, 1, 0, st>>>(hw);
    TP3D_CHECK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &capg, &deps, &nd));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = hw;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wnode;
    TP3D_CHECK(cudaGraphAddNode(&wnode, capg, deps, nd, &cp));
    TP3D_CHECK(cudaStreamUpdateCaptureDependencies(st, &wnode, 1, cudaStreamSetCaptureDependencies));
    std::swap(st, other);
    int rc = TP3D_OK;
    if (cudaStreamBeginCaptureToGraph(st, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      rc = TP3D_ERR_CUDA;
    } else {
      plain_next = true;
      rc = body(hw);
      cudaGraph_t out = nullptr;
      if (cudaStreamEndCapture(st, &out) != cudaSuccess) rc = TP3D_ERR_CUDA;
    }
    std::swap(st, other);
    plain_next = true;
    return rc;
  }

  // The CG iteration as a WHILE node in the graph being captured (the caller's
  // stage graph); the reliable-update branch inside becomes a nested IF node as
  // in capture_loop.  Nothing is instantiated here: the stage graph holds the loop.
  template <class Body>
  int capture_loop_into(Body body) {
    TP3D_CHECK(cudaMemsetAsync(loop_passes, 0, sizeof(unsigned int), st));
    long long* outer = t_capture_count;
    t_capture_count = &stage_loop_kernels;
    stage_loop_kernels = 0;
    const int rc = while_into(st_loop, [&](cudaGraphConditionalHandle hw) {
      in_loop_capture = true;
      branch_ok = true;
      pdl_region = true;
      plain_next = true;
      int r = body();
      pdl_region = false;
      set_loop_cond_kernel<<<1, 1, 0, st>>>(hw, state, loop_passes, (unsigned int)o.max_iterations + 16u);
      ++stage_loop_kernels;
      in_loop_capture = false;
      if (!branch_ok) r = TP3D_ERR_CUDA;
      return r;
    });
    t_capture_count = outer;
    if (rc) tp3d_set_last_error("capture of the CG loop into the stage graph failed");
    return rc;
  }

  // One solve of K U = F queued on the caller's (capturing) stream with no host
  // synchronisation: the host path's prologue (its state written by a kernel),
  // the CG loop as a WHILE node and the FP64 result.  The mixed form raises
  // *abort when the host path would have finished the solve with its FP64
  // fallback; the FP64 form runs the host path's restart loop (run, true
  // residual, restart) as a WHILE node and raises *abort where the host path
  // would have reported a failure.  *cg accumulates the CG iterations.
  int solve_into_capture(const double* F, double* U, int* abort, int* cg) {
    const long long nn = g.nnode(), ndof = 3 * nn;
    const int nb = grid_blocks(ndof);
    if (int e = enter()) return e;
    if (cyc_bar) TP3D_CHECK(cudaMemsetAsync(cyc_bar, 0, 2 * sizeof(unsigned int), st));
    TP3D_CHECK(cudaMemcpyAsync(u64, U, ndof * sizeof(double), cudaMemcpyDeviceToDevice, st));
    zero_fixed_kernel<<<grid_blocks(nn), 256, 0, st>>>(nn, u64, fix[0]);
    int rc = TP3D_OK;
    if (mixed) {
      init_state_kernel<<<1, 1, 0, st>>>(state, o.max_iterations, o.reliable_delta * o.reliable_delta);
      TP3D_CHECK(cudaMemcpyAsync(F_capture, F, ndof * sizeof(double), cudaMemcpyDeviceToDevice, st));
      masked_norm_kernel<<<grid_blocks(nn), 256, 0, st>>>(nn, F, fix[0], partials);
      finalize_kernel<<<1, 256, 0, st>>>(partials, grid_blocks(nn), state, kFinBB, o.rtol * o.rtol, nullptr);
      OpIO<double> r;
      r.u = u64;
      r.out = r64;
      r.b = F;
      rc |= fine<double, kModeResid>(r);
      dot_kernel<double><<<nb, 256, 0, st>>>(ndof, r64, r64, partials, nullptr, nullptr);
      finalize_kernel<<<1, 256, 0, st>>>(partials, nb, state, kFinRRInit, 0.0, nullptr);
      demote_kernel<<<nb, 256, 0, st>>>(ndof, r64, K32.r, state, 1);
      TP3D_CHECK(cudaMemsetAsync(K32.u, 0, ndof * sizeof(float), st));
      float* z = vcycle<float>(0, K32.r, &state->done, &rc);
      dot_kernel<float><<<nb, 256, 0, st>>>(ndof, K32.r, z, partials, &state->done, nullptr);
      finalize_kernel<<<1, 256, 0, st>>>(partials, nb, state, kFinRZInit, 0.0, nullptr);
      cg_p_kernel<float><<<nb, 256, 0, st>>>(ndof, z, K32.p, state, 1);
      if (rc == TP3D_OK) rc = capture_loop_into([&]() { return mixed_iteration(); });
      flush_kernel<<<nb, 256, 0, st>>>(ndof, u64, K32.u, state, 1);
      solve_status_kernel<<<1, 1, 0, st>>>(state, abort, cg);
    } else {
      if (!restart_state) return TP3D_ERR_ARG;  // allocated before the capture (tp3d_stage_capture)
      restart_init_kernel<<<1, 1, 0, st>>>(restart_state);
      if (rc == TP3D_OK)
        rc = while_into(st_restart, [&](cudaGraphConditionalHandle hr) {
          int r = TP3D_OK;
          init_state_budget_kernel<<<1, 1, 0, st>>>(state, restart_state, o.max_iterations);
          masked_norm_kernel<<<grid_blocks(nn), 256, 0, st>>>(nn, F, fix[0], partials);
          finalize_kernel<<<1, 256, 0, st>>>(partials, grid_blocks(nn), state, kFinBB, o.rtol * o.rtol, nullptr);
          OpIO<double> io;
          io.u = K64.u;
          io.out = K64.r;
          io.b = F;
          r |= fine<double, kModeResid>(io);
          dot_kernel<double><<<nb, 256, 0, st>>>(ndof, K64.r, K64.r, partials, nullptr, nullptr);
          finalize_kernel<<<1, 256, 0, st>>>(partials, nb, state, kFinRRInit, 0.0, nullptr);
          double* z = vcycle<double>(0, K64.r, &state->done, &r);
          dot_kernel<double><<<nb, 256, 0, st>>>(ndof, K64.r, z, partials, &state->done, nullptr);
          finalize_kernel<<<1, 256, 0, st>>>(partials, nb, state, kFinRZInit, 0.0, nullptr);
          cg_p_kernel<double><<<nb, 256, 0, st>>>(ndof, z, K64.p, state, 1);
          if (r == TP3D_OK) r = capture_loop_into([&]() { return pcg64_iteration(); });
          // the true residual, into state->rr where the host path's check reads it
          if (r == TP3D_OK) r = true_residual(F, K64.u, K64.q, &state->rr);
          restart_decide_kernel<<<1, 1, 0, st>>>(hr, state, restart_state, o.rtol, o.max_restarts,
                                                 o.max_iterations, abort, cg);
          return r;
        });
    }
    TP3D_CHECK(cudaMemcpyAsync(U, u64, ndof * sizeof(double), cudaMemcpyDeviceToDevice, st));
    TP3D_CHECK_LAUNCH();
    if (rc) return rc;
    return leave();
  }

  // ---------------- FP64 PCG ----------------
  int pcg64_iteration() {
    const long long ndof = 3 * g.nnode();
    int* done = &state->done;
    const int nb = grid_blocks(ndof);
    KrylovVec<double>& K = K64;
    OpIO<double> io;
    io.u = K.p;
    io.out = K.q;
    io.partials = partials;
    io.done = done;
    io.fin = state;
    io.fin_op = kFinPQ;
    io.fin_count = fin_count;
    int rc = fine<double, kModeCgQ>(io);
    const CoarseFirstStep<double> fs0 = first_step<double>(0);
    count_bytes((fs0.x0 ? 9.0 : 6.0) * 8.0 * ndof);
    launch(kPdlFine, cg_update_kernel<double>, dim3(nb), dim3(256), 0, ndof, K.u, (const double*)K.p, K.r,
           (const double*)K.q, state, partials, (int)kFinRR, fin_count, fs0);
    bool dot_done = false;
    double* z = vcycle<double>(0, K.r, done, &rc, fs0.x0 != nullptr, kFinRZ, &dot_done);
    if (!dot_done) {
      count_bytes(2.0 * 8.0 * ndof);
      launch(kPdlFine, dot_kernel<double>, dim3(nb), dim3(256), 0, ndof, (const double*)K.r, (const double*)z, partials,
             (const int*)done, (const int*)nullptr, state, (int)kFinRZ, fin_count);
    }
    count_bytes(3.0 * 8.0 * ndof);
    launch(kPdlFine, cg_p_kernel<double>, dim3(nb), dim3(256), 0, ndof, (const double*)z, K.p,
           (const PcgState*)state, 0);
    TP3D_CHECK_LAUNCH();
    return rc;
  }

  // One PCG run from K64.u; returns status, fills state_host[0].
  int pcg64_run(const double* F, double rtol, int max_iters) {
    const long long nn = g.nnode(), ndof = 3 * nn;
    const int nb = grid_blocks(ndof);
    int rc = TP3D_OK;
    if (!capture_loop<double>(K64, [&]() { return pcg64_iteration(); }))
      rc = capture<double>(K64, [&]() { return pcg64_iteration(); });
    if (rc) return rc;
    PcgState init{};
    init.max_iters = max_iters;
    TP3D_CHECK(cudaMemcpyAsync(state, &init, sizeof(PcgState), cudaMemcpyHostToDevice, st));
    masked_norm_kernel<<<grid_blocks(nn), 256, 0, st>>>(nn, F, fix[0], partials); count_launch();
    finalize_kernel<<<1, 256, 0, st>>>(partials, grid_blocks(nn), state, kFinBB, rtol * rtol, nullptr); count_launch();
    OpIO<double> io;
    io.u = K64.u;
    io.out = K64.r;
    io.b = F;
    rc |= fine<double, kModeResid>(io);
    dot_kernel<double><<<nb, 256, 0, st>>>(ndof, K64.r, K64.r, partials, nullptr, nullptr); count_launch();
    finalize_kernel<<<1, 256, 0, st>>>(partials, nb, state, kFinRRInit, 0.0, nullptr); count_launch();
    double* z = vcycle<double>(0, K64.r, &state->done, &rc);
    dot_kernel<double><<<nb, 256, 0, st>>>(ndof, K64.r, z, partials, &state->done, nullptr); count_launch();
    finalize_kernel<<<1, 256, 0, st>>>(partials, nb, state, kFinRZInit, 0.0, nullptr); count_launch();
    cg_p_kernel<double><<<nb, 256, 0, st>>>(ndof, z, K64.p, state, 1); count_launch();
    TP3D_CHECK_LAUNCH();
    if (rc) return rc;
    return replay<double>(K64, max_iters);
  }

  // ||F - K u||^2 over free DOFs into *out (device), FP64.
  int true_residual(const double* F, const double* u, double* rbuf, double* out) {
    const long long ndof = 3 * g.nnode();
    const int nb = grid_blocks(ndof);
    OpIO<double> io;
    io.u = u;
    io.out = rbuf;
    io.b = F;
    int rc = fine<double, kModeResid>(io);
    dot_kernel<double><<<nb, 256, 0, st>>>(ndof, rbuf, rbuf, partials, nullptr, nullptr); count_launch();
    finalize_kernel<<<1, 256, 0, st>>>(partials, nb, state, kFinValue, 0.0, out); count_launch();
    return rc;
  }

  // The true residual of a design with 1e-9 voids has an attainable floor
  // (about eps times the condition-weighted ||K|| ||u|| / ||f||) that can sit
  // above rtol even though the recursive CG residual keeps falling.  Restart
  // from the true residual while that still gains at least a factor of 2; once
  // a restart stops gaining, the solve has reached the floor and is accepted
  // (last_floor = true, last_relres = the true residual).
  int solve64(const double* F) {
    int total = 0, restarts = 0, rc = TP3D_OK;
    double relres = 0.0, prev = INFINITY;
    last_floor = false;
    for (;;) {
      rc = pcg64_run(F, o.rtol, std::max(1, o.max_iterations - total));
      if (rc < 0) return rc;
      const PcgState s = state_host[0];
      total += s.iters;
      rc = status_of(s);
      if (rc < 0) return rc;
      if (s.bb == 0.0) {
        relres = 0.0;
        break;
      }
      // the recursive residual may have drifted from the true one: check
      double* tr = &state->rr;  // scratch slot, the state is re-initialised per run
      if (int e = true_residual(F, K64.u, K64.q, tr)) return e;
      double rr_true = 0.0;
      TP3D_CHECK(cudaMemcpyAsync(&rr_true, tr, sizeof(double), cudaMemcpyDeviceToHost, st));
      TP3D_CHECK(cudaStreamSynchronize(st));
      relres = std::sqrt(std::max(rr_true, 0.0) / s.bb);
      if (!std::isfinite(relres)) {
        tp3d_set_last_error("non-finite residual in CG");
        return TP3D_ERR_NONFINITE;
      }
      if (relres <= 2.0 * o.rtol) {
        rc = TP3D_OK;
        break;
      }
      if (rc == TP3D_OK && relres > 0.5 * prev) {  // recursive target met, restarts no longer gain
        last_floor = true;
        break;
      }
      if (rc == TP3D_NOT_CONVERGED || restarts >= o.max_restarts || total >= o.max_iterations) {
        rc = TP3D_NOT_CONVERGED;
        break;
      }
      prev = relres;
      ++restarts;
    }
    last_iters = total;
    last_restarts = restarts;
    last_relres = relres;
    return rc;
  }

  // ---------------- mixed: FP32 CG with FP64 reliable updates ----------------
  int mixed_iteration() {
    const long long ndof = 3 * g.nnode();
    int* done = &state->done;
    const int nb = grid_blocks(ndof);
    KrylovVec<float>& K = K32;
    OpIO<float> io;
    io.u = K.p;
    io.out = K.q;
    io.partials = partials;
    io.done = done;
    io.fin = state;
    io.fin_op = kFinPQMixed;
    io.fin_count = fin_count;
    int rc = fine<float, kModeCgQ>(io);
    const CoarseFirstStep<float> fs0 = first_step<float>(0);
    count_bytes((fs0.x0 ? 9.0 : 6.0) * 4.0 * ndof);
    launch(kPdlFine, cg_update_kernel<float>, dim3(nb), dim3(256), 0, ndof, K.u, (const float*)K.p, K.r,
           (const float*)K.q, state, partials, (int)kFinRRMixed, fin_count, fs0);
    // reliable update (each kernel is also gated on state->update itself)
    rc |= update_branch([&]() {
      int brc = TP3D_OK;
      launch(kPdlFine, flush_kernel, dim3(nb), dim3(256), 0, ndof, u64, K.u, (const PcgState*)state, 0);
      OpIO<double> r;
      r.u = u64;
      r.out = r64;
      r.b = F_capture;
      r.done = done;
      r.gate = &state->update;
      brc |= fine<double, kModeResid>(r);
      launch(kPdlFine, dot_kernel<double>, dim3(nb), dim3(256), 0, ndof, (const double*)r64, (const double*)r64,
             partials, (const int*)done, (const int*)&state->update, state, (int)kFinRRHi, fin_count);
      launch(kPdlFine, demote_kernel, dim3(nb), dim3(256), 0, ndof, (const double*)r64, K.r, (const PcgState*)state, 0);
      if (fs0.x0) {  // the first smoothing step again, from the replaced residual
        launch(kPdlFine, smooth_zero_kernel<float>, dim3(nb), dim3(256), 0, ndof, (const float*)K.r,
               (const float*)fs0.dinv, fs0.omega, (const double*)fs0.coef, fs0.x0, fs0.d, (const int*)done);
      }
      launch(kPdlFine, clear_update_kernel, dim3(1), dim3(1), 0, state);
      return brc;
    });
    bool dot_done = false;
    float* z = vcycle<float>(0, K.r, done, &rc, fs0.x0 != nullptr, kFinRZMixed, &dot_done);
    if (!dot_done) {
      count_bytes(2.0 * 4.0 * ndof);
      launch(kPdlFine, dot_kernel<float>, dim3(nb), dim3(256), 0, ndof, (const float*)K.r, (const float*)z, partials,
             (const int*)done, (const int*)nullptr, state, (int)kFinRZMixed, fin_count);
    }
    count_bytes(3.0 * 4.0 * ndof);
    launch(kPdlFine, cg_p_kernel<float>, dim3(nb), dim3(256), 0, ndof, (const float*)z, K.p, (const PcgState*)state, 0);
    TP3D_CHECK_LAUNCH();
    return rc;
  }

  // The mixed solve up to its result in u64, without waiting for it.
  int solve_mixed_launch(const double* F) {
    const long long nn = g.nnode(), ndof = 3 * nn;
    const int nb = grid_blocks(ndof);
    last_floor = false;
    int rc = TP3D_OK;
    if (!capture_loop<float>(K32, [&]() { return mixed_iteration(); }))
      rc = capture<float>(K32, [&]() { return mixed_iteration(); });
    if (rc) return rc;
    PcgState init{};
    init.max_iters = o.max_iterations;
    init.delta2 = o.reliable_delta * o.reliable_delta;
    TP3D_CHECK(cudaMemcpyAsync(state, &init, sizeof(PcgState), cudaMemcpyHostToDevice, st));
    TP3D_CHECK(cudaMemcpyAsync(F_capture, F, ndof * sizeof(double), cudaMemcpyDeviceToDevice, st));
    masked_norm_kernel<<<grid_blocks(nn), 256, 0, st>>>(nn, F, fix[0], partials); count_launch();
    finalize_kernel<<<1, 256, 0, st>>>(partials, grid_blocks(nn), state, kFinBB, o.rtol * o.rtol, nullptr);
    count_launch();
    // FP64 residual of the initial guess, demoted to FP32
    OpIO<double> r;
    r.u = u64;
    r.out = r64;
    r.b = F;
    rc |= fine<double, kModeResid>(r);
    dot_kernel<double><<<nb, 256, 0, st>>>(ndof, r64, r64, partials, nullptr, nullptr); count_launch();
    finalize_kernel<<<1, 256, 0, st>>>(partials, nb, state, kFinRRInit, 0.0, nullptr); count_launch();
    demote_kernel<<<nb, 256, 0, st>>>(ndof, r64, K32.r, state, 1); count_launch();
    TP3D_CHECK(cudaMemsetAsync(K32.u, 0, ndof * sizeof(float), st));
    float* z = vcycle<float>(0, K32.r, &state->done, &rc);
    dot_kernel<float><<<nb, 256, 0, st>>>(ndof, K32.r, z, partials, &state->done, nullptr); count_launch();
    finalize_kernel<<<1, 256, 0, st>>>(partials, nb, state, kFinRZInit, 0.0, nullptr); count_launch();
    cg_p_kernel<float><<<nb, 256, 0, st>>>(ndof, z, K32.p, state, 1); count_launch();
    TP3D_CHECK_LAUNCH();
    if (rc) return rc;
    rc = replay<float>(K32, o.max_iterations);
    if (rc) return rc;
    flush_kernel<<<nb, 256, 0, st>>>(ndof, u64, K32.u, state, 1); count_launch();
    TP3D_CHECK_LAUNCH();
    return TP3D_OK;
  }

  // The mixed solve launched by solve_mixed_launch: reads its state (host
  // synchronisation) and, if FP32 could not resolve the system, finishes it
  // with the FP64 solver (*fallback set).  `before_fallback` runs first then
  // (the split entry point joins the caller's stream there).
  template <class Before>
  int solve_mixed_finish(const double* F, bool* fallback, Before before_fallback) {
    const long long ndof = 3 * g.nnode();
    *fallback = false;
    TP3D_CHECK(cudaStreamSynchronize(st));
    const PcgState s = state_host[0];
    last_iters = s.iters;
    last_updates = s.updates;
    last_relres = s.bb > 0.0 ? std::sqrt(std::max(s.rr_hi, 0.0) / s.bb) : 0.0;
    last_fallback = false;
    if (s.done == 1 || s.done == 5 || s.done == 7) return status_of(s);
    // FP32 could not resolve this system (cap, breakdown, non-finite, or a
    // stall far above the target): finish it with the FP64 solver.
    *fallback = true;
    if (int e = before_fallback()) return e;
    if (int e = ensure_fp64_buffers()) return e;
    if (s.done == 3 || s.done == 4) TP3D_CHECK(cudaMemsetAsync(u64, 0, ndof * sizeof(double), st));
    const int mixed_iters = s.iters;
    last_fallback = true;
    const int rc = solve64(F);
    last_iters += mixed_iters;
    return rc;
  }

  int solve_mixed(const double* F) {
    if (int rc = solve_mixed_launch(F)) return rc;
    bool fb = false;
    return solve_mixed_finish(F, &fb, [] { return TP3D_OK; });
  }

  // split solve (tp3d_solver_solve_begin / _end)
  bool pending = false;
  const double* pend_F = nullptr;
  double* pend_U = nullptr;
  int pend_rc = TP3D_OK;

  // FP64 Krylov and level vectors for the mixed form's fallback (allocated on first use).
  int ensure_fp64_buffers() {
    if (K64.r) return TP3D_OK;
    const long long ndof = 3 * g.nnode();
    K64.u = u64;
    K64.r = alloc<double>(ndof);
    K64.p = alloc<double>(ndof);
    K64.q = alloc<double>(ndof);
    for (int L = 0; L < nlev; ++L) {
      const long long n = 3 * grids[L].nnode();
      auto& a = L64[L];
      a.x[0] = alloc<double>(n);
      a.x[1] = alloc<double>(n);
      a.b = alloc<double>(n);
      a.r = alloc<double>(n);
      a.d = alloc<double>(n);
      if (!a.x[0] || !a.x[1] || !a.b || !a.r || !a.d) return TP3D_ERR_CUDA;
      if (L > 0) {
        a.A = alloc<double>(243 * grids[L].nnode());
        if (!a.A) return TP3D_ERR_CUDA;
        pack_level<double>(L, a.A);
      }
    }
    if (!K64.r || !K64.p || !K64.q) return TP3D_ERR_CUDA;
    TP3D_CHECK_LAUNCH();
    return TP3D_OK;
  }

  // Packed (apply-layout) copy of the level-L stencil.
  template <typename T>
  void pack_level(int L, T* S) {
    stencil_pack_kernel<T><<<grid_blocks(3 * grids[L].nnode()), 256, 0, st>>>(grids[L], A64[L], fix[L], S);
    count_launch();
  }
  bool last_fallback = false;
};

// KE1[s] = P_s^T KE P_s: interpolation from a coarse element's corners to its
// fine sub-element s, weights prod(1 - |pos - 2 o| / 2) with pos = s + o(a).
static void coarse_subelement_tables(const double* KE, double* out) {
  for (int s = 0; s < 8; ++s) {
    double P[24][24] = {};
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b) {
        const int px = corner_ox(s) + corner_ox(a), py = corner_oy(s) + corner_oy(a), pz = corner_oz(s) + corner_oz(a);
        const double w = std::max(0.0, 1.0 - std::abs(px - 2 * corner_ox(b)) / 2.0) *
                         std::max(0.0, 1.0 - std::abs(py - 2 * corner_oy(b)) / 2.0) *
                         std::max(0.0, 1.0 - std::abs(pz - 2 * corner_oz(b)) / 2.0);
        for (int c = 0; c < 3; ++c) P[3 * a + c][3 * b + c] = w;
      }
    double KP[24][24];
    for (int i = 0; i < 24; ++i)
      for (int j = 0; j < 24; ++j) {
        double t = 0;
        for (int k = 0; k < 24; ++k) t += KE[i * 24 + k] * P[k][j];
        KP[i][j] = t;
      }
    for (int i = 0; i < 24; ++i)
      for (int j = 0; j < 24; ++j) {
        double t = 0;
        for (int k = 0; k < 24; ++k) t += P[k][i] * KP[k][j];
        out[s * 576 + i * 24 + j] = t;
      }
  }
}

// KE2[f] = Q_f^T KE Q_f for the 64 fine elements f = fx + 4 fy + 16 fz of a
// level-2 element: Q_f interpolates from the level-2 element's corners to
// fine element f's corners, weights prod(1 - |pos - 4 o(b)| / 4), pos = f + o(a).
static void level2_element_tables(const double* KE, double* out) {
  for (int f = 0; f < 64; ++f) {
    const int fx = f & 3, fy = (f >> 2) & 3, fz = f >> 4;
    double W[8][8];
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b)
        W[a][b] = std::max(0.0, 1.0 - std::abs(fx + corner_ox(a) - 4 * corner_ox(b)) / 4.0) *
                  std::max(0.0, 1.0 - std::abs(fy + corner_oy(a) - 4 * corner_oy(b)) / 4.0) *
                  std::max(0.0, 1.0 - std::abs(fz + corner_oz(a) - 4 * corner_oz(b)) / 4.0);
    for (int A = 0; A < 8; ++A)
      for (int c = 0; c < 3; ++c)
        for (int B = 0; B < 8; ++B)
          for (int d = 0; d < 3; ++d) {
            double t = 0.0;
            for (int a = 0; a < 8; ++a) {
              if (W[a][A] == 0.0) continue;
              for (int b = 0; b < 8; ++b)
                if (W[b][B] != 0.0) t += W[a][A] * KE[(3 * a + c) * 24 + 3 * b + d] * W[b][B];
            }
            out[(size_t)f * 576 + (3 * A + c) * 24 + 3 * B + d] = t;
          }
  }
}

extern "C" void tp3d_solver_default_opts(tp3d_solver_opts* o) {
  if (!o) return;
  o->precision = TP3D_PRECISION_FP64;
  o->max_iterations = 2000;
  o->rtol = 1e-10;
  o->pre_sweeps = 1;
  o->post_sweeps = 1;
  o->omega = 0.6;
  o->coarsest_max_dofs = 500;
  o->max_levels = 12;
  o->smoother = 0;
  o->cheb_ratio = 30.0;
  o->power_iterations = 12;
  o->inner_density = 0;
  o->reliable_delta = 0.05;
  o->max_restarts = 3;
  o->fine_operator = 0;
  o->fused_cycle_dofs = 0;
  o->galerkin = 0;
  o->coarse_sweeps = 2;
  o->device_loop = 1;
  o->deep_sweeps = 4;
  o->pdl = 2;
  o->coarse_bf16 = 99;
  o->split_dofs = 16384;
  o->deep_cta = 1;
  o->block_sweeps = 0;
  o->resid_restrict_dofs = 0;
  o->spectra_streams = 1;
  o->cluster_cycle = 1;
  o->fine_slab_depth = 0;
  o->coarse_node_major = 1;
  o->ritz_start = 1;
  o->cheb_ratio_coarse = 0.0;
}

extern "C" int tp3d_solver_create(int nelx, int nely, int nelz, const double* KE_host, const uint8_t* fixed_dofs,
                                  const tp3d_solver_opts* opts, void* stream, tp3d_solver** out) {
  if (!out || !KE_host || !fixed_dofs || nelx < 1 || nely < 1 || nelz < 1) return TP3D_ERR_ARG;
  *out = nullptr;
  tp3d_solver* s = new tp3d_solver();
  if (opts) s->o = *opts;
  else tp3d_solver_default_opts(&s->o);
  s->pdl = s->o.pdl != 0;
  auto fail = [&](int rc, const char* msg) {
    tp3d_set_last_error(msg);
    delete s;
    return rc;
  };
  tp3d_solver_opts& o = s->o;
  if (o.pre_sweeps < 1 || o.pre_sweeps > kMaxCheb || o.post_sweeps < 0 || o.post_sweeps > kMaxCheb ||
      o.max_iterations < 1 || !(o.rtol > 0.0) || o.coarsest_max_dofs < 1 || o.max_levels < 1 ||
      !(o.cheb_ratio > 1.0) || !(o.cheb_ratio_coarse == 0.0 || o.cheb_ratio_coarse > 1.0) ||
      o.power_iterations < 2 || !(o.reliable_delta > 0.0 && o.reliable_delta < 1.0))
    return fail(TP3D_ERR_ARG, "invalid solver options");
  if (o.coarse_sweeps < 0 || o.coarse_sweeps > kMaxCheb) return fail(TP3D_ERR_ARG, "invalid coarse_sweeps");
  if (o.deep_sweeps < 0 || o.deep_sweeps > kMaxCheb) return fail(TP3D_ERR_ARG, "invalid deep_sweeps");
  if (o.block_sweeps < 0 || o.block_sweeps > kMaxCheb) return fail(TP3D_ERR_ARG, "invalid block_sweeps");
  if (o.resid_restrict_dofs < 0) return fail(TP3D_ERR_ARG, "invalid resid_restrict_dofs");
  if (o.pdl < 0 || o.pdl > 3) return fail(TP3D_ERR_ARG, "invalid pdl");
  if (o.split_dofs < 0) return fail(TP3D_ERR_ARG, "invalid split_dofs");
  if (o.coarse_bf16 < 0) return fail(TP3D_ERR_ARG, "invalid coarse_bf16");
  if (o.smoother != 1 && o.pre_sweeps != o.post_sweeps)
    return fail(TP3D_ERR_ARG, "pre_sweeps and post_sweeps must be equal: the Chebyshev V-cycle preconditions CG and "
                              "must stay symmetric");
  if (o.omega <= 0.0) o.omega = 0.6;
  s->mixed = o.precision == TP3D_PRECISION_MIXED;
  const bool mixed = s->mixed;
  s->g = Grid{nelx, nely, nelz};
  s->user = (cudaStream_t)stream;
  if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_in, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_out, cudaEventDisableTiming) != cudaSuccess)
    return fail(TP3D_ERR_CUDA, "stream creation failed");
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, dev);
  for (int i = 0; i < 576; ++i) {
    s->ke64.k[i] = KE_host[i];
    s->ke32.k[i] = (float)KE_host[i];
  }
  s->ke_cls = ke_classes(KE_host, s->kcls64);
  if (o.fine_operator < 0 || o.fine_operator > 2 + kWhtVariants)
    return fail(TP3D_ERR_ARG, "invalid fine_operator option");
  if (o.fine_slab_depth < 0) return fail(TP3D_ERR_ARG, "invalid fine_slab_depth option");
  {
    double m[8][3][3];
    s->wht_ok = o.fine_operator != 1 && wht_blocks_from_ke(KE_host, m);
    for (int t = 0; t < 8; ++t)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          s->wb64.m[t][i][j] = s->wht_ok ? m[t][i][j] : 0.0;
          s->wb32.m[t][i][j] = (float)s->wb64.m[t][i][j];
        }
  }
  s->tile = mixed ? (o.inner_density == 1 ? choose_tile<float, EFromBF16>(s->g, s->nsm)
                                           : choose_tile<float, EFromF32>(s->g, s->nsm))
                  : choose_tile<double, EFromF64>(s->g, s->nsm);
  if (s->tile.tiles_y * s->tile.tiles_x * s->tile.zchunks > kMaxPartials)
    return fail(TP3D_ERR_ARG, "grid too large for the partial-sum buffer");
  // levels
  s->grids.push_back(s->g);
  while ((int)s->grids.size() < o.max_levels) {
    const Grid& f = s->grids.back();
    if (3 * f.nnode() <= o.coarsest_max_dofs) break;
    const Grid c = coarse_grid(f);
    if (c.nx == f.nx && c.ny == f.ny && c.nz == f.nz) break;
    s->grids.push_back(c);
  }
  if (3 * s->grids.back().nnode() > 3000) s->grids.resize(1);  // dense coarsest would be too large
  s->nlev = (int)s->grids.size();
  // first level (>= 1, above the coarsest) small enough for the fused coarse cycle
  s->cyc_L0 = 0;
  if (o.fused_cycle_dofs > 0)
    for (int L = 1; L < s->nlev - 1; ++L)
      if (3 * s->grids[L].nnode() <= o.fused_cycle_dofs) {
        s->cyc_L0 = L;
        break;
      }
  if (s->nlev > kCycleMaxLevels) s->cyc_L0 = 0;

  if (s->cyc_L0 > 0) {
    s->cyc_blocks64 = s->cycle_blocks<double>(s->cyc_L0);
    s->cyc_blocks32 = s->cycle_blocks<float>(s->cyc_L0);
    s->cyc_bar = s->alloc<unsigned int>(2);
    if (!s->cyc_blocks64 || !s->cyc_blocks32 || !s->cyc_bar) s->cyc_L0 = 0;
  }
  s->partials = s->alloc<double>(kMaxPartials);
  s->fin_count = s->alloc<unsigned int>(1);
  if (s->fin_count) cudaMemset(s->fin_count, 0, sizeof(unsigned int));
  if (o.ritz_start) {
    const long long ndof = 3 * s->g.nnode();
    s->rz_q1 = s->alloc<double>(ndof);
    s->rz_q2 = s->alloc<double>(ndof);
    s->rz_part = s->alloc<double>(5 * (size_t)s->grid_blocks(ndof));
    s->rz_coef = s->alloc<double>(2);
    s->rz_gate = s->alloc<int>(1);
    s->rz_count = s->alloc<unsigned int>(1);
    if (s->rz_count) cudaMemset(s->rz_count, 0, sizeof(unsigned int));
  }
  s->loop_passes = s->alloc<unsigned int>(1);
  // The side stream (element chain, coarsest stencil and inverse: the longest
  // chain of the set-up) gets the highest priority, so that its blocks are
  // scheduled ahead of the level builds and power iterations running beside it.
  int prio_lo = 0, prio_hi = 0;
  cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
  if (cudaMallocHost(&s->loop_pass_host, sizeof(unsigned int)) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->st_branch, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithPriority(&s->st_side, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_side_in, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_side_out, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_side_elem, cudaEventDisableTiming) != cudaSuccess)
    return fail(TP3D_ERR_CUDA, "solver setup failed");
  s->state = s->alloc<PcgState>(1);
  unsigned int* cnt = s->alloc<unsigned int>(4);
  if (!s->partials || !s->state || !cnt) return fail(TP3D_ERR_CUDA, "allocation failed");
  if (cudaMallocHost(&s->state_host, 2 * sizeof(PcgState)) != cudaSuccess) return fail(TP3D_ERR_CUDA, "pinned alloc");
  for (int L = 0; L < s->nlev; ++L) {
    uint8_t* f = s->alloc<uint8_t>(s->grids[L].nnode());
    if (!f) return fail(TP3D_ERR_CUDA, "allocation failed");
    s->fix.push_back(f);
  }
  if (s->enter()) return fail(TP3D_ERR_CUDA, "stream ordering failed");
  cudaMemsetAsync(cnt, 0, 4 * sizeof(unsigned int), s->st);
  pack_mask_kernel<<<s->grid_blocks(s->g.nnode()), 256, 0, s->st>>>(s->g.nnode(), fixed_dofs, s->fix[0], cnt);
  // Coarse constraints: a coarse node is fixed when a fixed fine node lies within
  // one fine step of it (dilation), so coarse problems never float even for
  // small clamp patches.
  for (int L = 1; L < s->nlev; ++L)
    coarse_mask_kernel<<<s->grid_blocks(s->grids[L].nnode()), 256, 0, s->st>>>(s->grids[L - 1], s->grids[L],
                                                                                s->fix[L - 1], s->fix[L], 1, cnt + 1);
  if (cudaStreamSynchronize(s->st) != cudaSuccess) return fail(TP3D_ERR_CUDA, "mask setup failed");

  const long long nele = s->g.nele();
  s->E64 = s->alloc<double>(nele);
  if (mixed) {
    if (o.inner_density == 1) s->rho16 = s->alloc<__nv_bfloat16>(nele);
    else s->E32 = s->alloc<float>(nele);
  }
  double ke1[8 * 576];
  coarse_subelement_tables(KE_host, ke1);
  s->KE1 = s->alloc<double>(8 * 576);
  cudaMemcpy(s->KE1, ke1, sizeof(ke1), cudaMemcpyHostToDevice);
  if (o.galerkin < 0 || o.galerkin > 1) return fail(TP3D_ERR_ARG, "invalid galerkin option");
  if (o.galerkin == 0 && s->nlev > 2) {
    std::vector<double> ke2((size_t)64 * 576);
    level2_element_tables(KE_host, ke2.data());
    s->KE2 = s->alloc<double>(64 * 576);
    if (s->KE2) cudaMemcpy(s->KE2, ke2.data(), ke2.size() * sizeof(double), cudaMemcpyHostToDevice);
    s->Kel.assign(s->nlev, nullptr);
    for (int L = 2; L < s->nlev; ++L) s->Kel[L] = s->alloc<double>((size_t)576 * s->grids[L].nele());
  }
  s->A64.assign(s->nlev, nullptr);
  s->S16.assign(s->nlev, nullptr);
  s->SN3.assign(s->nlev, nullptr);
  s->st_pow.assign(s->nlev, nullptr);
  s->ev_pow_in.assign(s->nlev, nullptr);
  s->ev_pow_out.assign(s->nlev, nullptr);
  if ((long long)s->nlev * kSpectraPartials > kMaxPartials) return fail(TP3D_ERR_ARG, "too many levels");
  for (int L = 0; L < s->nlev; ++L)
    if (cudaStreamCreateWithFlags(&s->st_pow[L], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_pow_in[L], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_pow_out[L], cudaEventDisableTiming) != cudaSuccess)
      return fail(TP3D_ERR_CUDA, "solver setup failed");
  s->L64.resize(s->nlev);
  if (mixed) s->L32.resize(s->nlev);
  for (int L = 0; L < s->nlev; ++L) {
    const long long nn = s->grids[L].nnode(), ndof = 3 * nn;
    if (L > 0) s->A64[L] = s->alloc<double>(243 * nn);
    s->coef.push_back(s->alloc<double>(kCoefLen));
    auto& a = s->L64[L];
    a.dinv = s->alloc<double>(ndof);  // FP64 diagonal (the mixed form rounds it)
    if (!mixed) {
      if (L > 0) a.A = s->alloc<double>(243 * nn);
      a.x[0] = s->alloc<double>(ndof); a.x[1] = s->alloc<double>(ndof);
      a.b = s->alloc<double>(ndof); a.r = s->alloc<double>(ndof); a.d = s->alloc<double>(ndof);
    } else {
      auto& b = s->L32[L];
      b.x[0] = s->alloc<float>(ndof); b.x[1] = s->alloc<float>(ndof);
      b.b = s->alloc<float>(ndof); b.r = s->alloc<float>(ndof); b.d = s->alloc<float>(ndof);
      b.dinv = s->alloc<float>(ndof);
      // bf16 stencils with the Chebyshev smoother only: its interval comes from
      // the operator's own power iteration, whereas damped Jacobi's fixed omega
      // leaves omega lambda_max(Dinv A) near 2 with no margin for the rounding.
      // Not on the dense coarsest level, nor inside a fused coarse cycle.
      const bool bf16 = L >= 1 && L <= s->o.coarse_bf16 && s->o.smoother != 1 && L < s->nlev - 1 &&
                        !(s->cyc_L0 > 0 && L >= s->cyc_L0);
      if (bf16) s->S16[L] = s->alloc<__nv_bfloat16>(243 * nn);
      else if (L > 0) b.A = s->alloc<float>(243 * nn);
      // bf16 levels apply their stencil node-major (the cluster or block cycle's
      // levels run from their own node-major rows in shared memory)
      if (bf16 && s->o.coarse_node_major) s->SN3[L] = s->alloc<__nv_bfloat16>((size_t)kNM3Row * nn);
    }
  }
  s->cn = (int)(3 * s->grids.back().nnode());
  if (s->nlev > 1) {
    s->cdense = s->alloc<double>((size_t)s->cn * s->cn);
    s->cinv64 = s->alloc<double>((size_t)s->cn * s->cn);
    if (mixed) s->cinv32 = s->alloc<float>((size_t)s->cn * s->cn);
    s->cstatus = s->alloc<int>(1);
  }
  const long long ndof = 3 * s->g.nnode();
  for (int L = 0; L < s->nlev; ++L) s->pv.push_back(s->alloc<double>(3 * s->grids[L].nnode()));
  s->u64 = s->alloc<double>(ndof);
  if (!mixed) {
    s->K64.u = s->u64;
    s->K64.r = s->alloc<double>(ndof);
    s->K64.p = s->alloc<double>(ndof);
    s->K64.q = s->alloc<double>(ndof);
  } else {
    s->r64 = s->alloc<double>(ndof);
    s->F_capture = s->alloc<double>(ndof);
    s->K32.u = s->alloc<float>(ndof);
    s->K32.r = s->alloc<float>(ndof);
    s->K32.p = s->alloc<float>(ndof);
    s->K32.q = s->alloc<float>(ndof);
  }
  for (void* p : s->allocs)
    if (!p) return fail(TP3D_ERR_CUDA, "allocation failed");
  // the last smoothed level in one block when its operator fits in shared memory
  if (mixed && o.deep_cta && s->nlev >= 3 && s->cyc_L0 == 0) {
    const int L = s->nlev - 2;
    const bool b16 = s->S16[L] != nullptr;
    const long long nn = s->grids[L].nnode(), nnc = s->grids[L + 1].nnode();
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    auto bytes = [&](bool inv) {
      return b16 ? deep_smem_bytes<float, __nv_bfloat16>(nn, nnc, inv) : deep_smem_bytes<float, float>(nn, nnc, inv);
    };
    s->deep_inv_smem = bytes(true) <= (size_t)optin;  // the coarsest inverse too, when it fits
    const size_t smem = bytes(s->deep_inv_smem);
    const int e = b16 ? ensure_dynamic_smem(deep_cycle_kernel<float, __nv_bfloat16>, smem)
                      : ensure_dynamic_smem(deep_cycle_kernel<float, float>, smem);
    if (e == TP3D_OK) {
      if (b16) s->deep_SN = s->alloc<__nv_bfloat16>((size_t)nn * kDeepRow);
      if (!b16 || s->deep_SN) {
        s->deep_L = L;
        s->deep_smem = smem;
      }
    }
    cudaGetLastError();
  }
  // the two last smoothed levels and the coarsest solve as one cluster, when
  // both levels hold bf16 stencils and a cluster of 8 (or 16) CTAs holds them
  if (mixed && o.cluster_cycle && s->deep_L >= 2 && s->deep_SN && s->S16[s->deep_L - 1]) {
    const int L = s->deep_L - 1;
    const int nA = (int)s->grids[L].nnode(), nB = (int)s->grids[L + 1].nnode(), nC = (int)s->grids[L + 2].nnode();
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    for (int C : {8, 16}) {
      const size_t smem = cl_layout(nA, nB, nC, C).total;
      if (smem > (size_t)optin || nC < C) continue;
      if (ensure_dynamic_smem(cluster_cycle_kernel, smem) != TP3D_OK) break;
      if (C > 8 && cudaFuncSetAttribute(cluster_cycle_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                       cudaSuccess)
        break;
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)C);
      cfg.blockDim = dim3(kClThreads);
      cfg.dynamicSmemBytes = smem;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = (unsigned)C;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int nclusters = 0;
      if (cudaOccupancyMaxActiveClusters(&nclusters, cluster_cycle_kernel, &cfg) != cudaSuccess || nclusters < 1)
        continue;
      s->clu_SN = s->alloc<__nv_bfloat16>((size_t)nA * kDeepRow);
      if (s->clu_SN) {
        s->clu_L = L;
        s->clu_C = C;
        s->clu_smem = smem;
      }
      break;
    }
    cudaGetLastError();
  }
  if (cudaStreamSynchronize(s->st) != cudaSuccess || cudaGetLastError() != cudaSuccess)
    return fail(TP3D_ERR_CUDA, "setup failed");
  *out = s;
  return TP3D_OK;
}

extern "C" int tp3d_solver_destroy(tp3d_solver* s) {
  if (!s) return TP3D_OK;
  delete s;
  return TP3D_OK;
}

// lambda_max(Dinv A) of level L by power iteration, then its Chebyshev
// coefficients; all on the device, on the stream `ps` (each level has its own,
// so the levels' iterations, latency-bound on the small levels, overlap one
// another and the builds of the levels after them).  The operators are those of
// the solve's own precision (FP32 in the mixed form: two digits of lambda_max
// suffice).  The first set-up starts from a pseudo-random vector; later ones
// from the previous (normalised) dominant vector, which tracks the slowly
// changing design in fewer steps.

template <typename T>
static int spectra_level(tp3d_solver* s, int L, cudaStream_t ps) {
  const bool warm = s->have_spectra;
  const int N = warm ? std::max(3, s->o.power_iterations / 3) : s->o.power_iterations;
  const long long nn = s->grids[L].nnode(), ndof = 3 * nn;
  const int nb = s->grid_blocks(ndof);
  auto& lv = s->levels<T>()[L];
  T* w[2] = {lv.x[0], lv.x[1]};
  double* pa = s->partials + (size_t)L * kSpectraPartials;
  double* pb = pa + kSpectraPartials / 2;
  std::swap(s->st, ps);  // apply_level launches on s->st
  cudaStream_t st = s->st;
  int rc = TP3D_OK;
  if (warm) {
    if constexpr (sizeof(T) == 8) {
      rc = cuda_status(cudaMemcpyAsync(w[0], s->pv[L], ndof * sizeof(double), cudaMemcpyDeviceToDevice, st));
    } else {
      convert_kernel<double, T><<<nb, 256, 0, st>>>(ndof, s->pv[L], w[0]);
      count_launch();
    }
  } else {
    random_vector_kernel<T><<<s->grid_blocks(nn), 256, 0, st>>>(nn, s->fix[L], w[0]);
    count_launch();
  }
  int cur = 0;
  for (int k = 0; k < N && rc == TP3D_OK; ++k) {
    OpIO<T> io;
    io.u = w[cur];
    io.out = w[1 - cur];
    io.dinv = lv.dinv;
    rc = s->apply_level<T, kModeDinvApply>(L, io);
    cur = 1 - cur;
  }
  if (rc == TP3D_OK) {
    dot_kernel<T><<<nb, 256, 0, st>>>(ndof, w[cur], w[cur], pa, nullptr, nullptr);
    dot_kernel<T><<<nb, 256, 0, st>>>(ndof, w[1 - cur], w[1 - cur], pb, nullptr, nullptr);
    const double ratio = (L >= 1 && s->o.cheb_ratio_coarse > 0.0) ? s->o.cheb_ratio_coarse : s->o.cheb_ratio;
    cheb_setup_kernel<<<1, 256, 0, st>>>(pa, nb, pb, nb, ratio, 1.1, s->coef[L]);
    scale_copy_kernel<T><<<nb, 256, 0, st>>>(ndof, w[cur], s->coef[L] + kCoefLen - 1, s->pv[L]);
    for (int i = 0; i < 4; ++i) count_launch();
    rc = cuda_status(cudaGetLastError());
  }
  std::swap(s->st, ps);
  return rc;
}

// Level L's power iteration on its own stream, after what the solver's stream
// has queued so far (level L's operator); the solver's stream joins all of them
// at the end of the set-up (join_spectra).
static int fork_spectra(tp3d_solver* s, int L) {
  if (s->o.smoother == 1 || L >= s->nlev - 1 + (s->nlev == 1 ? 1 : 0)) return TP3D_OK;
  if (!s->o.spectra_streams)  // in order on the solver's stream
    return s->mixed ? spectra_level<float>(s, L, s->st) : spectra_level<double>(s, L, s->st);
  cudaStream_t ps = s->st_pow[L];
  TP3D_CHECK(cudaEventRecord(s->ev_pow_in[L], s->st));
  TP3D_CHECK(cudaStreamWaitEvent(ps, s->ev_pow_in[L], 0));
  if (int rc = s->mixed ? spectra_level<float>(s, L, ps) : spectra_level<double>(s, L, ps)) return rc;
  TP3D_CHECK(cudaEventRecord(s->ev_pow_out[L], ps));
  return TP3D_OK;
}

static int join_spectra(tp3d_solver* s) {
  if (s->o.smoother == 1) return TP3D_OK;
  for (int L = 0; L < s->nlev - 1 + (s->nlev == 1 ? 1 : 0) && s->o.spectra_streams; ++L)
    TP3D_CHECK(cudaStreamWaitEvent(s->st, s->ev_pow_out[L], 0));
  s->have_spectra = true;
  return TP3D_OK;
}

extern "C" int tp3d_solver_set_density(tp3d_solver* s, const double* rho, double penal) {
  if (!s || !rho || !(penal > 0.0)) return TP3D_ERR_ARG;
  s->penal = penal;
  const bool mixed = s->mixed;
  const long long nele = s->g.nele();
  cudaStream_t st = s->st;
  if (int rc = s->enter()) return rc;
  moduli_kernel<<<s->grid_blocks(nele), 256, 0, st>>>(nele, rho, penal, s->E64, s->E32, s->rho16); count_launch();
  const long long nn0 = s->g.nnode();
  fine_diag_inv_kernel<double, EFromF64><<<s->grid_blocks(nn0), 256, 0, st>>>(s->g, s->ke64, EFromF64{s->E64},
                                                                               s->fix[0], s->L64[0].dinv);
  count_launch();
  if (mixed && s->rho16) {
    fine_diag_inv_kernel<float, EFromBF16><<<s->grid_blocks(nn0), 256, 0, st>>>(
        s->g, s->ke64, EFromBF16{s->rho16, (float)penal}, s->fix[0], s->L32[0].dinv);
    count_launch();
  } else if (mixed) {
    fine_diag_inv_kernel<float, EFromF32><<<s->grid_blocks(nn0), 256, 0, st>>>(s->g, s->ke64, EFromF32{s->E32},
                                                                                s->fix[0], s->L32[0].dinv);
    count_launch();
  }
  TP3D_CHECK_LAUNCH();
  if (!s->fine_chosen) {
    if (int rc = s->choose_fine_form<double>()) return rc;
    if (mixed)
      if (int rc = s->choose_fine_form<float>()) return rc;
    s->fine_chosen = true;
  }
  if (int rc = fork_spectra(s, 0)) return rc;
  // The coarsest inverse (one block) runs on a side stream while the level
  // builds and the power iterations use the rest of the GPU; its status is read
  // after both.
  auto coarsest_gj = [&](cudaStream_t cs) -> int {
    const int L = s->nlev - 1;
    const int n = s->cn;
    TP3D_CHECK(cudaMemsetAsync(s->cdense, 0, (size_t)n * n * sizeof(double), cs));
    dense_from_stencil_kernel<<<s->grid_blocks(s->grids[L].nnode()), 256, 0, cs>>>(s->grids[L], s->A64[L], s->fix[L],
                                                                                    s->cdense);
    count_launch();
    if (n <= kGjRegMaxN) {
      dense_gj_inverse_reg_kernel<<<1, 512, 0, cs>>>(n, s->cdense, s->cinv64, s->cstatus);
      count_launch();
    } else {
      const size_t smem = 2 * (size_t)n * sizeof(double);
      if (smem > 48 * 1024)
        if (int rc = ensure_dynamic_smem(dense_gj_inverse_kernel, smem)) return rc;
      dense_gj_inverse_kernel<<<1, 1024, smem, cs>>>(n, s->cdense, s->cinv64, 0, s->cstatus);
      count_launch();
    }
    if (mixed) {
      convert_kernel<double, float><<<s->grid_blocks((long long)n * n), 256, 0, cs>>>((long long)n * n, s->cinv64,
                                                                                      s->cinv32);
      count_launch();
    }
    TP3D_CHECK_LAUNCH();
    return TP3D_OK;
  };
  // Element matrices of levels >= 2 depend only on the fine moduli: they are
  // built on the side stream while level 1 is built here, and the coarsest
  // level's stencil and dense inverse follow them there.
  const bool elem_chain = s->o.galerkin == 0 && s->nlev > 2;
  const int Lc = s->nlev - 1;
  if (elem_chain) {
    TP3D_CHECK(cudaEventRecord(s->ev_side_in, st));
    TP3D_CHECK(cudaStreamWaitEvent(s->st_side, s->ev_side_in, 0));
    for (int L = 2; L < s->nlev; ++L) {
      const unsigned ne = (unsigned)s->grids[L].nele();
      if (L == 2) elem2_from_fine_kernel<<<ne, 576, 0, s->st_side>>>(s->grids[0], s->grids[2], s->E64, s->KE2, s->Kel[2]);
      else elem_coarsen_kernel<<<ne, 576, 0, s->st_side>>>(s->grids[L - 1], s->grids[L], s->Kel[L - 1], s->Kel[L]);
      count_launch();
    }
    TP3D_CHECK(cudaEventRecord(s->ev_side_elem, s->st_side));
    const Grid& gc = s->grids[Lc];
    const long long nn = gc.nnode();
    stencil_from_elems_kernel<float><<<(unsigned)((nn + 31) / 32), kBuildThreads, 0, s->st_side>>>(
        gc, s->Kel[Lc], s->A64[Lc], s->fix[Lc], nullptr, nullptr);
    stencil_diag_inv_kernel<double><<<s->grid_blocks(nn), 256, 0, s->st_side>>>(gc, s->A64[Lc], s->fix[Lc],
                                                                                 s->L64[Lc].dinv);
    count_launch();
    count_launch();
    if (int rc = coarsest_gj(s->st_side)) return rc;
    TP3D_CHECK(cudaEventRecord(s->ev_side_out, s->st_side));
  }
  for (int L = 1; L < (elem_chain ? Lc : s->nlev); ++L) {
    const Grid& gf = s->grids[L - 1];
    const Grid& gc = s->grids[L];
    const unsigned nb = (unsigned)((gc.nnode() + 31) / 32);
    if (L == 2 && elem_chain) TP3D_CHECK(cudaStreamWaitEvent(st, s->ev_side_elem, 0));
    // the builders also write the packed (apply) layout of the solve's
    // precision (bf16 where the level holds its stencil in bf16)
    float* P32 = mixed && !s->S16[L] ? s->L32[L].A : nullptr;
    double* P64 = mixed ? nullptr : s->L64[L].A;
    // a level applied node-major needs its packed bf16 layout only for the
    // fused residual-restriction kernel
    __nv_bfloat16* N16 = s->SN3[L];
    __nv_bfloat16* P16 = s->S16[L] && (!N16 || 3 * gc.nnode() <= s->o.resid_restrict_dofs) ? s->S16[L] : nullptr;
    bool packed = true;
    if (L == 1) {
      if (s->S16[L]) build_level1_kernel<__nv_bfloat16><<<nb, kBuildThreads, 0, st>>>(gf, gc, s->E64, s->KE1, s->A64[1], s->fix[1], P16, N16);
      else if (mixed) build_level1_kernel<float><<<nb, kBuildThreads, 0, st>>>(gf, gc, s->E64, s->KE1, s->A64[1], s->fix[1], P32, nullptr);
      else build_level1_kernel<double><<<nb, kBuildThreads, 0, st>>>(gf, gc, s->E64, s->KE1, s->A64[1], s->fix[1], P64, nullptr);
    } else if (s->o.galerkin == 0) {
      if (s->S16[L]) stencil_from_elems_kernel<__nv_bfloat16><<<nb, kBuildThreads, 0, st>>>(gc, s->Kel[L], s->A64[L], s->fix[L], P16, N16);
      else if (mixed) stencil_from_elems_kernel<float><<<nb, kBuildThreads, 0, st>>>(gc, s->Kel[L], s->A64[L], s->fix[L], P32, nullptr);
      else stencil_from_elems_kernel<double><<<nb, kBuildThreads, 0, st>>>(gc, s->Kel[L], s->A64[L], s->fix[L], P64, nullptr);
    } else {
      rap_kernel<<<nb, kBuildThreads, 0, st>>>(gf, gc, s->A64[L - 1], s->A64[L]);
      packed = false;
    }
    count_launch();
    const long long nn = gc.nnode();
    stencil_diag_inv_kernel<double><<<s->grid_blocks(nn), 256, 0, st>>>(gc, s->A64[L], s->fix[L], s->L64[L].dinv);
    count_launch();
    if (mixed) {
      convert_kernel<double, float><<<s->grid_blocks(3 * nn), 256, 0, st>>>(3 * nn, s->L64[L].dinv, s->L32[L].dinv);
      count_launch();
      if (!packed && s->S16[L]) {
        stencil_pack_sym_kernel<__nv_bfloat16><<<s->grid_blocks(3 * nn), 256, 0, st>>>(gc, s->A64[L], s->fix[L],
                                                                                      s->S16[L]);
        count_launch();
      } else if (!packed) {
        s->pack_level<float>(L, s->L32[L].A);
      }
      if (s->L64[L].A) s->pack_level<double>(L, s->L64[L].A);  // the mixed form's FP64 fallback
    } else if (!packed) {
      s->pack_level<double>(L, s->L64[L].A);
    }
    if (L == s->deep_L && s->deep_SN) {
      deep_pack_kernel<<<s->grid_blocks(nn * kDeepRow), 256, 0, st>>>(gc, s->A64[L], s->fix[L], s->deep_SN);
      count_launch();
    }
    if (s->SN3[L] && !packed) {  // the builders write the node-major rows themselves
      nm3_pack_kernel<<<s->grid_blocks(nn * kNM3Row), 256, 0, st>>>(gc, s->S16[L], s->SN3[L]);
      count_launch();
    }
    if (L == s->clu_L && s->clu_SN) {
      deep_pack_kernel<<<s->grid_blocks(nn * kDeepRow), 256, 0, st>>>(gc, s->A64[L], s->fix[L], s->clu_SN);
      count_launch();
    }
    TP3D_CHECK_LAUNCH();
    if (int rc = fork_spectra(s, L)) return rc;
  }
  if (s->nlev > 1 && !elem_chain) {
    TP3D_CHECK(cudaEventRecord(s->ev_side_in, st));
    TP3D_CHECK(cudaStreamWaitEvent(s->st_side, s->ev_side_in, 0));
    if (int rc = coarsest_gj(s->st_side)) return rc;
    TP3D_CHECK(cudaEventRecord(s->ev_side_out, s->st_side));
  }
  if (int rc = join_spectra(s)) return rc;
  // the solve waits for the coarsest inverse; its status (shifted attempts,
  // diagonal fallback) stays on the device until tp3d_solver_stats reads it
  if (s->nlev > 1) TP3D_CHECK(cudaStreamWaitEvent(st, s->ev_side_out, 0));
  TP3D_CHECK_LAUNCH();
  s->have_density = true;
  return s->leave();
}

extern "C" int tp3d_solver_solve(tp3d_solver* s, const double* F, double* U, int* iterations, double* relres) {
  if (!s || !F || !U) return TP3D_ERR_ARG;
  if (!s->have_density) {
    tp3d_set_last_error("tp3d_solver_set_density must be called before solve");
    return TP3D_ERR_ARG;
  }
  cudaStream_t st = s->st;
  const long long nn = s->g.nnode(), ndof = 3 * nn;
  if (int e = s->enter()) return e;
  if (s->cyc_bar) TP3D_CHECK(cudaMemsetAsync(s->cyc_bar, 0, 2 * sizeof(unsigned int), st));
  TP3D_CHECK(cudaMemcpyAsync(s->u64, U, ndof * sizeof(double), cudaMemcpyDeviceToDevice, st));
  zero_fixed_kernel<<<s->grid_blocks(nn), 256, 0, st>>>(nn, s->u64, s->fix[0]); count_launch();
  s->last_updates = 0;
  s->last_restarts = 0;
  int rc = s->mixed ? s->solve_mixed(F) : s->solve64(F);
  if (rc < 0 && rc != TP3D_ERR_NONFINITE) return rc;
  TP3D_CHECK(cudaMemcpyAsync(U, s->u64, ndof * sizeof(double), cudaMemcpyDeviceToDevice, st));
  TP3D_CHECK(cudaStreamSynchronize(st));
  if (int e = s->leave()) return e;
  if (iterations) *iterations = s->last_iters;
  if (relres) *relres = s->last_relres;
  return rc;
}

extern "C" int tp3d_solver_solve_begin(tp3d_solver* s, const double* F, double* U) {
  if (!s || !F || !U) return TP3D_ERR_ARG;
  if (!s->have_density) {
    tp3d_set_last_error("tp3d_solver_set_density must be called before solve");
    return TP3D_ERR_ARG;
  }
  if (s->pending) {
    tp3d_set_last_error("tp3d_solver_solve_end must follow tp3d_solver_solve_begin");
    return TP3D_ERR_ARG;
  }
  if (!s->mixed) {  // the FP64 form reads its residual between restarts: it completes here
    s->pend_rc = tp3d_solver_solve(s, F, U, nullptr, nullptr);
    return s->pend_rc < 0 ? s->pend_rc : TP3D_OK;
  }
  cudaStream_t st = s->st;
  const long long nn = s->g.nnode(), ndof = 3 * nn;
  if (int e = s->enter()) return e;
  if (s->cyc_bar) TP3D_CHECK(cudaMemsetAsync(s->cyc_bar, 0, 2 * sizeof(unsigned int), st));
  TP3D_CHECK(cudaMemcpyAsync(s->u64, U, ndof * sizeof(double), cudaMemcpyDeviceToDevice, st));
  zero_fixed_kernel<<<s->grid_blocks(nn), 256, 0, st>>>(nn, s->u64, s->fix[0]); count_launch();
  s->last_updates = 0;
  s->last_restarts = 0;
  if (int rc = s->solve_mixed_launch(F)) return rc;
  TP3D_CHECK(cudaMemcpyAsync(U, s->u64, ndof * sizeof(double), cudaMemcpyDeviceToDevice, st));
  if (int e = s->leave()) return e;
  s->pending = true;
  s->pend_F = F;
  s->pend_U = U;
  return TP3D_OK;
}

extern "C" int tp3d_solver_solve_end(tp3d_solver* s, int* iterations, double* relres, int* replaced) {
  if (!s) return TP3D_ERR_ARG;
  if (replaced) *replaced = 0;
  int rc = s->pend_rc;
  if (s->pending) {
    s->pending = false;
    cudaStream_t st = s->st;
    const long long ndof = 3 * s->g.nnode();
    bool fb = false;
    // a fallback solve waits for the caller's work queued since begin (it read U)
    rc = s->solve_mixed_finish(s->pend_F, &fb, [&] { return s->enter(); });
    if (fb) {
      if (rc >= 0 || rc == TP3D_ERR_NONFINITE)
        TP3D_CHECK(cudaMemcpyAsync(s->pend_U, s->u64, ndof * sizeof(double), cudaMemcpyDeviceToDevice, st));
      TP3D_CHECK(cudaStreamSynchronize(st));
      if (int e = s->leave()) return e;
      if (replaced) *replaced = 1;
    }
    if (rc < 0 && rc != TP3D_ERR_NONFINITE) return rc;
  }
  s->pend_rc = TP3D_OK;
  if (iterations) *iterations = s->last_iters;
  if (relres) *relres = s->last_relres;
  return rc;
}

extern "C" int tp3d_solver_apply_f64(tp3d_solver* s, const double* u, double* y) {
  if (!s || !u || !y || !s->have_density) return TP3D_ERR_ARG;
  if (int rc = s->enter()) return rc;
  OpIO<double> io;
  io.u = u;
  io.out = y;
  if (int rc = s->fine<double, kModeApply>(io)) return rc;
  return s->leave();
}

extern "C" int tp3d_solver_apply_f32(tp3d_solver* s, const float* u, float* y) {
  if (!s || !u || !y || !s->have_density || !s->mixed) return TP3D_ERR_ARG;
  if (int rc = s->enter()) return rc;
  OpIO<float> io;
  io.u = u;
  io.out = y;
  if (int rc = s->fine<float, kModeApply>(io)) return rc;
  return s->leave();
}

// Coarse level L's operator as the V-cycle applies it (mixed form, FP32
// vectors of 3 x the level's nodes): y = A_L u on the free DOFs, u on fixed ones.
extern "C" int tp3d_solver_apply_level_f32(tp3d_solver* s, int level, const float* u, float* y) {
  if (!s || !u || !y || !s->have_density || !s->mixed || level < 1 || level >= s->nlev - 1) return TP3D_ERR_ARG;
  if (int rc = s->enter()) return rc;
  OpIO<float> io;
  io.u = u;
  io.out = y;
  if (int rc = s->apply_level<float, kModeApply>(level, io)) return rc;
  return s->leave();
}

// Average duration of one fine-operator launch (Apply mode) over back-to-back
// launches with cold inputs (see time_fine_cold).
extern "C" int tp3d_solver_time_apply(tp3d_solver* s, int fp32, int launches, double* ms_per_launch) {
  if (!s || !ms_per_launch || launches < 1 || !s->have_density) return TP3D_ERR_ARG;
  if (fp32 && !s->mixed) return TP3D_ERR_ARG;
  if (int rc = s->enter()) return rc;
  const int rc = fp32 ? s->time_fine_cold<float>(launches, ms_per_launch)
                      : s->time_fine_cold<double>(launches, ms_per_launch);
  if (rc) return rc;
  return s->leave();
}

extern "C" int tp3d_solver_time_level(tp3d_solver* s, int level, int fp32, int launches, double* ms_per_launch,
                                      double* bytes_per_launch) {
  if (!s || !ms_per_launch || !bytes_per_launch || launches < 1 || !s->have_density || level < 0 ||
      level >= s->nlev - (s->nlev > 1 ? 1 : 0))
    return TP3D_ERR_ARG;
  if (fp32 && !s->mixed) return TP3D_ERR_ARG;
  if (int rc = s->enter()) return rc;
  if (!fp32 && s->mixed)
    if (int rc = s->ensure_fp64_buffers()) return rc;
  const int rc = fp32 ? s->time_level_cold<float>(level, launches, ms_per_launch, bytes_per_launch)
                      : s->time_level_cold<double>(level, launches, ms_per_launch, bytes_per_launch);
  if (rc) return rc;
  return s->leave();
}

// Smoothing degrees by measurement, a coordinate search from the current
// setting: the deeper levels' degree (2, 4, 6), then level 1's (1, 2, 3) with
// the best of those, then the fine level's (1, 2).  The cost of a candidate is
// its solve of K U = F from U0:
//   criterion 0 (latency, one design on the GPU): the faster of two timed
//     solves (after a first one that captures the iteration graph), on the host
//     clock around the whole solve, its host wait included;
//   criterion 1 (throughput, designs sharing the GPU): the solve's algorithmic
//     bytes, CG iterations times the bytes of one iteration (one solve).
// The cheapest candidate that converged without the mixed form's FP64
// fallback is kept.  The choice is cached per process for the grid, precision
// and criterion; a later call applies it without solving.
extern "C" int tp3d_solver_autotune(tp3d_solver* s, const double* F, const double* U0, int criterion,
                                    double* report, int nreport) {
  if (!s || !F || !U0 || (nreport > 0 && !report)) return TP3D_ERR_ARG;
  if (!s->have_density) {
    tp3d_set_last_error("tp3d_solver_set_density must be called before autotune");
    return TP3D_ERR_ARG;
  }
  if (s->o.smoother == 1) {
    tp3d_set_last_error("autotune searches Chebyshev degrees; the damped-Jacobi smoother has none");
    return TP3D_ERR_ARG;
  }
  if (criterion != 0 && criterion != 1) {
    tp3d_set_last_error("autotune criterion must be 0 (solve time) or 1 (solve bytes)");
    return TP3D_ERR_ARG;
  }
  const DegreeKey key{s->g.nx, s->g.ny, s->g.nz, (s->mixed ? 1 : 0) + 2 * criterion};
  auto apply = [&](const Degrees& d) {
    s->o.pre_sweeps = s->o.post_sweeps = d.fine;
    s->o.coarse_sweeps = d.coarse;
    s->o.deep_sweeps = d.deep;
    s->o.block_sweeps = 0;
    s->drop_graphs();
  };
  std::vector<double> rep(10, 0.0);
  {
    std::lock_guard<std::mutex> lk(degree_mu());
    auto it = degree_cache().find(key);
    if (it != degree_cache().end()) {
      apply(it->second);
      s->tuned = 2;
      rep = {(double)it->second.fine, (double)it->second.coarse, (double)it->second.deep, 0, 0, 0, 1,
             (double)criterion, 0, 0};
      for (int i = 0; i < std::min<int>(nreport, (int)rep.size()); ++i) report[i] = rep[i];
      return TP3D_OK;
    }
  }
  const long long ndof = 3 * s->g.nnode();
  double* U = nullptr;
  if (cudaMalloc(&U, ndof * sizeof(double)) != cudaSuccess) {
    tp3d_set_last_error("autotune: allocation failed");
    return TP3D_ERR_CUDA;
  }
  struct Free {
    double* p;
    ~Free() { cudaFree(p); }
  } guard{U};
  const Degrees start{s->o.pre_sweeps, s->pre_sweeps(1), s->pre_sweeps(2)};
  // U0 and F may still be in flight on the caller's stream: the copies below
  // run on the solver's stream, so order it after the caller's work first
  if (int e = s->enter()) return e;
  auto run = [&](double* sec) -> int {
    TP3D_CHECK(cudaMemcpyAsync(U, U0, ndof * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
    const auto t0 = std::chrono::steady_clock::now();
    int it = 0;
    double rr = 0.0;
    const int rc = tp3d_solver_solve(s, F, U, &it, &rr);
    *sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rc == TP3D_OK && s->last_fallback) return TP3D_NOT_CONVERGED;
    return rc;
  };
  std::map<std::tuple<int, int, int>, double> seen;
  int tried = 0;
  int last_cost_iters = 0;
  double last_cost_bytes = 0.0;
  // time of a candidate (infinite if it did not converge); <0 on a CUDA error
  auto measure = [&](const Degrees& d, double* t) -> int {
    auto k = std::make_tuple(d.fine, d.coarse, d.deep);
    auto it = seen.find(k);
    if (it != seen.end()) {
      *t = it->second;
      return TP3D_OK;
    }
    apply(d);
    double t1 = 0.0, t2 = 0.0, t3 = 0.0;
    int rc = run(&t1);
    if (criterion == 0) {
      if (rc == TP3D_OK) rc = run(&t2);
      if (rc == TP3D_OK) rc = run(&t3);
    }
    ++tried;
    if (rc < 0 && rc != TP3D_ERR_NONFINITE) return rc;
    const double bytes = (double)s->last_iters * (s->mixed ? s->K32.graph_bytes : s->K64.graph_bytes);
    *t = rc != TP3D_OK ? INFINITY : criterion == 0 ? std::min(t2, t3) * 1e3 : bytes * 1e-9;
    last_cost_iters = s->last_iters;
    last_cost_bytes = s->mixed ? s->K32.graph_bytes : s->K64.graph_bytes;
    seen[k] = *t;
    return TP3D_OK;
  };
  Degrees best_d = start;
  double best = INFINITY, t_start = INFINITY;
  if (int rc = measure(start, &t_start)) return rc;
  best = t_start;
  for (int pass = 0; pass < 3; ++pass) {
    const std::vector<int> values = pass == 0 ? std::vector<int>{2, 4, 6}
                                    : pass == 1 ? std::vector<int>{1, 2, 3} : std::vector<int>{1, 2};
    const Degrees base = best_d;
    for (int v : values) {
      Degrees d = base;
      (pass == 0 ? d.deep : pass == 1 ? d.coarse : d.fine) = v;
      double t = 0.0;
      if (int rc = measure(d, &t)) return rc;
      if (t < best) {
        best = t;
        best_d = d;
      }
    }
  }
  apply(best_d);
  s->tuned = 1;
  {
    std::lock_guard<std::mutex> lk(degree_mu());
    degree_cache()[key] = best_d;
  }
  rep = {(double)best_d.fine, (double)best_d.coarse, (double)best_d.deep, best, t_start, (double)tried,
         0, (double)criterion, (double)last_cost_iters, last_cost_bytes};
  for (int i = 0; i < std::min<int>(nreport, (int)rep.size()); ++i) report[i] = rep[i];
  return TP3D_OK;
}

extern "C" int tp3d_solver_ritz_start(tp3d_solver* s, const double* F, double* U, double* U_prev, int have_prev) {
  if (!s || !F || !U || !U_prev || !s->have_density) return TP3D_ERR_ARG;
  if (!s->rz_q1) {
    tp3d_set_last_error("the solver was created without ritz_start");
    return TP3D_ERR_ARG;
  }
  if (int rc = s->enter()) return rc;
  if (int rc = s->ritz_start(F, U, U_prev, have_prev, nullptr)) return rc;
  return s->leave();
}

extern "C" int tp3d_warm_start(double* U, double* U_prev, long long n, int have_prev, void* stream) {
  if (!U || !U_prev || n < 0) return TP3D_ERR_ARG;
  if (n == 0) return TP3D_OK;
  const int nb = (int)std::min<long long>((n + 255) / 256, 1184);
  warm_start_kernel<<<nb, 256, 0, (cudaStream_t)stream>>>(n, U, U_prev, have_prev);
  count_launch();
  TP3D_CHECK_LAUNCH();
  return TP3D_OK;
}

extern "C" int tp3d_solver_stats(tp3d_solver* s, double* out, int n) {
  if (!s || !out) return TP3D_ERR_ARG;
  std::vector<double> lam(s->nlev, 0.0);
  if (s->have_density && s->o.smoother != 1) {
    cudaStreamSynchronize(s->st);
    for (int L = 0; L < s->nlev; ++L) cudaMemcpy(&lam[L], s->coef[L] + 1, sizeof(double), cudaMemcpyDeviceToHost);
  }
  int gj_status = 0;
  if (s->have_density && s->nlev > 1) {
    cudaStreamSynchronize(s->st_side);
    cudaMemcpy(&gj_status, s->cstatus, sizeof(int), cudaMemcpyDeviceToHost);
  }
  const bool coarse_fallback = gj_status == kGjFallback;
  std::vector<double> v = {(double)s->nlev, (double)s->last_iters, (double)s->last_updates, s->last_relres,
                           (double)s->last_restarts, (double)s->cn, (double)s->tile.TY, (double)s->tile.TX,
                           (double)s->tile.ZC, coarse_fallback ? 1.0 : 0.0, lam.empty() ? 0.0 : lam[0],
                           s->last_floor ? 1.0 : 0.0, s->last_fallback ? 1.0 : 0.0,
                           s->use_wht64 ? 1.0 + s->wt64.variant : 0.0,
                           s->mixed ? (s->use_wht32 ? 1.0 + s->wt32.variant : 0.0) : -1.0,
                           (double)s->cyc_L0, (s->mixed ? s->K32.loop : s->K64.loop) ? 1.0 : 0.0,
                           s->pdl ? (double)s->o.pdl : 0.0,
                           (double)std::count_if(s->S16.begin(), s->S16.end(), [](const void* p) { return p; }),
                           (double)gj_status, (double)s->deep_L,
                           s->mixed ? s->K32.graph_bytes : s->K64.graph_bytes,
                           (double)(s->mixed ? s->K32.graph_kernels : s->K64.graph_kernels),
                           (double)s->tuned, (double)s->o.pre_sweeps, (double)s->pre_sweeps(1),
                           (double)s->pre_sweeps(2),
                           (double)(s->mixed ? (s->use_wht32 ? s->wt32.ZC : 0) : (s->use_wht64 ? s->wt64.ZC : 0)),
                           (double)(s->mixed ? (s->use_wht32 ? s->wt32.nthr : 0) : (s->use_wht64 ? s->wt64.nthr : 0)),
                           (double)s->clu_L, (double)s->clu_C,
                           (double)(s->mixed ? (s->use_wht32 ? s->wt32.TY : 0) : (s->use_wht64 ? s->wt64.TY : 0)),
                           (double)(s->mixed ? (s->use_wht32 ? s->wt32.TX : 0) : (s->use_wht64 ? s->wt64.TX : 0))};
  const int m = std::min<int>(n, (int)v.size());
  for (int i = 0; i < m; ++i) out[i] = v[i];
  return m;
}

// ---------------------------------------------------------------------------
// A projection stage of the SIMP loop as one CUDA graph.
//
// The loop body of pytopo3d/core/optimizer.py:578-696 (warm start, moduli and
// multigrid set-up, the solves, sensitivities, OC bisection, re-projection) is
// captured once per stage into the body of a WHILE node whose condition a
// kernel sets at the end of every pass: change > tolx and the stage's
// iteration limit not reached (optimizer.py:578).  Each solve's CG loop is a
// nested WHILE node (the FP64 form's restart loop one more).  One launch runs
// the stage; the host reads the per-iteration record once.  Where the host
// path would have decided differently inside a solve (the mixed form's FP64
// fallback; an FP64 solve the host path reports as failed) the pass raises the
// abort flag: the rest of the iteration is skipped (an IF node), the
// warm-started initial guesses are kept in U_bak, the loop ends, and the
// caller runs that iteration on the host path before launching again.
// ---------------------------------------------------------------------------
struct tp3d_stage {
  cudaGraphExec_t exec = nullptr;
  tp3d_solver* s = nullptr;
  int* counters = nullptr;
  long long body_kernels = 0, loop_kernels = 0;
};

namespace {

// Adds a conditional IF node on handle h after the work captured so far on
// `cs` and starts capturing its body on `body_st`.
int begin_if_body(cudaStream_t cs, cudaStream_t body_st, cudaGraphConditionalHandle h) {
  cudaStreamCaptureStatus st;
  cudaGraph_t capg = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  TP3D_CHECK(cudaStreamGetCaptureInfo(cs, &st, nullptr, &capg, &deps, &nd));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeIf;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  TP3D_CHECK(cudaGraphAddNode(&node, capg, deps, nd, &cp));
  TP3D_CHECK(cudaStreamUpdateCaptureDependencies(cs, &node, 1, cudaStreamSetCaptureDependencies));
  TP3D_CHECK(cudaStreamBeginCaptureToGraph(body_st, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal));
  return TP3D_OK;
}

int stage_body(tp3d_solver* s, const tp3d_stage_desc* d, cudaStream_t cs, cudaStream_t cs2,
               cudaGraphConditionalHandle h_stage, long long* body_kernels) {
  const Grid& g = s->g;
  const long long ndof = 3 * g.nnode(), nele = g.nele();
  const int nb = s->grid_blocks(ndof);
  int* ctr = d->counters;
  if (s->rz_q1) {
    // Rayleigh-Ritz start: it needs the new operator, so the set-up comes first
    // (the host path's order); the history test is read from the counters
    if (int rc = tp3d_solver_set_density(s, d->rho_p, d->penal)) return rc;
    for (int k = 0; k < d->ncases; ++k) {
      double* U = d->U + (size_t)k * ndof;
      if (int rc = s->enter()) return rc;
      if (int rc = s->ritz_start(d->F + (size_t)k * ndof, U, d->U_prev + (size_t)k * ndof, 0, ctr)) return rc;
      if (int rc = s->leave()) return rc;
      TP3D_CHECK(cudaMemcpyAsync(d->U_bak + (size_t)k * ndof, U, ndof * sizeof(double), cudaMemcpyDeviceToDevice,
                                 cs));
    }
  } else {
    for (int k = 0; k < d->ncases; ++k) {
      double* U = d->U + (size_t)k * ndof;
      warm_start_dev_kernel<<<nb, 256, 0, cs>>>(ndof, U, d->U_prev + (size_t)k * ndof, ctr);
      TP3D_CHECK(cudaMemcpyAsync(d->U_bak + (size_t)k * ndof, U, ndof * sizeof(double), cudaMemcpyDeviceToDevice,
                                 cs));
    }
    *body_kernels += d->ncases;
    if (int rc = tp3d_solver_set_density(s, d->rho_p, d->penal)) return rc;
  }
  for (int k = 0; k < d->ncases; ++k)
    if (int rc = s->solve_into_capture(d->F + (size_t)k * ndof, d->U + (size_t)k * ndof, ctr + kStAbort,
                                       ctr + kStCg))
      return rc;
  // the iteration's second half, skipped when a solve raised the abort flag
  cudaGraphConditionalHandle hg = 0;
  {
    cudaStreamCaptureStatus st;
    cudaGraph_t capg = nullptr;
    TP3D_CHECK(cudaStreamGetCaptureInfo(cs, &st, nullptr, &capg, nullptr, nullptr));
    TP3D_CHECK(cudaGraphConditionalHandleCreate(&hg, capg, 0, cudaGraphCondAssignDefault));
  }
  stage_gate_kernel<<<1, 1, 0, cs>>>(hg, ctr);
  if (int rc = begin_if_body(cs, cs2, hg)) return rc;
  int rc = TP3D_OK;
  for (int k = 0; k < d->ncases && rc == TP3D_OK; ++k) {
    rc = tp3d_sensitivity(g.nx, g.ny, g.nz, d->rmin, d->U + (size_t)k * ndof, d->KE_host, d->rho_p, d->dproj,
                          d->Hs, d->free_mask, d->penal, d->ce, k == 0 ? d->dc_dx : d->dc_acc, d->dv_dx,
                          d->c + std::min(k, 1), d->sens_scratch, cs2);
    if (rc == TP3D_OK && k > 0) {
      accumulate_case_kernel<<<s->grid_blocks(nele), 256, 0, cs2>>>(nele, d->dc_dx, d->dc_acc, d->c);
      ++*body_kernels;
    }
  }
  if (rc == TP3D_OK)
    rc = tp3d_oc_update(g.nx, g.ny, g.nz, d->rmin, d->x, d->dc_dx, d->dv_dx, d->Hs, d->solid, d->void_, d->move,
                        d->target_free_volume, d->beta, d->eta, d->max_bisection, d->bisection_tol, d->x_new,
                        d->rho_new, d->oc_stats, d->oc_scratch, cs2);
  if (rc == TP3D_OK &&
      cudaMemcpyAsync(d->x, d->x_new, nele * sizeof(double), cudaMemcpyDeviceToDevice, cs2) != cudaSuccess)
    rc = TP3D_ERR_CUDA;
  if (rc == TP3D_OK)
    rc = tp3d_filter_project(g.nx, g.ny, g.nz, d->rmin, d->x, d->Hs, d->beta, d->eta, d->solid, d->void_, d->rho_f,
                             d->rho_p, d->dproj, cs2);
  cudaGraph_t out = nullptr;
  if (cudaStreamEndCapture(cs2, &out) != cudaSuccess && rc == TP3D_OK) rc = TP3D_ERR_CUDA;
  if (rc) return rc;
  stage_next_kernel<<<1, 1, 0, cs>>>(h_stage, ctr, d->c, d->oc_stats, d->record, d->tolx);
  *body_kernels += 4 + 2 * d->ncases;  // gate, next, OC, projection, sensitivity launches
  TP3D_CHECK_LAUNCH();
  return TP3D_OK;
}

}  // namespace

namespace {
// What a capture needs but may not create while capturing: streams, the
// restart state, and the mixed form's FP64 fallback hierarchy (so that the
// captured set-up refreshes it exactly as the host path's does).
int stage_prepare(tp3d_solver* s) {
  if (!s->restart_state) s->restart_state = s->alloc<double>(4);
  if (!s->restart_state) return TP3D_ERR_CUDA;
  if (!s->st_loop) TP3D_CHECK(cudaStreamCreateWithFlags(&s->st_loop, cudaStreamNonBlocking));
  if (!s->st_restart) TP3D_CHECK(cudaStreamCreateWithFlags(&s->st_restart, cudaStreamNonBlocking));
  if (s->mixed) {
    if (int e = s->enter()) return e;
    if (int e = s->ensure_fp64_buffers()) return e;
    if (int e = s->leave()) return e;
  }
  return TP3D_OK;
}

bool stage_desc_ok(const tp3d_stage_desc* d) {
  return d && d->ncases >= 1 && d->F && d->U && d->U_prev && d->U_bak && d->x && d->x_new && d->rho_f && d->rho_p &&
         d->dproj && d->rho_new && d->dc_dx && d->dv_dx && d->ce && d->c && d->Hs && d->free_mask && d->KE_host &&
         d->sens_scratch && d->oc_scratch && d->oc_stats && d->record && d->counters &&
         (d->ncases == 1 || d->dc_acc);
}
}  // namespace

extern "C" int tp3d_stage_capture(tp3d_solver* s, const tp3d_stage_desc* d, void* stream, tp3d_stage** out) {
  if (!s || !out || !stage_desc_ok(d)) return TP3D_ERR_ARG;
  if (!s->have_density || !s->fine_chosen || s->pending) {
    tp3d_set_last_error("tp3d_stage_capture: run one loop body on the host path first");
    return TP3D_ERR_ARG;
  }
  (void)stream;
  *out = nullptr;
  if (int e = stage_prepare(s)) return e;
  cudaStream_t cs = nullptr, cs2 = nullptr;
  TP3D_CHECK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  TP3D_CHECK(cudaStreamCreateWithFlags(&cs2, cudaStreamNonBlocking));
  TP3D_CHECK(cudaDeviceSynchronize());
  auto* gph = new tp3d_stage();
  gph->s = s;
  gph->counters = d->counters;
  int rc = TP3D_OK;
  for (int attempt = 0; attempt < 2; ++attempt) {
    cudaGraph_t G = nullptr;
    cudaGraphConditionalHandle hs = 0;
    rc = TP3D_OK;
    if (cudaGraphCreate(&G, 0) != cudaSuccess ||
        cudaGraphConditionalHandleCreate(&hs, G, 1, cudaGraphCondAssignDefault) != cudaSuccess)
      rc = TP3D_ERR_CUDA;
    cudaGraphNodeParams cp = {};
    cudaGraphNode_t wnode;
    if (rc == TP3D_OK) {
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = hs;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      if (cudaGraphAddNode(&wnode, G, nullptr, 0, &cp) != cudaSuccess) rc = TP3D_ERR_CUDA;
    }
    bool capturing = false;
    cudaStream_t saved_user = s->user;
    if (rc == TP3D_OK) {
      capturing = cudaStreamBeginCaptureToGraph(cs, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      if (!capturing) rc = TP3D_ERR_CUDA;
    }
    if (rc == TP3D_OK) {
      s->user = cs;
      long long nk = 0;
      t_capture_count = &nk;
      rc = stage_body(s, d, cs, cs2, hs, &gph->body_kernels);
      t_capture_count = nullptr;
      gph->body_kernels += nk;
      gph->loop_kernels = s->stage_loop_kernels;
      s->user = saved_user;
    }
    if (capturing) {
      cudaGraph_t o2 = nullptr;
      if (cudaStreamEndCapture(cs, &o2) != cudaSuccess && rc == TP3D_OK) rc = TP3D_ERR_CUDA;
    }
    if (rc == TP3D_OK && cudaGraphInstantiate(&gph->exec, G, 0) != cudaSuccess) rc = TP3D_ERR_CUDA;
    if (G) cudaGraphDestroy(G);
    cudaGetLastError();
    if (rc == TP3D_OK) break;
    if (gph->exec) cudaGraphExecDestroy(gph->exec);
    gph->exec = nullptr;
    gph->body_kernels = 0;
    if (!s->pdl) break;
    s->pdl = false;  // retry in plain stream order
  }
  cudaStreamDestroy(cs);
  cudaStreamDestroy(cs2);
  if (rc) {
    delete gph;
    if (!*tp3d_last_error()) tp3d_set_last_error("stage graph capture failed");
    return rc;
  }
  *out = gph;
  return TP3D_OK;
}

extern "C" int tp3d_stage_run(tp3d_stage* g, void* stream, int* iterations, int* aborted) {
  if (!g || !g->exec) return TP3D_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  TP3D_CHECK(cudaGraphLaunch(g->exec, st));
  int c[kStCount] = {};
  TP3D_CHECK(cudaMemcpyAsync(c, g->counters, sizeof(c), cudaMemcpyDeviceToHost, st));
  TP3D_CHECK(cudaStreamSynchronize(st));
  if (iterations) *iterations = c[kStIter];
  if (aborted) *aborted = c[kStAbort];
  return TP3D_OK;
}

extern "C" int tp3d_stage_count_launches(tp3d_stage* g, long long passes, long long cg_iterations) {
  if (!g) return TP3D_ERR_ARG;
  add_launches(passes * g->body_kernels + cg_iterations * g->loop_kernels);
  return TP3D_OK;
}

extern "C" int tp3d_stage_destroy(tp3d_stage* g) {
  if (!g) return TP3D_OK;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  delete g;
  return TP3D_OK;
}

// ---------------------------------------------------------------------------
// Many designs in one graph launch: each design's loop body (as in the stage
// graph above, its own solver and buffers) in a WHILE node of its own, all of
// them parallel branches of one graph.  One launch advances every design by up
// to its counters' iteration limit; the designs share nothing but the GPU, so
// their kernels overlap as the graph's branches allow.  No host thread drives
// a design while the graph runs.
// ---------------------------------------------------------------------------
struct tp3d_batch {
  cudaGraphExec_t exec = nullptr;
  std::vector<long long> body_kernels, loop_kernels;
};

extern "C" int tp3d_batch_capture(tp3d_solver* const* solvers, const tp3d_stage_desc* descs, int n, void* stream,
                                  tp3d_batch** out) {
  if (!solvers || !descs || !out || n < 1) return TP3D_ERR_ARG;
  (void)stream;
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    tp3d_solver* s = solvers[i];
    if (!s || !stage_desc_ok(&descs[i])) return TP3D_ERR_ARG;
    if (!s->have_density || !s->fine_chosen || s->pending) {
      tp3d_set_last_error("tp3d_batch_capture: run one loop body of every design on the host path first");
      return TP3D_ERR_ARG;
    }
    if (int e = stage_prepare(s)) return e;
  }
  std::vector<cudaStream_t> sts(3 * n + 1, nullptr);
  std::vector<cudaEvent_t> evs(2 * n, nullptr);
  for (auto& st : sts) TP3D_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  for (auto& ev : evs) TP3D_CHECK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  TP3D_CHECK(cudaDeviceSynchronize());
  auto* b = new tp3d_batch();
  b->body_kernels.assign(n, 0);
  b->loop_kernels.assign(n, 0);
  int rc = TP3D_OK;
  for (int attempt = 0; attempt < 2; ++attempt) {
    rc = TP3D_OK;
    cudaStream_t root = sts[0];
    cudaGraph_t G = nullptr;
    if (cudaStreamBeginCapture(root, cudaStreamCaptureModeThreadLocal) != cudaSuccess) rc = TP3D_ERR_CUDA;
    for (int i = 0; i < n && rc == TP3D_OK; ++i) {
      tp3d_solver* s = solvers[i];
      cudaStream_t br = sts[1 + 3 * i], body = sts[2 + 3 * i], ifs = sts[3 + 3 * i];
      // fork a branch for design i from the graph's start (every branch waits on
      // the same fork event, so no branch depends on another) and add its WHILE
      // node there
      if (i == 0 && cudaEventRecord(evs[0], root) != cudaSuccess) {
        rc = TP3D_ERR_CUDA;
        break;
      }
      if (cudaStreamWaitEvent(br, evs[0], 0) != cudaSuccess) {
        rc = TP3D_ERR_CUDA;
        break;
      }
      cudaStreamCaptureStatus cst;
      cudaGraph_t capg = nullptr;
      const cudaGraphNode_t* deps = nullptr;
      size_t nd = 0;
      cudaGraphConditionalHandle h = 0;
      cudaGraphNodeParams cp = {};
      cudaGraphNode_t wnode;
      if (cudaStreamGetCaptureInfo(br, &cst, nullptr, &capg, &deps, &nd) != cudaSuccess ||
          cudaGraphConditionalHandleCreate(&h, capg, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
        rc = TP3D_ERR_CUDA;
        break;
      }
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      if (cudaGraphAddNode(&wnode, capg, deps, nd, &cp) != cudaSuccess ||
          cudaStreamUpdateCaptureDependencies(br, &wnode, 1, cudaStreamSetCaptureDependencies) != cudaSuccess ||
          cudaStreamBeginCaptureToGraph(body, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        rc = TP3D_ERR_CUDA;
        break;
      }
      cudaStream_t saved_user = s->user;
      s->user = body;
      long long nk = 0;
      t_capture_count = &nk;
      rc = stage_body(s, &descs[i], body, ifs, h, &b->body_kernels[i]);
      t_capture_count = nullptr;
      b->body_kernels[i] += nk;
      b->loop_kernels[i] = s->stage_loop_kernels;
      s->user = saved_user;
      cudaGraph_t ob = nullptr;
      if (cudaStreamEndCapture(body, &ob) != cudaSuccess && rc == TP3D_OK) rc = TP3D_ERR_CUDA;
      if (rc == TP3D_OK && cudaEventRecord(evs[2 * i + 1], br) != cudaSuccess) rc = TP3D_ERR_CUDA;
    }
    // join every branch at the end
    for (int i = 0; i < n && rc == TP3D_OK; ++i)
      if (cudaStreamWaitEvent(root, evs[2 * i + 1], 0) != cudaSuccess) rc = TP3D_ERR_CUDA;
    if (cudaStreamEndCapture(root, &G) != cudaSuccess && rc == TP3D_OK) rc = TP3D_ERR_CUDA;
    if (rc == TP3D_OK && cudaGraphInstantiate(&b->exec, G, 0) != cudaSuccess) rc = TP3D_ERR_CUDA;
    if (G) cudaGraphDestroy(G);
    cudaGetLastError();
    if (rc == TP3D_OK) break;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    b->body_kernels.assign(n, 0);
    bool any_pdl = false;
    for (int i = 0; i < n; ++i) {
      any_pdl = any_pdl || solvers[i]->pdl;
      solvers[i]->pdl = false;  // retry in plain stream order
    }
    if (!any_pdl) break;
  }
  for (auto& st : sts) cudaStreamDestroy(st);
  for (auto& ev : evs) cudaEventDestroy(ev);
  if (rc) {
    delete b;
    if (!*tp3d_last_error()) tp3d_set_last_error("batch graph capture failed");
    return rc;
  }
  *out = b;
  return TP3D_OK;
}

extern "C" int tp3d_batch_run(tp3d_batch* b, void* stream) {
  if (!b || !b->exec) return TP3D_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  TP3D_CHECK(cudaGraphLaunch(b->exec, st));
  TP3D_CHECK(cudaStreamSynchronize(st));
  return TP3D_OK;
}

extern "C" int tp3d_batch_count_launches(tp3d_batch* b, const long long* passes, const long long* cg_iterations) {
  if (!b || !passes || !cg_iterations) return TP3D_ERR_ARG;
  for (size_t i = 0; i < b->body_kernels.size(); ++i)
    add_launches(passes[i] * b->body_kernels[i] + cg_iterations[i] * b->loop_kernels[i]);
  return TP3D_OK;
}

extern "C" int tp3d_batch_destroy(tp3d_batch* b) {
  if (!b) return TP3D_OK;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  delete b;
  return TP3D_OK;
}
