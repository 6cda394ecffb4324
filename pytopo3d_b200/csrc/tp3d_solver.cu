// Multigrid-preconditioned CG on the matrix-free H8 operator, plain FP64 and
// mixed (FP32 inner PCG with BF16 densities inside FP64 iterative refinement).
//
// Replaces, per SIMP iteration, the reference's
//   K = assemble(kron(E, KE)); Kff = K[free][:, free]; Uf = solver_func(Kff, F[free])
// (pytopo3d/core/optimizer.py:584-594; pytopo3d/utils/solver.py:15-73).
//
// One PCG iteration is captured once into a CUDA graph and replayed; every
// kernel reads its scalars (alpha, beta, stop flag) from device memory, so the
// host only polls the stop flag between replays.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "tp3d_mg.cuh"

namespace tp3d {

namespace {
// While a graph is being captured launches are counted into the graph's tally.
thread_local long long* t_capture_count = nullptr;
}
inline void count_launch() {
  if (t_capture_count) ++*t_capture_count;
  else add_launches(1);
}

struct PcgState {
  double rz, pq, rr, bb, alpha, beta, tol2, rr0;
  int done, iters, max_iters, pad;
};

enum FinalizeOp : int { kFinBB = 0, kFinRRInit, kFinRZInit, kFinPQ, kFinRR, kFinRZ };

__global__ void finalize_kernel(const double* __restrict__ partials, int n, PcgState* st, int op, double rtol2) {
  __shared__ double red[32];
  if (op >= kFinPQ && *(volatile int*)&st->done) return;
  const double s = sum_partials(partials, n, red);
  if (threadIdx.x != 0) return;
  switch (op) {
    case kFinBB:
      st->bb = s;
      st->tol2 = rtol2 * s;
      st->iters = 0;
      st->done = (s == 0.0) ? 1 : 0;
      if (!isfinite(s)) st->done = 4;
      break;
    case kFinRRInit:
      st->rr = s;
      st->rr0 = s;
      if (!st->done && s <= st->tol2) st->done = 1;
      if (!isfinite(s)) st->done = 4;
      break;
    case kFinRZInit:
      st->rz = s;
      break;
    case kFinPQ:
      st->pq = s;
      if (!(s > 0.0) || !isfinite(s)) {
        st->done = 3;
      } else {
        st->alpha = st->rz / s;
      }
      break;
    case kFinRR:
      st->rr = s;
      st->iters += 1;
      if (!isfinite(s)) st->done = 4;
      else if (s <= st->tol2) st->done = 1;
      else if (st->iters >= st->max_iters) st->done = 2;
      break;
    case kFinRZ:
      st->beta = s / st->rz;
      st->rz = s;
      break;
  }
}

template <typename T>
__global__ void dot_kernel(long long n, const T* __restrict__ a, const T* __restrict__ b, double* partials,
                           const int* done) {
  if (done && *(volatile const int*)done) return;
  __shared__ double red[32];
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s += (double)a[i] * (double)b[i];
  s = block_sum(s, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// ||b||^2 over free DOFs
__global__ void masked_norm_kernel(long long nn, const double* __restrict__ b, const uint8_t* __restrict__ fix,
                                   double* partials) {
  __shared__ double red[32];
  double s = 0.0;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn; n += (long long)gridDim.x * blockDim.x) {
    const int f = fix[n];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      if (!((f >> c) & 1)) s += b[3 * n + c] * b[3 * n + c];
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

template <typename T>
__global__ void cg_update_kernel(long long n, T* u, const T* __restrict__ p, T* r, const T* __restrict__ q,
                                 const PcgState* st, double* partials) {
  if (*(volatile const int*)&st->done) return;
  __shared__ double red[32];
  const T a = (T)st->alpha;
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    u[i] += a * p[i];
    const T ri = r[i] - a * q[i];
    r[i] = ri;
    s += (double)ri * (double)ri;
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

template <typename T>
__global__ void cg_p_kernel(long long n, const T* __restrict__ z, T* p, const PcgState* st, int init) {
  if (!init && *(volatile const int*)&st->done) return;
  const T b = init ? T(0) : (T)st->beta;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = init ? z[i] : z[i] + b * p[i];
}

__global__ void zero_fixed_kernel(long long nn, double* u, const uint8_t* __restrict__ fix) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn; n += (long long)gridDim.x * blockDim.x) {
    const int f = fix[n];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      if ((f >> c) & 1) u[3 * n + c] = 0.0;
  }
}

__global__ void moduli_kernel(long long n, const double* __restrict__ rho, double penal, double* E,
                              __nv_bfloat16* rho16) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const double r = rho[e];
    const double rp = (penal == 2.0) ? r * r : pow(r, penal);
    E[e] = kEmin + (kE0 - kEmin) * rp;
    if (rho16) rho16[e] = __double2bfloat16(r);
  }
}

// r32 = r64 * s ; u64 += d32 / s
__global__ void scale_down_kernel(long long n, const double* __restrict__ r, double s, float* out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (float)(r[i] * s);
}
__global__ void axpy_up_kernel(long long n, const float* __restrict__ d, double s, double* u) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    u[i] += (double)d[i] * s;
}
template <typename Tsrc, typename Tdst>
__global__ void convert_kernel(long long n, const Tsrc* __restrict__ a, Tdst* b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = (Tdst)a[i];
}
__global__ void dense_shift_kernel(int n, double* D, double shift) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) D[(size_t)i * n + i] += shift;
}

// ---------------------------------------------------------------------------

constexpr int kMaxPartials = 1 << 16;

template <typename T>
struct LevelVec {
  T* x[2] = {nullptr, nullptr};
  T* b = nullptr;
  T* r = nullptr;
  T* dinv = nullptr;
  T* A = nullptr;  // stencil (levels >= 1)
};

template <typename T>
struct PcgVec {
  T *u = nullptr, *r = nullptr, *p = nullptr, *q = nullptr;
  T* z = nullptr;  // points into level-0 storage (set at capture)
  cudaGraphExec_t graph = nullptr;
  long long graph_kernels = 0;
};

struct Tile {
  int TY = 32, TX = 8, ZC = 8, tiles_y = 1, tiles_x = 1, zchunks = 1, threads = 256;
};

Tile choose_tile(const Grid& g, int nsm) {
  const int NX = g.nx + 1, NY = g.ny + 1, NZ = g.nz + 1;
  Tile best;
  double best_cost = 1e300;
  for (int ky = 1; ky <= NY; ++ky) {
    const int TY = (NY + ky - 1) / ky;
    if (TY > 64) continue;
    if (TY < 8 && ky > 1) break;
    for (int kx = 1; kx <= NX; ++kx) {
      const int TX = (NX + kx - 1) / kx;
      if (TY * TX > 256) continue;
      const int thr = ((TY * TX + 31) / 32) * 32;
      // launched thread-slots per node plane, penalise tiny blocks and halo overhead
      const double slots = (double)ky * kx * thr;
      const double halo = (double)(TY + 2) * (TX + 2) / ((double)TY * TX);
      const double cost = slots * (1.0 + 0.35 * (halo - 1.0)) * (thr < 128 ? 1.3 : 1.0);
      if (cost < best_cost) {
        best_cost = cost;
        best.TY = TY;
        best.TX = TX;
        best.tiles_y = ky;
        best.tiles_x = kx;
        best.threads = thr;
      }
      break;  // smallest kx with TY*TX <= 256 for this ky
    }
  }
  // z chunk: aim for >= 3 blocks per SM
  const long long planes = (long long)best.tiles_y * best.tiles_x;
  int zc = 16;
  while (zc > 4 && planes * ((NZ + zc - 1) / zc) < 3LL * nsm) zc /= 2;
  best.ZC = zc;
  best.zchunks = (NZ + zc - 1) / zc;
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
  KEP<double> ke64{};
  KEP<float> ke32{};
  double* KE1 = nullptr;
  double penal = 3.0;
  bool have_density = false;

  std::vector<Grid> grids;
  std::vector<uint8_t*> fix;
  std::vector<double*> A64;  // stencils (index 0 unused)
  int nlev = 1;
  int cn = 0;  // coarsest dense size
  double* cdense = nullptr;
  double* cwork = nullptr;
  double* cinv64 = nullptr;
  float* cinv32 = nullptr;
  int* cstatus = nullptr;

  double* E64 = nullptr;
  __nv_bfloat16* rho16 = nullptr;

  std::vector<LevelVec<double>> L64;
  std::vector<LevelVec<float>> L32;
  PcgVec<double> P64;
  PcgVec<float> P32;
  double* res64 = nullptr;

  double* partials = nullptr;
  PcgState* state = nullptr;
  PcgState* state_host = nullptr;  // two pinned slots
  Tile tile;
  std::vector<void*> allocs;

  // stats of last solve
  int last_iters = 0, last_refinements = 0, last_inner_total = 0;
  double last_relres = 0.0;

  template <typename T>
  T* alloc(size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return nullptr;
    allocs.push_back(p);
    return (T*)p;
  }
  ~tp3d_solver() {
    if (st) cudaStreamSynchronize(st);
    if (P64.graph) cudaGraphExecDestroy(P64.graph);
    if (P32.graph) cudaGraphExecDestroy(P32.graph);
    for (void* p : allocs) cudaFree(p);
    if (state_host) cudaFreeHost(state_host);
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

  // ---------------- fine-level operator ----------------
  template <typename T, int MODE>
  int fine(const T* u, T* out, const T* b, const T* dinv, T omega, double* part, const int* done) {
    const dim3 grid(tile.tiles_y * tile.tiles_x, tile.zchunks);
    const size_t smem = fine_smem_bytes<T>(tile.TY, tile.TX);
    if constexpr (sizeof(T) == 8) {
      FineParams<double, EFromF64> p;
      p.ke = ke64;
      p.g = g;
      p.TY = tile.TY; p.TX = tile.TX; p.ZC = tile.ZC; p.tiles_y = tile.tiles_y; p.tiles_x = tile.tiles_x;
      p.u = u; p.fix = fix[0]; p.esrc = EFromF64{E64}; p.out = out; p.b = b; p.dinv = dinv; p.omega = omega;
      p.partials = part; p.done = done;
      fine_apply_kernel<double, MODE, EFromF64><<<grid, tile.threads, smem, st>>>(p); count_launch();
    } else {
      FineParams<float, EFromBF16> p;
      p.ke = ke32;
      p.g = g;
      p.TY = tile.TY; p.TX = tile.TX; p.ZC = tile.ZC; p.tiles_y = tile.tiles_y; p.tiles_x = tile.tiles_x;
      p.u = u; p.fix = fix[0]; p.esrc = EFromBF16{rho16, (float)penal}; p.out = out; p.b = b; p.dinv = dinv;
      p.omega = omega; p.partials = part; p.done = done;
      fine_apply_kernel<float, MODE, EFromBF16><<<grid, tile.threads, smem, st>>>(p); count_launch();
    }
    TP3D_CHECK_LAUNCH();
    return TP3D_OK;
  }
  int fine_partials() const { return tile.tiles_y * tile.tiles_x * tile.zchunks; }

  template <typename T>
  std::vector<LevelVec<T>>& levels() {
    if constexpr (sizeof(T) == 8) return L64;
    else return L32;
  }

  // One operator application at level L (mode), returns number of partials written (CgQ only).
  template <typename T, int MODE>
  int apply_level(int L, const T* u, T* out, const T* b, const T* dinv, T omega, double* part, const int* done) {
    if (L == 0) return fine<T, MODE>(u, out, b, dinv, omega, part, done);
    const Grid& gl = grids[L];
    stencil_apply_kernel<T, MODE><<<grid_blocks(gl.nnode()), 256, 0, st>>>(gl, levels<T>()[L].A, fix[L], u, out, b,
                                                                            dinv, omega, part, done); count_launch();
    TP3D_CHECK_LAUNCH();
    return TP3D_OK;
  }

  // V-cycle on level L with right-hand side b; returns the buffer holding x.
  template <typename T>
  T* vcycle(int L, const T* b, const int* done, int* rc) {
    auto& lv = levels<T>()[L];
    const Grid& gl = grids[L];
    const long long ndof = 3 * gl.nnode();
    if (nlev == 1) {  // no hierarchy: Jacobi preconditioner
      jacobi_zero_kernel<T><<<grid_blocks(ndof), 256, 0, st>>>(ndof, b, lv.dinv, T(1), lv.x[0], done); count_launch();
      if (cudaGetLastError() != cudaSuccess) *rc = TP3D_ERR_CUDA;
      return lv.x[0];
    }
    if (L == nlev - 1) {
      const T* inv;
      if constexpr (sizeof(T) == 8) inv = cinv64; else inv = cinv32;
      dense_matvec_kernel<T><<<std::max(1, std::min(cn / 8 + 1, nsm)), 256, 0, st>>>(cn, inv, b, lv.x[0], done); count_launch();
      if (cudaGetLastError() != cudaSuccess) *rc = TP3D_ERR_CUDA;
      return lv.x[0];
    }
    const T om = (T)o.omega;
    int cur = 0;
    jacobi_zero_kernel<T><<<grid_blocks(ndof), 256, 0, st>>>(ndof, b, lv.dinv, om, lv.x[cur], done); count_launch();
    for (int s = 1; s < o.pre_sweeps; ++s) {
      *rc |= apply_level<T, kModeJacobi>(L, lv.x[cur], lv.x[1 - cur], b, lv.dinv, om, nullptr, done);
      cur = 1 - cur;
    }
    *rc |= apply_level<T, kModeResid>(L, lv.x[cur], lv.r, b, nullptr, T(0), nullptr, done);
    auto& lc = levels<T>()[L + 1];
    restrict_kernel<T><<<grid_blocks(grids[L + 1].nnode()), 256, 0, st>>>(gl, grids[L + 1], lv.r, fix[L + 1], lc.b,
                                                                           done); count_launch();
    T* xc = vcycle<T>(L + 1, lc.b, done, rc);
    prolong_add_kernel<T><<<grid_blocks(gl.nnode()), 256, 0, st>>>(gl, grids[L + 1], xc, fix[L], lv.x[cur], done); count_launch();
    for (int s = 0; s < o.post_sweeps; ++s) {
      *rc |= apply_level<T, kModeJacobi>(L, lv.x[cur], lv.x[1 - cur], b, lv.dinv, om, nullptr, done);
      cur = 1 - cur;
    }
    if (cudaGetLastError() != cudaSuccess) *rc = TP3D_ERR_CUDA;
    return lv.x[cur];
  }

  // Enqueue one PCG iteration (captured into a graph).
  template <typename T>
  int pcg_iteration(PcgVec<T>& P) {
    const long long ndof = 3 * g.nnode();
    int* done = &state->done;
    const int nb = grid_blocks(ndof);
    int rc = fine<T, kModeCgQ>(P.p, P.q, nullptr, nullptr, T(0), partials, done);
    finalize_kernel<<<1, 256, 0, st>>>(partials, fine_partials(), state, kFinPQ, 0.0); count_launch();
    cg_update_kernel<T><<<nb, 256, 0, st>>>(ndof, P.u, P.p, P.r, P.q, state, partials); count_launch();
    finalize_kernel<<<1, 256, 0, st>>>(partials, nb, state, kFinRR, 0.0); count_launch();
    T* z = vcycle<T>(0, P.r, done, &rc);
    P.z = z;
    dot_kernel<T><<<nb, 256, 0, st>>>(ndof, P.r, z, partials, done); count_launch();
    finalize_kernel<<<1, 256, 0, st>>>(partials, nb, state, kFinRZ, 0.0); count_launch();
    cg_p_kernel<T><<<nb, 256, 0, st>>>(ndof, z, P.p, state, 0); count_launch();
    TP3D_CHECK_LAUNCH();
    return rc;
  }

  template <typename T>
  int ensure_graph(PcgVec<T>& P) {
    if (P.graph) return TP3D_OK;
    cudaGraph_t gr;
    TP3D_CHECK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    long long nk = 0;
    t_capture_count = &nk;
    int rc = pcg_iteration<T>(P);
    t_capture_count = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &gr);
    P.graph_kernels = nk;
    if (rc || e != cudaSuccess) {
      tp3d_set_last_error("PCG graph capture failed");
      return TP3D_ERR_CUDA;
    }
    e = cudaGraphInstantiate(&P.graph, gr, 0);
    cudaGraphDestroy(gr);
    TP3D_CHECK(e);
    return TP3D_OK;
  }

  // PCG on P.u (initial guess already in P.u, fixed DOFs zero) for right-hand side b.
  template <typename T>
  int pcg(PcgVec<T>& P, const T* b, double rtol, int max_iters, int* iters_out, double* relres_out) {
    const long long ndof = 3 * g.nnode();
    const long long nn = g.nnode();
    const int nb = grid_blocks(ndof);
    int rc = ensure_graph<T>(P);
    if (rc) return rc;
    // host-written constants
    PcgState init{};
    init.max_iters = max_iters;
    TP3D_CHECK(cudaMemcpyAsync(state, &init, sizeof(PcgState), cudaMemcpyHostToDevice, st));
    // ||b||^2 over free DOFs
    if constexpr (sizeof(T) == 8) {
      masked_norm_kernel<<<grid_blocks(nn), 256, 0, st>>>(nn, b, fix[0], partials); count_launch();
      finalize_kernel<<<1, 256, 0, st>>>(partials, grid_blocks(nn), state, kFinBB, rtol * rtol); count_launch();
    } else {
      // b is already masked (built from a masked FP64 residual)
      dot_kernel<T><<<nb, 256, 0, st>>>(ndof, b, b, partials, nullptr); count_launch();
      finalize_kernel<<<1, 256, 0, st>>>(partials, nb, state, kFinBB, rtol * rtol); count_launch();
    }
    // r = b - A u
    rc |= fine<T, kModeResid>(P.u, P.r, b, nullptr, T(0), nullptr, nullptr);
    dot_kernel<T><<<nb, 256, 0, st>>>(ndof, P.r, P.r, partials, nullptr); count_launch();
    finalize_kernel<<<1, 256, 0, st>>>(partials, nb, state, kFinRRInit, 0.0); count_launch();
    T* z = vcycle<T>(0, P.r, &state->done, &rc);
    dot_kernel<T><<<nb, 256, 0, st>>>(ndof, P.r, z, partials, &state->done); count_launch();
    finalize_kernel<<<1, 256, 0, st>>>(partials, nb, state, kFinRZInit, 0.0); count_launch();
    cg_p_kernel<T><<<nb, 256, 0, st>>>(ndof, z, P.p, state, 1); count_launch();
    TP3D_CHECK_LAUNCH();
    if (rc) return rc;
    // replay iterations; poll the flag with a two-deep pipeline
    const int chunk = 4;
    int launched = 0;
    cudaEvent_t ev[2];
    cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
    int which = 0;
    bool pending = false;
    int status = TP3D_OK;
    while (true) {
      for (int k = 0; k < chunk; ++k) {
        if (cudaGraphLaunch(P.graph, st) != cudaSuccess) {
          status = TP3D_ERR_CUDA;
          break;
        }
        add_launches(P.graph_kernels);
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
      if (launched > max_iters + 2 * chunk) {
        cudaEventSynchronize(ev[1 - which]);
        break;
      }
      if (status) break;
    }
    cudaMemcpyAsync(state_host, state, sizeof(PcgState), cudaMemcpyDeviceToHost, st);
    TP3D_CHECK(cudaStreamSynchronize(st));
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    if (status) return status;
    const PcgState s = state_host[0];
    if (iters_out) *iters_out = s.iters;
    if (relres_out) *relres_out = s.bb > 0 ? std::sqrt(std::max(s.rr, 0.0) / s.bb) : 0.0;
    if (s.done == 1) return TP3D_OK;
    if (s.done == 2) return TP3D_NOT_CONVERGED;
    if (s.done == 3 || s.done == 4) {
      tp3d_set_last_error(s.done == 3 ? "PCG breakdown (p'Ap <= 0)" : "non-finite residual in PCG");
      return TP3D_ERR_NONFINITE;
    }
    return TP3D_NOT_CONVERGED;
  }
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

extern "C" void tp3d_solver_default_opts(tp3d_solver_opts* o) {
  if (!o) return;
  o->precision = TP3D_PRECISION_FP64;
  o->max_iterations = 2000;
  o->rtol = 1e-10;
  o->pre_sweeps = 2;
  o->post_sweeps = 2;
  o->omega = 0.6;
  o->coarsest_max_dofs = 500;
  o->max_levels = 12;
  o->inner_rtol = 1e-4;
  o->max_refinements = 30;
}

extern "C" int tp3d_solver_create(int nelx, int nely, int nelz, const double* KE_host, const uint8_t* fixed_dofs,
                                  const tp3d_solver_opts* opts, void* stream, tp3d_solver** out) {
  if (!out || !KE_host || !fixed_dofs || nelx < 1 || nely < 1 || nelz < 1) return TP3D_ERR_ARG;
  *out = nullptr;
  tp3d_solver* s = new tp3d_solver();
  if (opts) s->o = *opts;
  else tp3d_solver_default_opts(&s->o);
  if (s->o.pre_sweeps < 1) s->o.pre_sweeps = 1;
  if (s->o.post_sweeps < 0) s->o.post_sweeps = 0;
  if (s->o.omega <= 0.0) s->o.omega = 0.6;
  s->g = Grid{nelx, nely, nelz};
  s->user = (cudaStream_t)stream;
  if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_in, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_out, cudaEventDisableTiming) != cudaSuccess) {
    tp3d_set_last_error("stream creation failed");
    delete s;
    return TP3D_ERR_CUDA;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, dev);
  for (int i = 0; i < 576; ++i) {
    s->ke64.k[i] = KE_host[i];
    s->ke32.k[i] = (float)KE_host[i];
  }
  s->tile = choose_tile(s->g, s->nsm);
  auto fail = [&](int rc, const char* msg) {
    tp3d_set_last_error(msg);
    delete s;
    return rc;
  };
  // levels
  s->grids.push_back(s->g);
  while ((int)s->grids.size() < std::max(1, s->o.max_levels)) {
    const Grid& f = s->grids.back();
    if (3 * f.nnode() <= s->o.coarsest_max_dofs) break;
    const Grid c = coarse_grid(f);
    if (c.nx == f.nx && c.ny == f.ny && c.nz == f.nz) break;
    s->grids.push_back(c);
  }
  // if the coarsest is still too big for the dense solve, drop MG (Jacobi-PCG)
  if (3 * s->grids.back().nnode() > 3000) s->grids.resize(1);
  s->nlev = (int)s->grids.size();
  const bool mixed = s->o.precision == TP3D_PRECISION_MIXED;

  s->partials = s->alloc<double>(kMaxPartials);
  s->state = s->alloc<PcgState>(1);
  unsigned int* cnt = s->alloc<unsigned int>(4);
  if (!s->partials || !s->state || !cnt) return fail(TP3D_ERR_CUDA, "allocation failed");
  if (cudaMallocHost(&s->state_host, 2 * sizeof(PcgState)) != cudaSuccess) return fail(TP3D_ERR_CUDA, "pinned alloc");
  for (int L = 0; L < s->nlev; ++L) {
    const Grid& gl = s->grids[L];
    uint8_t* f = s->alloc<uint8_t>(gl.nnode());
    if (!f) return fail(TP3D_ERR_CUDA, "allocation failed");
    s->fix.push_back(f);
  }
  if (s->enter()) return fail(TP3D_ERR_CUDA, "stream ordering failed");
  cudaMemsetAsync(cnt, 0, 4 * sizeof(unsigned int), s->st);
  pack_mask_kernel<<<s->grid_blocks(s->g.nnode()), 256, 0, s->st>>>(s->g.nnode(), fixed_dofs, s->fix[0], cnt); count_launch();
  for (int L = 1; L < s->nlev; ++L) {
    unsigned int h[2] = {0, 0};
    cudaMemsetAsync(cnt + 1, 0, sizeof(unsigned int), s->st);
    coarse_mask_kernel<<<s->grid_blocks(s->grids[L].nnode()), 256, 0, s->st>>>(s->grids[L - 1], s->grids[L],
                                                                                s->fix[L - 1], s->fix[L], 0, cnt + 1); count_launch();
    cudaMemcpyAsync(h, cnt, 2 * sizeof(unsigned int), cudaMemcpyDeviceToHost, s->st);
    cudaStreamSynchronize(s->st);
    if (h[1] == 0 && h[0] > 0) {
      cudaMemsetAsync(cnt + 1, 0, sizeof(unsigned int), s->st);
      coarse_mask_kernel<<<s->grid_blocks(s->grids[L].nnode()), 256, 0, s->st>>>(
          s->grids[L - 1], s->grids[L], s->fix[L - 1], s->fix[L], 1, cnt + 1); count_launch();
    }
  }
  if (cudaStreamSynchronize(s->st) != cudaSuccess) return fail(TP3D_ERR_CUDA, "mask setup failed");

  const long long nele = s->g.nele();
  s->E64 = s->alloc<double>(nele);
  if (mixed) s->rho16 = s->alloc<__nv_bfloat16>(nele);
  double ke1[8 * 576];
  coarse_subelement_tables(KE_host, ke1);
  s->KE1 = s->alloc<double>(8 * 576);
  cudaMemcpy(s->KE1, ke1, sizeof(ke1), cudaMemcpyHostToDevice);
  s->A64.assign(s->nlev, nullptr);
  s->L64.resize(s->nlev);
  if (mixed) s->L32.resize(s->nlev);
  for (int L = 0; L < s->nlev; ++L) {
    const long long nn = s->grids[L].nnode(), ndof = 3 * nn;
    if (L > 0) s->A64[L] = s->alloc<double>(243 * nn);
    auto& a = s->L64[L];
    if (!mixed) {
      a.x[0] = s->alloc<double>(ndof); a.x[1] = s->alloc<double>(ndof);
      a.b = s->alloc<double>(ndof); a.r = s->alloc<double>(ndof); a.dinv = s->alloc<double>(ndof);
      a.A = s->A64[L];
    } else {
      auto& b = s->L32[L];
      b.x[0] = s->alloc<float>(ndof); b.x[1] = s->alloc<float>(ndof);
      b.b = s->alloc<float>(ndof); b.r = s->alloc<float>(ndof); b.dinv = s->alloc<float>(ndof);
      if (L > 0) b.A = s->alloc<float>(243 * nn);
    }
  }
  s->cn = (int)(3 * s->grids.back().nnode());
  if (s->nlev > 1) {
    s->cdense = s->alloc<double>((size_t)s->cn * s->cn);
    s->cwork = s->alloc<double>((size_t)s->cn * s->cn);
    s->cinv64 = s->alloc<double>((size_t)s->cn * s->cn);
    if (mixed) s->cinv32 = s->alloc<float>((size_t)s->cn * s->cn);
    s->cstatus = s->alloc<int>(1);
  }
  const long long ndof = 3 * s->g.nnode();
  if (!mixed) {
    s->P64.u = s->alloc<double>(ndof); s->P64.r = s->alloc<double>(ndof);
    s->P64.p = s->alloc<double>(ndof); s->P64.q = s->alloc<double>(ndof);
  } else {
    s->P64.u = s->alloc<double>(ndof);
    s->res64 = s->alloc<double>(ndof);
    s->P32.u = s->alloc<float>(ndof); s->P32.r = s->alloc<float>(ndof);
    s->P32.p = s->alloc<float>(ndof); s->P32.q = s->alloc<float>(ndof);
    s->L64[0].dinv = nullptr;
  }
  for (void* p : s->allocs)
    if (!p) return fail(TP3D_ERR_CUDA, "allocation failed");
  if (s->tile.tiles_y * s->tile.tiles_x * s->tile.zchunks > kMaxPartials)
    return fail(TP3D_ERR_ARG, "grid too large for the partial-sum buffer");
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

extern "C" int tp3d_solver_set_density(tp3d_solver* s, const double* rho, double penal) {
  if (!s || !rho || !(penal > 0.0)) return TP3D_ERR_ARG;
  s->penal = penal;
  const bool mixed = s->o.precision == TP3D_PRECISION_MIXED;
  const long long nele = s->g.nele();
  cudaStream_t st = s->st;
  if (int rc = s->enter()) return rc;
  moduli_kernel<<<s->grid_blocks(nele), 256, 0, st>>>(nele, rho, penal, s->E64, s->rho16); count_launch();
  const long long nn0 = s->g.nnode();
  if (!mixed) {
    fine_diag_inv_kernel<double, EFromF64><<<s->grid_blocks(nn0), 256, 0, st>>>(s->g, s->ke64, EFromF64{s->E64},
                                                                                 s->fix[0], s->L64[0].dinv); count_launch();
  } else {
    fine_diag_inv_kernel<float, EFromBF16><<<s->grid_blocks(nn0), 256, 0, st>>>(
        s->g, s->ke64, EFromBF16{s->rho16, (float)penal}, s->fix[0], s->L32[0].dinv); count_launch();
  }
  TP3D_CHECK_LAUNCH();
  for (int L = 1; L < s->nlev; ++L) {
    const Grid& gf = s->grids[L - 1];
    const Grid& gc = s->grids[L];
    const unsigned nb = (unsigned)((gc.nnode() + 31) / 32);
    if (L == 1) {
      build_level1_kernel<<<nb, kBuildThreads, 0, st>>>(gf, gc, s->E64, s->KE1, s->A64[1]); count_launch();
    } else {
      rap_kernel<<<nb, kBuildThreads, 0, st>>>(gf, gc, s->A64[L - 1], s->A64[L]); count_launch();
    }
    TP3D_CHECK_LAUNCH();
    const long long nn = gc.nnode();
    if (!mixed) {
      stencil_diag_inv_kernel<double><<<s->grid_blocks(nn), 256, 0, st>>>(gc, s->A64[L], s->fix[L], s->L64[L].dinv); count_launch();
    } else {
      stencil_diag_inv_kernel<float><<<s->grid_blocks(nn), 256, 0, st>>>(gc, s->A64[L], s->fix[L], s->L32[L].dinv); count_launch();
      convert_kernel<double, float><<<s->grid_blocks(243 * nn), 256, 0, st>>>(243 * nn, s->A64[L], s->L32[L].A); count_launch();
    }
    TP3D_CHECK_LAUNCH();
  }
  if (s->nlev > 1) {
    const int L = s->nlev - 1;
    const int n = s->cn;
    double shift = 0.0;
    for (int attempt = 0; attempt < 4; ++attempt) {
      TP3D_CHECK(cudaMemsetAsync(s->cdense, 0, (size_t)n * n * sizeof(double), st));
      dense_from_stencil_kernel<<<s->grid_blocks(s->grids[L].nnode()), 256, 0, st>>>(s->grids[L], s->A64[L],
                                                                                      s->fix[L], s->cdense); count_launch();
      if (shift > 0.0) {
        dense_shift_kernel<<<s->grid_blocks(n), 256, 0, st>>>(n, s->cdense, shift); count_launch();
      }
      dense_inverse_kernel<<<1, 1024, 0, st>>>(n, s->cdense, s->cwork, s->cinv64, s->cstatus); count_launch();
      TP3D_CHECK_LAUNCH();
      int status = 0;
      TP3D_CHECK(cudaMemcpyAsync(&status, s->cstatus, sizeof(int), cudaMemcpyDeviceToHost, st));
      TP3D_CHECK(cudaStreamSynchronize(st));
      if (status == 0) break;
      // not positive definite (e.g. a floating coarse problem): shift relative to the mean diagonal
      std::vector<double> diag(1);
      shift = (shift == 0.0) ? 1e-10 : shift * 1e3;
      double dsum = 0.0;
      {
        // estimate mean diagonal from the stencil's centre entries
        std::vector<double> h(243 * s->grids[L].nnode());
        cudaMemcpy(h.data(), s->A64[L], h.size() * sizeof(double), cudaMemcpyDeviceToHost);
        const long long nnL = s->grids[L].nnode();
        for (long long i = 0; i < nnL; ++i)
          for (int c = 0; c < 3; ++c) dsum += h[(size_t)stencil_k(13, c, c) * nnL + i];
        dsum /= (double)n;
      }
      shift *= std::max(dsum, 1e-30);
    }
    if (mixed)
      convert_kernel<double, float><<<s->grid_blocks((long long)n * n), 256, 0, st>>>((long long)n * n, s->cinv64,
                                                                                      s->cinv32); count_launch();
  }
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
  const int nb = s->grid_blocks(ndof);
  int rc = TP3D_OK;
  if (int e = s->enter()) return e;
  TP3D_CHECK(cudaMemcpyAsync(s->P64.u, U, ndof * sizeof(double), cudaMemcpyDeviceToDevice, st));
  zero_fixed_kernel<<<s->grid_blocks(nn), 256, 0, st>>>(nn, s->P64.u, s->fix[0]); count_launch();
  s->last_refinements = 0;
  s->last_inner_total = 0;
  if (s->o.precision == TP3D_PRECISION_FP64) {
    int it = 0;
    double rr = 0;
    rc = s->pcg<double>(s->P64, F, s->o.rtol, s->o.max_iterations, &it, &rr);
    s->last_iters = it;
    s->last_relres = rr;
  } else {
    // FP64 iterative refinement around an FP32 multigrid PCG
    double bb = 0.0;
    masked_norm_kernel<<<s->grid_blocks(nn), 256, 0, st>>>(nn, F, s->fix[0], s->partials); count_launch();
    finalize_kernel<<<1, 256, 0, st>>>(s->partials, s->grid_blocks(nn), s->state, kFinBB, 0.0); count_launch();
    TP3D_CHECK(cudaMemcpyAsync(s->state_host, s->state, sizeof(PcgState), cudaMemcpyDeviceToHost, st));
    TP3D_CHECK(cudaStreamSynchronize(st));
    bb = s->state_host->bb;
    double relres_v = 0.0;
    rc = TP3D_NOT_CONVERGED;
    if (bb == 0.0) {
      TP3D_CHECK(cudaMemsetAsync(s->P64.u, 0, ndof * sizeof(double), st));
      rc = TP3D_OK;
    } else {
      for (int k = 0; k <= s->o.max_refinements; ++k) {
        rc |= s->fine<double, kModeResid>(s->P64.u, s->res64, F, nullptr, 0.0, nullptr, nullptr);
        dot_kernel<double><<<nb, 256, 0, st>>>(ndof, s->res64, s->res64, s->partials, nullptr); count_launch();
        finalize_kernel<<<1, 256, 0, st>>>(s->partials, nb, s->state, kFinBB, 0.0); count_launch();
        TP3D_CHECK(cudaMemcpyAsync(s->state_host, s->state, sizeof(PcgState), cudaMemcpyDeviceToHost, st));
        TP3D_CHECK(cudaStreamSynchronize(st));
        const double rr = s->state_host->bb;
        relres_v = std::sqrt(rr / bb);
        if (!std::isfinite(relres_v)) {
          rc = TP3D_ERR_NONFINITE;
          tp3d_set_last_error("non-finite residual in refinement");
          break;
        }
        if (relres_v <= s->o.rtol) {
          rc = TP3D_OK;
          break;
        }
        if (k == s->o.max_refinements) {
          rc = TP3D_NOT_CONVERGED;
          break;
        }
        const double sc = 1.0 / std::sqrt(rr);
        scale_down_kernel<<<nb, 256, 0, st>>>(ndof, s->res64, sc, s->L32[0].b); count_launch();
        TP3D_CHECK(cudaMemsetAsync(s->P32.u, 0, ndof * sizeof(float), st));
        int it = 0;
        double inner_rel = 0;
        const int irc = s->pcg<float>(s->P32, s->L32[0].b, s->o.inner_rtol, s->o.max_iterations, &it, &inner_rel);
        if (irc < 0) {
          rc = irc;
          break;
        }
        s->last_inner_total += it;
        s->last_refinements = k + 1;
        axpy_up_kernel<<<nb, 256, 0, st>>>(ndof, s->P32.u, 1.0 / sc, s->P64.u); count_launch();
      }
    }
    s->last_iters = s->last_inner_total;
    s->last_relres = relres_v;
  }
  TP3D_CHECK(cudaMemcpyAsync(U, s->P64.u, ndof * sizeof(double), cudaMemcpyDeviceToDevice, st));
  TP3D_CHECK(cudaStreamSynchronize(st));
  if (int e = s->leave()) return e;
  if (iterations) *iterations = s->last_iters;
  if (relres) *relres = s->last_relres;
  return rc;
}

extern "C" int tp3d_solver_apply_f64(tp3d_solver* s, const double* u, double* y) {
  if (!s || !u || !y || !s->have_density) return TP3D_ERR_ARG;
  if (int rc = s->enter()) return rc;
  if (int rc = s->fine<double, kModeApply>(u, y, nullptr, nullptr, 0.0, nullptr, nullptr)) return rc;
  return s->leave();
}

extern "C" int tp3d_solver_apply_f32(tp3d_solver* s, const float* u, float* y) {
  if (!s || !u || !y || !s->have_density || !s->rho16) return TP3D_ERR_ARG;
  if (int rc = s->enter()) return rc;
  if (int rc = s->fine<float, kModeApply>(u, y, nullptr, nullptr, 0.0f, nullptr, nullptr)) return rc;
  return s->leave();
}

extern "C" int tp3d_solver_time_apply(tp3d_solver* s, int fp32, int launches, double* ms_per_launch) {
  if (!s || !ms_per_launch || launches < 1 || !s->have_density) return TP3D_ERR_ARG;
  if (fp32 && !s->rho16) return TP3D_ERR_ARG;
  if (int rc = s->enter()) return rc;
  cudaEvent_t a, b;
  TP3D_CHECK(cudaEventCreate(&a));
  TP3D_CHECK(cudaEventCreate(&b));
  int rc = TP3D_OK;
  // inputs: the current PCG vectors (any finite data times the same work)
  auto run = [&]() {
    for (int i = 0; i < launches && rc == TP3D_OK; ++i) {
      if (fp32) rc = s->fine<float, kModeApply>(s->P32.p, s->P32.q, nullptr, nullptr, 0.0f, nullptr, nullptr);
      else rc = s->fine<double, kModeApply>(s->P64.u, s->L64.empty() || !s->P64.q ? s->res64 : s->P64.q,
                                            nullptr, nullptr, 0.0, nullptr, nullptr);
    }
  };
  run();  // warm-up
  TP3D_CHECK(cudaEventRecord(a, s->st));
  run();
  TP3D_CHECK(cudaEventRecord(b, s->st));
  TP3D_CHECK(cudaEventSynchronize(b));
  float ms = 0.f;
  TP3D_CHECK(cudaEventElapsedTime(&ms, a, b));
  *ms_per_launch = ms / launches;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc) return rc;
  return s->leave();
}

extern "C" int tp3d_solver_stats(tp3d_solver* s, double* out, int n) {
  if (!s || !out) return TP3D_ERR_ARG;
  const double v[] = {(double)s->nlev, (double)s->last_iters, (double)s->last_refinements, s->last_relres,
                      (double)s->last_inner_total, (double)s->cn, (double)s->tile.TY, (double)s->tile.TX,
                      (double)s->tile.ZC};
  const int m = std::min<int>(n, (int)(sizeof(v) / sizeof(v[0])));
  for (int i = 0; i < m; ++i) out[i] = v[i];
  return m;
}
