// Vector kernels of the Krylov solvers: reductions, CG updates, Chebyshev
// coefficients, reliable-update bookkeeping.  Every scalar (alpha, beta,
// stop flags) lives in device memory so that one solver iteration can be
// captured into a CUDA graph and replayed without host round trips.
#pragma once

#include "tp3d_cgstate.cuh"
#include "tp3d_mg.cuh"

namespace tp3d {

__global__ void finalize_kernel(const double* __restrict__ partials, int n, PcgState* st, int op, double rtol2,
                                double* out) {
  pdl_entry();
  __shared__ double red[32];
  if (finalize_skipped(st, op)) return;
  const double s = sum_partials(partials, n, red);
  if (threadIdx.x != 0) return;
  finalize_apply(s, st, op, rtol2, out);
}

__global__ void clear_update_kernel(PcgState* st) {
  pdl_entry();
  st->update = 0;
}

// Linear extrapolation of successive solutions as the next initial guess:
// U <- 2 U - U_prev and U_prev <- U (old), or only U_prev <- U when there is no
// history yet.
__global__ void warm_start_kernel(long long n, double* U, double* U_prev, int have_prev) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double u = U[i];
    if (have_prev) U[i] = 2.0 * u - U_prev[i];
    U_prev[i] = u;
  }
}

// Conditions of the device-side CG loop (CUDA graph conditional nodes).
// Reliable-update branch: a pending update on a running solve.
__global__ void set_update_cond_kernel(cudaGraphConditionalHandle h, const PcgState* st) {
  const bool go = *(volatile const int*)&st->done == 0 && *(volatile const int*)&st->update != 0;
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

// Iteration loop: continue while the solve runs.  The loop also counts its
// own passes and stops after `limit` of them, so it ends even if no kernel of
// the body ever updated the state.
__global__ void set_loop_cond_kernel(cudaGraphConditionalHandle h, const PcgState* st, unsigned int* passes,
                                     unsigned int limit) {
  const unsigned int n = *passes + 1u;
  *passes = n;
  const bool go = *(volatile const int*)&st->done == 0 && n < limit;
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

// a . b into per-block partials; with fin_count, the last block applies op to st.
template <typename T>
__global__ void dot_kernel(long long n, const T* __restrict__ a, const T* __restrict__ b, double* partials,
                           const int* done, const int* gate, PcgState* st = nullptr, int op = 0,
                           unsigned int* fin_count = nullptr) {
  pdl_entry();
  if ((done && *(volatile const int*)done) || (gate && *(volatile const int*)gate == 0)) return;
  __shared__ double red[32];
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s += (double)a[i] * (double)b[i];
  s = block_sum(s, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
  if (fin_count) last_block_finalize(partials, gridDim.x, fin_count, st, op, red);
}

// ||b||^2 over free DOFs
__global__ void masked_norm_kernel(long long nn, const double* __restrict__ b, const uint8_t* __restrict__ fix,
                                   double* partials) {
  pdl_entry();
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

// u += alpha p; r -= alpha q; partials of ||r||^2 (with fin_count, the last
// block applies op to st)
// With fs.x0 set, also the V-cycle's first smoothing step from the new
// residual (pointwise: x0 = w dinv r, d = x0), as smooth_zero_kernel computes it.
template <typename T>
__global__ void cg_update_kernel(long long n, T* u, const T* __restrict__ p, T* r, const T* __restrict__ q,
                                 PcgState* st, double* partials, int op = 0, unsigned int* fin_count = nullptr,
                                 CoarseFirstStep<T> fs = CoarseFirstStep<T>{}) {
  pdl_entry();
  if (*(volatile const int*)&st->done) return;
  __shared__ double red[32];
  const T a = (T)st->alpha;
  const T w = fs.x0 ? (fs.coef ? (T)fs.coef[0] : fs.omega) : T(0);
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    u[i] += a * p[i];
    const T ri = r[i] - a * q[i];
    r[i] = ri;
    s += (double)ri * (double)ri;
    if (fs.x0) {
      const T v = w * fs.dinv[i] * ri;
      fs.x0[i] = v;
      if (fs.d) fs.d[i] = v;
    }
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
  if (fin_count) last_block_finalize(partials, gridDim.x, fin_count, st, op, red);
}

// p = z + beta p (or p = z)
template <typename T>
__global__ void cg_p_kernel(long long n, const T* __restrict__ z, T* p, const PcgState* st, int init) {
  pdl_entry();
  if (!init && *(volatile const int*)&st->done) return;
  const T b = init ? T(0) : (T)st->beta;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = init ? z[i] : z[i] + b * p[i];
}

// Reliable update: u64 += x32, x32 = 0 (only when st->update, or always with force).
__global__ void flush_kernel(long long n, double* u, float* x, const PcgState* st, int force) {
  pdl_entry();
  if (!force && (*(volatile const int*)&st->done || *(volatile const int*)&st->update == 0)) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    u[i] += (double)x[i];
    x[i] = 0.0f;
  }
}

// r32 = float(r64), gated like the reliable update
__global__ void demote_kernel(long long n, const double* __restrict__ r, float* out, const PcgState* st, int force) {
  pdl_entry();
  if (!force && (*(volatile const int*)&st->done || *(volatile const int*)&st->update == 0)) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (float)r[i];
}

__global__ void zero_fixed_kernel(long long nn, double* u, const uint8_t* __restrict__ fix) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn; n += (long long)gridDim.x * blockDim.x) {
    const int f = fix[n];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      if ((f >> c) & 1) u[3 * n + c] = 0.0;
  }
}

// E = Emin + (1 - Emin) rho^p (optimizer.py:584-586); optional FP32 / BF16 copies.
__global__ void moduli_kernel(long long n, const double* __restrict__ rho, double penal, double* E, float* E32,
                              __nv_bfloat16* rho16) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const double r = rho[e];
    const double rp = (penal == 2.0) ? r * r : pow(r, penal);
    const double Ev = kEmin + (kE0 - kEmin) * rp;
    E[e] = Ev;
    if (E32) E32[e] = (float)Ev;
    if (rho16) rho16[e] = __double2bfloat16(r);
  }
}

template <typename Tsrc, typename Tdst>
__global__ void convert_kernel(long long n, const Tsrc* __restrict__ a, Tdst* b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = (Tdst)a[i];
}

// Deterministic pseudo-random start vector on free DOFs (power iteration).
template <typename T>
__global__ void random_vector_kernel(long long nn, const uint8_t* __restrict__ fix, T* v) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn; n += (long long)gridDim.x * blockDim.x) {
    const int f = fix[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      unsigned long long h = (unsigned long long)(3 * n + c) * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
      h ^= h >> 29;
      h *= 0xBF58476D1CE4E5B9ull;
      h ^= h >> 32;
      const double r = 2.0 * (double)(h >> 11) * (1.0 / 9007199254740992.0) - 1.0;  // [-1, 1)
      v[3 * n + c] = ((f >> c) & 1) ? T(0) : (T)r;
    }
  }
}

constexpr int kMaxCheb = 8;
constexpr int kCoefLen = 2 * kMaxCheb + 2;

// Chebyshev coefficients from a power-iteration estimate of lambda_max(Dinv A):
// lam = ||v_N|| / ||v_{N-1}||.  Target interval [hi / ratio, hi], hi = safety * lam.
// coef = [1/theta, lam_est, c1_1, c2_1, ...] with
//   rho_0 = delta/theta, rho_k = 1/(2 theta/delta - rho_{k-1}),
//   c1_k = rho_k rho_{k-1}, c2_k = 2 rho_k / delta.
__global__ void cheb_setup_kernel(const double* __restrict__ pa, int na, const double* __restrict__ pb, int nb,
                                  double ratio, double safety, double* coef) {
  __shared__ double red[32];
  const double a = sum_partials(pa, na, red);
  const double b = sum_partials(pb, nb, red);
  if (threadIdx.x != 0) return;
  double lam = (b > 0.0) ? sqrt(a / b) : 2.0;
  if (!isfinite(lam) || lam <= 0.0) lam = 2.0;
  coef[kCoefLen - 1] = (a > 0.0 && isfinite(a)) ? 1.0 / sqrt(a) : 0.0;  // normaliser of the last iterate
  const double hi = safety * lam, lo = hi / ratio;
  const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo);
  coef[0] = 1.0 / theta;
  coef[1] = lam;
  double rho = delta / theta;
  for (int k = 1; k < kMaxCheb; ++k) {
    const double rn = 1.0 / (2.0 * theta / delta - rho);
    coef[2 * k] = rn * rho;
    coef[2 * k + 1] = 2.0 * rn / delta;
    rho = rn;
  }
}

// dst = src * (*scale)
template <typename T>
__global__ void scale_copy_kernel(long long n, const T* __restrict__ src, const double* __restrict__ scale,
                                  double* dst) {
  const double s = *scale;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = (double)src[i] * s;
}

}  // namespace tp3d

namespace tp3d {

// ---------------------------------------------------------------------------
// Kernels of the captured SIMP stage (one CUDA graph per projection stage):
// every host decision of the loop body becomes a device value.
// ---------------------------------------------------------------------------

// Stage counters (device ints): iteration of the launch, abort flag, CG
// iterations of the running iteration, iteration limit of the launch, solves
// done before the launch.
enum StageCounter : int { kStIter = 0, kStAbort, kStCg, kStLimit, kStBase, kStCount };
constexpr int kStageRecord = 8;  // doubles per recorded iteration

// A conditional node's value is assigned its default only when the graph is
// launched: a WHILE node nested in another loop's body is re-armed by this
// kernel before each entry.
__global__ void arm_conditional_kernel(cudaGraphConditionalHandle h) { cudaGraphSetConditional(h, 1u); }

// The solver state of a new solve, as the host path writes it before a solve.
__global__ void init_state_kernel(PcgState* st, int max_iters, double delta2) {
  PcgState z{};
  z.max_iters = max_iters;
  z.delta2 = delta2;
  *st = z;
}

// Extrapolated initial guess (warm_start_kernel) with the history test on the
// device: the last two solutions exist once base + iteration >= 2 solves were done.
__global__ void warm_start_dev_kernel(long long n, double* U, double* U_prev, const int* ctr) {
  const int have_prev = ctr[kStBase] + ctr[kStIter] >= 2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double u = U[i];
    if (have_prev) U[i] = 2.0 * u - U_prev[i];
    U_prev[i] = u;
  }
}

// Rayleigh-Ritz initial guess from the last two solutions U1 = U and
// U2 = U_prev under the current operator K: the x = a U1 + b U2 that minimises
// the energy x'Kx / 2 - F'x over span{U1, U2}, which contains the linear
// extrapolation 2 U1 - U2 of warm_start_kernel, so it starts CG at least as
// close in the energy norm.  Gate: whether both solutions exist (the host's
// flag, or the stage counters' history test when ctr is given).
__global__ void ritz_gate_kernel(int* gate, int have_prev, const int* ctr) {
  *gate = ctr ? (ctr[kStBase] + ctr[kStIter] >= 2) : (have_prev != 0);
}

// Per-block sums of U1.KU1, U1.KU2, U2.KU2, F.U1, F.U2 (q1 = K U1, q2 = K U2;
// fixed DOFs of U are zero, so they add nothing); the last block adds the
// partials in a fixed order and solves the 2x2 Galerkin system for (a, b).  A
// nearly dependent pair (det <= 1e-10 G11 G22) falls back to the best multiple
// of U1, anything non-finite to U1 itself.
__global__ void ritz_dot_kernel(long long n, const double* __restrict__ F, const double* __restrict__ U1,
                                const double* __restrict__ U2, const double* __restrict__ q1,
                                const double* __restrict__ q2, const int* gate, double* partials,
                                unsigned int* count, double* coef) {
  if (*(volatile const int*)gate == 0) return;
  __shared__ double red[32];
  __shared__ int s_last;
  double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double a = U1[i], b = U2[i], f = F[i], x = q1[i], y = q2[i];
    v[0] = fma(a, x, v[0]);
    v[1] = fma(a, y, v[1]);
    v[2] = fma(b, y, v[2]);
    v[3] = fma(f, a, v[3]);
    v[4] = fma(f, b, v[4]);
  }
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const double t = block_sum(v[k], red);
    if (threadIdx.x == 0) partials[k * gridDim.x + blockIdx.x] = t;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(count, 1u) == gridDim.x - 1u;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double tot[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    double t = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) t += __ldcg(&partials[k * gridDim.x + i]);
    tot[k] = block_sum(t, red);
  }
  if (threadIdx.x == 0) {
    const double g11 = tot[0], g12 = tot[1], g22 = tot[2], r1 = tot[3], r2 = tot[4];
    double a = 1.0, b = 0.0;
    const double det = g11 * g22 - g12 * g12;
    if (g11 > 0.0 && g22 > 0.0 && det > 1e-10 * g11 * g22) {
      a = (r1 * g22 - r2 * g12) / det;
      b = (g11 * r2 - g12 * r1) / det;
    } else if (g11 > 0.0) {
      a = r1 / g11;
    }
    if (!isfinite(a) || !isfinite(b)) {
      a = 1.0;
      b = 0.0;
    }
    coef[0] = a;
    coef[1] = b;
    *count = 0u;
  }
}

// U <- a U1 + b U2 where the gate is open (else U stays U1), U_prev <- U1.
__global__ void ritz_combine_kernel(long long n, double* U, double* U_prev, const double* coef, const int* gate) {
  const bool on = *(volatile const int*)gate != 0;
  const double a = on ? coef[0] : 1.0, b = on ? coef[1] : 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double u1 = U[i], u2 = U_prev[i];
    if (on) U[i] = a * u1 + b * u2;
    U_prev[i] = u1;
  }
}

// After a queued mixed solve: whether the host path would have accepted it
// without its FP64 fallback (converged, or at its residual floor).  Otherwise
// *abort is raised.  The solve's CG iterations are summed into *cg.
__global__ void solve_status_kernel(const PcgState* st, int* abort, int* cg) {
  const PcgState s = *st;
  if (!(s.done == 1 || s.done == 5)) *abort = 1;
  *cg += s.iters;
}

// Restart state of an FP64 solve queued in a stage graph (the host path's
// solve64 loop): [0] residual of the previous run, [1] CG iterations so far,
// [2] restarts so far.
__global__ void restart_init_kernel(double* rs) {
  rs[0] = INFINITY;
  rs[1] = 0.0;
  rs[2] = 0.0;
}

// The solver state of the next run of that loop: the iteration budget left.
__global__ void init_state_budget_kernel(PcgState* st, const double* rs, int max_iters) {
  PcgState z{};
  z.max_iters = max(1, max_iters - (int)rs[1]);
  *st = z;
}

// After a run and its true residual (st->rr = ||f - K u||^2): the decisions of
// the host path's solve64, taken on the device.  Accept (relative residual
// within 2 rtol, or the residual floor: a converged run whose restart no
// longer halved it), restart (set the loop condition), or hand the solve back
// to the host (breakdown, non-finite, not converged within the budget).
__global__ void restart_decide_kernel(cudaGraphConditionalHandle h, const PcgState* st, double* rs, double rtol,
                                      int max_restarts, int max_iters, int* abort, int* cg) {
  const PcgState s = *st;
  const double total = rs[1] + s.iters;
  rs[1] = total;
  *cg += s.iters;
  bool again = false;
  if (s.done == 3 || s.done == 4 || s.done == 7) {
    *abort = 1;
  } else if (s.bb != 0.0) {
    const bool run_ok = s.done == 1 || s.done == 5;
    const double relres = sqrt(fmax(s.rr, 0.0) / s.bb);
    if (!isfinite(relres)) {
      *abort = 1;
    } else if (relres <= 2.0 * rtol) {
      // accepted
    } else if (run_ok && relres > 0.5 * rs[0]) {
      // residual floor: accepted
    } else if (!run_ok || rs[2] >= max_restarts || total >= max_iters) {
      *abort = 1;
    } else {
      rs[0] = relres;
      rs[2] += 1.0;
      again = true;
    }
  }
  cudaGraphSetConditional(h, again ? 1u : 0u);
}

// Several load cases: dc += dc_case, c[0] += c[1] (the host path's sums).
__global__ void accumulate_case_kernel(long long n, double* dc, const double* __restrict__ dc_case, double* c) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dc[i] += dc_case[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) c[0] += c[1];
}

// Gate of the iteration's second half (sensitivities, OC, projection).
__global__ void stage_gate_kernel(cudaGraphConditionalHandle h, const int* ctr) {
  cudaGraphSetConditional(h, ctr[kStAbort] == 0 ? 1u : 0u);
}

// End of an iteration: record [c, lambda, volume, steps, change, CG
// iterations, lambda bracket] at the iteration's slot, advance the counter and
// decide the stage loop (change > tolx and below the limit, no abort).
__global__ void stage_next_kernel(cudaGraphConditionalHandle h, int* ctr, const double* __restrict__ c,
                                  const double* __restrict__ oc, double* record, double tolx) {
  if (ctr[kStAbort]) {
    cudaGraphSetConditional(h, 0u);
    return;
  }
  const int it = ctr[kStIter];
  double* r = record + (size_t)it * kStageRecord;
  r[0] = c[0];
  r[1] = oc[0];
  r[2] = oc[1];
  r[3] = oc[2];
  r[4] = oc[3];
  r[5] = (double)ctr[kStCg];
  r[6] = oc[5];
  r[7] = oc[6];
  ctr[kStIter] = it + 1;
  ctr[kStCg] = 0;
  const bool go = oc[3] > tolx && it + 1 < ctr[kStLimit];
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

}  // namespace tp3d
