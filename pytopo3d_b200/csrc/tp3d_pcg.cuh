// Vector kernels of the Krylov solvers: reductions, CG updates, Chebyshev
// coefficients, reliable-update bookkeeping.  Every scalar (alpha, beta,
// stop flags) lives in device memory so that one solver iteration can be
// captured into a CUDA graph and replayed without host round trips.
#pragma once

#include "tp3d_mg.cuh"

namespace tp3d {

struct PcgState {
  double rz, pq, rr, bb, alpha, beta, tol2, rmax2;
  double delta2;   // reliable-update threshold (squared)
  double rr_hi;    // last FP64 residual norm^2
  double rr_best;  // smallest FP64 residual norm^2 so far
  // done: 0 running, 1 converged, 2 iteration cap, 3 breakdown, 4 non-finite,
  //       5 FP64 residual stalled at its attainable floor (accepted),
  //       6 FP64 residual stalled far above the target (mixed: fall back to FP64)
  int done;
  int iters, max_iters;
  int update;   // mixed precision: replace the residual this iteration
  int updates;  // count of reliable updates
  int stall;    // consecutive reliable updates that did not halve the FP64 residual
  int restart;  // mixed precision: FP32 p'Ap <= 0, restart the direction from z
  int nbreak;   // consecutive restarts
};

enum FinalizeOp : int {
  kFinBB = 0,    // bb = ||b||^2, tol2 = rtol^2 bb
  kFinRRInit,    // rr = ||r0||^2 (stop if already converged)
  kFinRZInit,    // rz = r.z
  kFinPQ,        // alpha = rz / p.q
  kFinRR,        // rr = ||r||^2, iteration count, stop test
  kFinRZ,        // beta = rz_new / rz
  kFinRRMixed,   // FP32 recursive residual: decide on a reliable update
  kFinRRHi,      // FP64 true residual after a reliable update: stop test
  kFinValue,     // plain sum into *out (no state change)
  kFinPQMixed,   // as kFinPQ, but a non-positive FP32 p'Ap restarts the direction
  kFinRZMixed,   // as kFinRZ, honouring a pending restart (beta = 0)
};

__global__ void finalize_kernel(const double* __restrict__ partials, int n, PcgState* st, int op, double rtol2,
                                double* out) {
  __shared__ double red[32];
  if (((op >= kFinPQ && op <= kFinRRMixed) || op >= kFinPQMixed) && *(volatile int*)&st->done) return;
  if (op == kFinRRHi && (*(volatile int*)&st->done || *(volatile int*)&st->update == 0)) return;
  const double s = sum_partials(partials, n, red);
  if (threadIdx.x != 0) return;
  switch (op) {
    case kFinBB:
      st->bb = s;
      st->tol2 = rtol2 * s;
      st->iters = 0;
      st->update = 0;
      st->updates = 0;
      st->done = (s == 0.0) ? 1 : 0;
      if (!isfinite(s)) st->done = 4;
      break;
    case kFinRRInit:
      st->rr = s;
      st->rmax2 = s;
      st->rr_hi = s;
      st->rr_best = s;
      st->stall = 0;
      if (!st->done && s <= st->tol2) st->done = 1;
      if (!isfinite(s)) st->done = 4;
      break;
    case kFinRZInit:
      st->rz = s;
      break;
    case kFinPQ:
      st->pq = s;
      if (!(s > 0.0) || !isfinite(s)) st->done = 3;
      else st->alpha = st->rz / s;
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
    case kFinRRMixed:
      st->rr = s;
      st->iters += 1;
      if (!isfinite(s)) {
        st->done = 4;
      } else {
        st->update = (st->restart || s <= st->delta2 * st->rmax2 || s <= st->tol2 || st->iters >= st->max_iters)
                         ? 1
                         : 0;
      }
      break;
    case kFinRRHi:
      st->rr_hi = s;
      st->rmax2 = s;
      st->updates += 1;
      if (!isfinite(s)) {
        st->done = 4;
      } else if (s <= st->tol2) {
        st->done = 1;
      } else {
        st->stall = (s > 0.25 * st->rr_best) ? st->stall + 1 : 0;
        st->rr_best = fmin(st->rr_best, s);
        // a stall is an attainable floor only once the residual is small; a stall
        // above 1e-6 relative is a failure (the host then falls back to FP64)
        if (st->stall >= 3) st->done = (s <= 1e-12 * st->bb) ? 5 : 6;
        else if (st->iters >= st->max_iters) st->done = 2;
      }
      break;
    case kFinValue:
      *out = s;
      break;
    case kFinPQMixed:
      // FP32 rounding next to 1e-9 voids can make p'Ap non-positive although K
      // is SPD: skip the step (alpha = 0), force a reliable update and restart
      // the direction from the new preconditioned residual.
      st->pq = s;
      if (!isfinite(s)) {
        st->done = 4;
      } else if (!(s > 0.0)) {
        st->alpha = 0.0;
        st->restart = 1;
        if (++st->nbreak > 5) st->done = 3;
      } else {
        st->alpha = st->rz / s;
      }
      break;
    case kFinRZMixed:
      if (st->restart) {
        st->beta = 0.0;
        st->restart = 0;
      } else {
        st->beta = s / st->rz;
        st->nbreak = 0;
      }
      st->rz = s;
      break;
  }
}

__global__ void clear_update_kernel(PcgState* st) { st->update = 0; }

template <typename T>
__global__ void dot_kernel(long long n, const T* __restrict__ a, const T* __restrict__ b, double* partials,
                           const int* done, const int* gate) {
  if ((done && *(volatile const int*)done) || (gate && *(volatile const int*)gate == 0)) return;
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

// u += alpha p; r -= alpha q; partials of ||r||^2
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

// p = z + beta p (or p = z)
template <typename T>
__global__ void cg_p_kernel(long long n, const T* __restrict__ z, T* p, const PcgState* st, int init) {
  if (!init && *(volatile const int*)&st->done) return;
  const T b = init ? T(0) : (T)st->beta;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = init ? z[i] : z[i] + b * p[i];
}

// Reliable update: u64 += x32, x32 = 0 (only when st->update, or always with force).
__global__ void flush_kernel(long long n, double* u, float* x, const PcgState* st, int force) {
  if (!force && (*(volatile const int*)&st->done || *(volatile const int*)&st->update == 0)) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    u[i] += (double)x[i];
    x[i] = 0.0f;
  }
}

// r32 = float(r64), gated like the reliable update
__global__ void demote_kernel(long long n, const double* __restrict__ r, float* out, const PcgState* st, int force) {
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

__global__ void dense_shift_kernel(int n, double* D, double shift) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) D[(size_t)i * n + i] += shift;
}

// Fallback coarsest "inverse": the inverse diagonal of the masked dense operator.
__global__ void dense_diag_inverse_kernel(int n, const double* __restrict__ Dorig, double* Inv) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * n;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / n), j = (int)(t % n);
    const double d = Dorig[(size_t)i * n + i];
    Inv[t] = (i == j && d > 0.0) ? 1.0 / d : 0.0;
  }
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
