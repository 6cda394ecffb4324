// The coarse end of the multigrid V-cycle in one cooperative launch.
//
// Below a few ten thousand DOFs a level's smoothing step, residual and grid
// transfer each touch too little data to fill the GPU, so as separate
// launches they cost their launch and drain latency, not their work.  This
// kernel runs the whole cycle from level L0 down to the dense coarsest level
// and back up (Chebyshev or damped-Jacobi smoothing, residual, restriction,
// coarsest matvec, prolongation) with a grid-wide barrier between dependent
// phases.  It computes exactly what the per-phase kernels compute: every phase
// is the same per-DOF / per-node device function, over a grid-stride loop.
//
// The barrier is bounded (grid_sync_flip): a block that waits too long raises
// the error flag, sets the CG state to "device wait expired" and leaves, so
// the host sees an error instead of a hang.
#pragma once

#include "tp3d_hex.cuh"

namespace tp3d {

constexpr int kCycleMaxLevels = 16;

template <typename T>
struct CycleLevel {
  Grid g{};
  const T* S = nullptr;  // packed stencil (levels >= 1)
  const uint8_t* fix = nullptr;
  const T* dinv = nullptr;
  const double* coef = nullptr;  // Chebyshev coefficients
  T* x[2] = {nullptr, nullptr};
  T* b = nullptr;
  T* r = nullptr;
  T* d = nullptr;
};

template <typename T>
struct CycleParams {
  CycleLevel<T> lv[kCycleMaxLevels];
  int L0 = 1, Lc = 1;  // first level of the cycle, coarsest (dense) level
  int pre = 2, post = 2;
  int cheb = 1;  // 1 Chebyshev, 0 damped Jacobi
  T omega = T(0);
  int cn = 0;               // coarsest dense size
  const T* inv = nullptr;   // its inverse, row-major
  int* done = nullptr;      // CG stop flag: skip when set; set to 7 when a barrier expires
  unsigned int* bar = nullptr;  // grid_sync_flip word
  int* bar_err = nullptr;
};

// Buffer index holding the smoothed iterate of a non-coarsest level after its
// cycle (the first smoothing step writes x[0], every later step flips).
__host__ __device__ constexpr int cycle_final_buffer(int pre, int post) { return (pre - 1 + post) & 1; }

// One smoothing step on level lv from x[cur] into x[1 - cur]: step index s of
// the Chebyshev recurrence (s == 0 starts a new recurrence) or damped Jacobi.
template <typename T, int MODE>
__device__ __forceinline__ void cycle_smooth_dof(const CycleLevel<T>& lv, int cur, int s, T omega, int i) {
  OpIO<T> io;
  io.u = lv.x[cur];
  io.out = lv.x[1 - cur];
  io.b = lv.b;
  io.dinv = lv.dinv;
  io.d = lv.d;
  io.coef = lv.coef;
  io.step = s;
  io.omega = omega;
  const int n = i / 3, c = i - 3 * n;
  const T kv = stencil_row<T, T, LdL2>(lv.g, lv.S, io.u, i);
  const bool fx = (lv.fix[n] >> c) & 1;
  double part = 0.0;
  op_epilogue<T, MODE>(io, i, fx, kv, fx ? T(0) : io.u[i], epi_load<T, MODE>(io, i), part);
}

template <typename T>
__global__ void __launch_bounds__(256) coarse_cycle_kernel(const __grid_constant__ CycleParams<T> p) {
  if (p.done && *(volatile const int*)p.done) return;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  auto sync = [&]() -> bool {
    if (grid_sync_flip(p.bar, p.bar_err)) return true;
    if (threadIdx.x == 0 && p.done) atomicExch(p.done, 7);
    return false;
  };
  auto smooth = [&](const CycleLevel<T>& lv, int cur, int s, bool first) -> bool {
    const int ndof = (int)(3 * lv.g.nnode());
    for (int i = tid; i < ndof; i += nth) {
      if (!p.cheb) cycle_smooth_dof<T, kModeJacobi>(lv, cur, s, p.omega, i);
      else if (first) cycle_smooth_dof<T, kModeChebFirst>(lv, cur, s, p.omega, i);
      else cycle_smooth_dof<T, kModeChebStep>(lv, cur, s, p.omega, i);
    }
    return sync();
  };

  // down: smooth from zero, residual, restriction.  The first smoothing step
  // from zero is pointwise, so below L0 it runs in the restriction's phase.
  auto smooth_zero = [&](const CycleLevel<T>& lv, int i) {
    const T w = p.cheb ? (T)lv.coef[0] : p.omega;
    const T v = w * lv.dinv[i] * lv.b[i];
    lv.x[0][i] = v;
    if (p.cheb) lv.d[i] = v;
  };
  if (p.L0 < p.Lc) {
    const int ndof = (int)(3 * p.lv[p.L0].g.nnode());
    for (int i = tid; i < ndof; i += nth) smooth_zero(p.lv[p.L0], i);
    if (!sync()) return;
  }
  for (int L = p.L0; L < p.Lc; ++L) {
    const CycleLevel<T>& lv = p.lv[L];
    const int ndof = (int)(3 * lv.g.nnode());
    int cur = 0;
    for (int s = 1; s < p.pre; ++s) {
      if (!smooth(lv, cur, s, false)) return;
      cur ^= 1;
    }
    for (int i = tid; i < ndof; i += nth) {
      const int n = i / 3, c = i - 3 * n;
      const bool fx = (lv.fix[n] >> c) & 1;
      lv.r[i] = fx ? T(0) : lv.b[i] - stencil_row<T, T, LdL2>(lv.g, lv.S, lv.x[cur], i);
    }
    if (!sync()) return;
    const CycleLevel<T>& lc = p.lv[L + 1];
    const int CX = lc.g.nx + 1, CY = lc.g.ny + 1;
    const int nnc = (int)lc.g.nnode();
    const bool smooth_next = L + 1 < p.Lc;
    for (int n = tid; n < nnc; n += nth) {
      const int Iy = n % CY, r = n / CY;
      restrict_node<T, LdL2>(lv.g, lc.g, lv.r, lc.fix, lc.b, r % CX, Iy, r / CX);
      if (smooth_next)
        for (int c = 0; c < 3; ++c) smooth_zero(lc, 3 * n + c);
    }
    if (!sync()) return;
  }
  // coarsest: x = Inv b, a warp per row
  {
    const CycleLevel<T>& lc = p.lv[p.Lc];
    const int warp = tid >> 5, lane = threadIdx.x & 31, nwarps = nth >> 5;
    for (int i = warp; i < p.cn; i += nwarps) {
      double s = 0.0;
      for (int j = lane; j < p.cn; j += 32) s += (double)p.inv[(size_t)i * p.cn + j] * (double)lc.b[j];
      s = warp_sum(s);
      if (lane == 0) lc.x[0][i] = (T)s;
    }
    if (!sync()) return;
  }
  // up: prolongation, post-smoothing
  for (int L = p.Lc - 1; L >= p.L0; --L) {
    const CycleLevel<T>& lv = p.lv[L];
    const CycleLevel<T>& lc = p.lv[L + 1];
    const T* xc = (L + 1 == p.Lc) ? lc.x[0] : lc.x[cycle_final_buffer(p.pre, p.post)];
    int cur = (p.pre - 1) & 1;
    const int FX = lv.g.nx + 1, FY = lv.g.ny + 1;
    const int nnf = (int)lv.g.nnode();
    for (int n = tid; n < nnf; n += nth) {
      const int iy = n % FY, r = n / FY;
      prolong_node<T, LdL2>(lv.g, lc.g, xc, lv.fix, lv.x[cur], r % FX, iy, r / FX);
    }
    if (!sync()) return;
    for (int s = 0; s < p.post; ++s) {
      if (!smooth(lv, cur, s, s == 0)) return;
      cur ^= 1;
    }
  }
}

}  // namespace tp3d
