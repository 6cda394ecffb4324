// The last smoothed level of the V-cycle and the coarsest solve in one thread
// block, with the level's operator in shared memory.
//
// At the bottom of the hierarchy a level holds a few hundred nodes: each of
// its smoothing steps, its residual, the grid transfers and the coarsest
// matrix-vector product, launched separately, cost a kernel's launch, ramp
// and drain for microseconds of work.  Here one block of 1024 threads runs the
// level's whole cycle with block barriers between the phases: it stages the
// level's packed stencil (bf16 or FP32), diagonal, masks and vectors in shared
// memory once, smooths, restricts the residual, multiplies by the coarsest
// inverse (read from global memory once), prolongs and smooths again, and
// writes the level's iterate back.  Every phase calls the same per-DOF and
// per-node device functions as the separate kernels, with plain loads from
// shared memory, so it computes what they compute.
#pragma once

#include "tp3d_hex.cuh"

namespace tp3d {

constexpr int kDeepThreads = 1024;

template <typename T, typename TS>
struct DeepParams {
  Grid g{}, gc{};               // the level and the coarsest level
  const TS* S = nullptr;        // the level's packed stencil
  const uint8_t* fix = nullptr;   // the level's node masks
  const uint8_t* fixc = nullptr;  // the coarsest level's node masks
  const T* dinv = nullptr;
  const double* coef = nullptr;  // Chebyshev coefficients of the level
  const T* inv = nullptr;        // coarsest inverse, cn x cn row-major
  int cn = 0;
  const T* b = nullptr;          // the level's right-hand side
  const T* x0 = nullptr;         // its first smoothing step (written by the restriction)
  const T* d0 = nullptr;         // and that step's Chebyshev direction
  T* xout = nullptr;             // the level's iterate after the cycle
  int pre = 1, post = 1;         // smoothing degrees (pre counts the step already taken)
  int cheb = 1;                  // 1 Chebyshev, 0 damped Jacobi
  T omega = T(0);
  const int* done = nullptr;
};

// Shared-memory bytes of the block for a level of `nn` nodes and a coarsest
// level of `nnc` nodes: stencil (81 coefficients per DOF), six level vectors
// (x[2], b, d, dinv, r), two coarsest vectors, node masks; 16-byte aligned parts.
template <typename T, typename TS>
__host__ __device__ constexpr size_t deep_smem_bytes(long long nn, long long nnc) {
  const size_t nd = (size_t)(3 * nn), ndc = (size_t)(3 * nnc);
  auto al = [](size_t x) { return (x + 15) & ~(size_t)15; };
  return al(81 * nd * sizeof(TS)) + 6 * al(nd * sizeof(T)) + 2 * al(ndc * sizeof(T)) + al((size_t)nn) +
         al((size_t)nnc);
}

template <typename T, typename TS>
__global__ void __launch_bounds__(kDeepThreads, 1) deep_cycle_kernel(const __grid_constant__ DeepParams<T, TS> p) {
  pdl_entry();
  if (p.done && *(volatile const int*)p.done) return;
  extern __shared__ __align__(16) unsigned char smem[];
  const long long nn = p.g.nnode(), nnc = p.gc.nnode();
  const int nd = (int)(3 * nn), ndc = (int)(3 * nnc);
  auto al = [](size_t x) { return (x + 15) & ~(size_t)15; };
  unsigned char* q = smem;
  TS* S = reinterpret_cast<TS*>(q);
  q += al(81 * (size_t)nd * sizeof(TS));
  T* x[2];
  x[0] = reinterpret_cast<T*>(q);
  q += al(nd * sizeof(T));
  x[1] = reinterpret_cast<T*>(q);
  q += al(nd * sizeof(T));
  T* b = reinterpret_cast<T*>(q);
  q += al(nd * sizeof(T));
  T* d = reinterpret_cast<T*>(q);
  q += al(nd * sizeof(T));
  T* dinv = reinterpret_cast<T*>(q);
  q += al(nd * sizeof(T));
  T* r = reinterpret_cast<T*>(q);
  q += al(nd * sizeof(T));
  T* bc = reinterpret_cast<T*>(q);
  q += al(ndc * sizeof(T));
  T* xc = reinterpret_cast<T*>(q);
  q += al(ndc * sizeof(T));
  uint8_t* fix = q;
  q += al((size_t)nn);
  uint8_t* fixc = q;

  const int t = threadIdx.x;
  // stage the operator (16-byte copies) and the level's state
  {
    const size_t nbytes = 81 * (size_t)nd * sizeof(TS);  // a multiple of 2 * 81 * 3 bytes
    const size_t n16 = nbytes / 16;
    const uint4* src = reinterpret_cast<const uint4*>(p.S);
    uint4* dst = reinterpret_cast<uint4*>(S);
    for (size_t k = t; k < n16; k += kDeepThreads) dst[k] = __ldg(src + k);
    const unsigned char* s8 = reinterpret_cast<const unsigned char*>(p.S);
    unsigned char* d8 = reinterpret_cast<unsigned char*>(S);
    for (size_t k = n16 * 16 + t; k < nbytes; k += kDeepThreads) d8[k] = s8[k];
  }
  for (int i = t; i < nd; i += kDeepThreads) {
    x[0][i] = p.x0[i];
    d[i] = p.d0 ? p.d0[i] : T(0);
    b[i] = p.b[i];
    dinv[i] = p.dinv[i];
  }
  for (int n = t; n < nn; n += kDeepThreads) fix[n] = p.fix[n];
  for (int n = t; n < nnc; n += kDeepThreads) fixc[n] = p.fixc[n];
  __syncthreads();

  int cur = 0;
  auto smooth = [&](int s, bool first) {
    OpIO<T> io;
    io.u = x[cur];
    io.out = x[1 - cur];
    io.b = b;
    io.dinv = dinv;
    io.d = d;
    io.coef = p.coef;
    io.step = s;
    io.omega = p.omega;
    double part = 0.0;
    for (int i = t; i < nd; i += kDeepThreads) {
      const int n = i / 3, c = i - 3 * n;
      const T kv = stencil_row<T, TS, LdPlain>(p.g, S, x[cur], i);
      const bool fx = (fix[n] >> c) & 1;
      const T own = fx ? T(0) : x[cur][i];
      if (!p.cheb) op_epilogue<T, kModeJacobi>(io, i, fx, kv, own, epi_load<T, kModeJacobi>(io, i), part);
      else if (first) op_epilogue<T, kModeChebFirst>(io, i, fx, kv, own, epi_load<T, kModeChebFirst>(io, i), part);
      else op_epilogue<T, kModeChebStep>(io, i, fx, kv, own, epi_load<T, kModeChebStep>(io, i), part);
    }
    __syncthreads();
    cur ^= 1;
  };

  // pre-smoothing (step 0 was taken by the restriction)
  for (int s = 1; s < p.pre; ++s) smooth(s, false);
  // residual
  for (int i = t; i < nd; i += kDeepThreads) {
    const int n = i / 3, c = i - 3 * n;
    const bool fx = (fix[n] >> c) & 1;
    r[i] = fx ? T(0) : b[i] - stencil_row<T, TS, LdPlain>(p.g, S, x[cur], i);
  }
  __syncthreads();
  // restriction to the coarsest level
  {
    const int CX = p.gc.nx + 1, CY = p.gc.ny + 1;
    for (int n = t; n < nnc; n += kDeepThreads) {
      const int Iy = n % CY, rr = n / CY;
      restrict_node<T, LdPlain>(p.g, p.gc, r, fixc, bc, rr % CX, Iy, rr / CX);
    }
  }
  __syncthreads();
  // coarsest solve: xc = Inv bc, a warp per row (FP64 accumulation)
  {
    const int warp = t >> 5, lane = t & 31;
    for (int i = warp; i < p.cn; i += kDeepThreads / 32) {
      double acc = 0.0;
      for (int j = lane; j < p.cn; j += 32) acc += (double)__ldg(&p.inv[(size_t)i * p.cn + j]) * (double)bc[j];
      acc = warp_sum(acc);
      if (lane == 0) xc[i] = (T)acc;
    }
  }
  __syncthreads();
  // prolongation
  {
    const int FX = p.g.nx + 1, FY = p.g.ny + 1;
    for (int n = t; n < nn; n += kDeepThreads) {
      const int iy = n % FY, rr = n / FY;
      prolong_node<T, LdPlain>(p.g, p.gc, xc, fix, x[cur], rr % FX, iy, rr / FX);
    }
  }
  __syncthreads();
  // post-smoothing
  for (int s = 0; s < p.post; ++s) smooth(s, s == 0);
  for (int i = t; i < nd; i += kDeepThreads) p.xout[i] = x[cur][i];
}

}  // namespace tp3d
