// Matrix-free trilinear-hexahedron elasticity operator and multigrid kernels.
//
// Replaces the reference's per-iteration CSR assembly (kron + add.at + the
// K[free][:,free] slice, pytopo3d/core/optimizer.py:584-591) and the sparse
// direct / CG solve (pytopo3d/utils/solver.py:15-73).
//
// Fine level: y = Z K(E) Z u + (I - Z) u, applied node by node from the 24x24
// element stiffness KE and the element moduli E (kernel in tp3d_fine.cuh).
// Z masks fixed DOFs.  This file holds what the fine and coarse operators
// share: modulus sources, the per-DOF epilogues of the smoother / residual /
// CG modes, the diagonal kernels and the grid transfers.
//
// Coarse levels: Galerkin operators P^T A P of the unmasked stiffness with
// trilinear P, stored as 27-point 3x3-block stencils (243 coefficients per
// node, structure-of-arrays) for the hierarchy build, and repacked DOF-major
// with the coarse fixed DOFs masked out for the apply kernels.
#pragma once

#include "tp3d_cgstate.cuh"
#include "tp3d_common.cuh"

namespace tp3d {

template <typename T>
struct KEP {
  T k[576];
};

// ----------------------------------------------------------------------------
// per-element modulus sources
// ----------------------------------------------------------------------------
struct EFromF64 {
  const double* E;
  __device__ __forceinline__ double operator()(long long e) const { return __ldg(&E[e]); }
};
struct EFromBF16 {
  const __nv_bfloat16* rho;
  float penal;
  __device__ __forceinline__ float operator()(long long e) const {
    const float r = __bfloat162float(rho[e]);
    const float rp = (penal == 3.0f) ? r * r * r : powf(r, penal);
    return 1.0e-9f + (1.0f - 1.0e-9f) * rp;
  }
};

struct EFromF32 {
  const float* E;
  __device__ __forceinline__ float operator()(long long e) const { return __ldg(&E[e]); }
};

enum ApplyMode : int {
  kModeApply = 0,      // out = K u (identity on fixed DOFs)
  kModeResid = 1,      // out = b - K u (0 on fixed DOFs)
  kModeJacobi = 2,     // out = u + omega Dinv (b - K u)
  kModeCgQ = 3,        // out = K u, partials += u . out
  kModeChebFirst = 4,  // d = c0 Dinv (b - K u); out = u + d
  kModeChebStep = 5,   // d = c1 d + c2 Dinv (b - K u); out = u + d
  kModeDinvApply = 6,  // out = Dinv K u (power iteration for lambda_max(Dinv K))
  kModeChebStepDot = 7,  // Chebyshev step (first step when io.step == 0), and partials += b . out
};

// Inputs / outputs shared by every operator kernel.
template <typename T>
struct OpIO {
  const T* u = nullptr;
  T* out = nullptr;
  const T* b = nullptr;
  const T* dinv = nullptr;
  T* d = nullptr;                // Chebyshev direction (read-modify-write at own DOF)
  const double* coef = nullptr;  // Chebyshev coefficients [c0, -, c1_1, c2_1, c1_2, c2_2, ...]
  int step = 0;
  T omega = T(0);
  double* partials = nullptr;
  const int* done = nullptr;  // skip when *done != 0
  const int* gate = nullptr;  // skip when *gate == 0
  // reductions (kModeCgQ, kModeChebStepDot): when fin_count is set, the last
  // block finishes the reduction and applies finalize op fin_op to *fin
  PcgState* fin = nullptr;
  int fin_op = 0;
  unsigned int* fin_count = nullptr;
};

template <typename T>
__device__ __forceinline__ bool op_skip(const OpIO<T>& io) {
  return (io.done && *(volatile const int*)io.done) || (io.gate && *(volatile const int*)io.gate == 0);
}

// Per-DOF epilogue inputs, loaded before the operator's FMAs so that their
// latency overlaps the arithmetic.
template <typename T>
struct EpiIn {
  T b = T(0), dinv = T(0), d = T(0);
};

template <int MODE>
__host__ __device__ constexpr bool epi_reads_b() {
  return MODE == kModeResid || MODE == kModeJacobi || MODE == kModeChebFirst || MODE == kModeChebStep ||
         MODE == kModeChebStepDot;
}
template <int MODE>
__host__ __device__ constexpr bool epi_reads_dinv() {
  return MODE == kModeJacobi || MODE == kModeChebFirst || MODE == kModeChebStep || MODE == kModeDinvApply ||
         MODE == kModeChebStepDot;
}
template <int MODE>
__host__ __device__ constexpr bool mode_reduces() {
  return MODE == kModeCgQ || MODE == kModeChebStepDot;
}

template <typename T, int MODE>
__device__ __forceinline__ EpiIn<T> epi_load(const OpIO<T>& io, long long i) {
  EpiIn<T> in;
  if (epi_reads_b<MODE>()) in.b = io.b[i];
  if (epi_reads_dinv<MODE>()) in.dinv = io.dinv[i];
  if (MODE == kModeChebStep || MODE == kModeChebStepDot) in.d = io.d[i];
  return in;
}

// Per-DOF epilogue; `own` is this DOF's input value (0 on fixed DOFs).
template <typename T, int MODE>
__device__ __forceinline__ void op_epilogue(const OpIO<T>& io, long long i, bool fx, T kv, T own, const EpiIn<T>& in,
                                            double& part) {
  if (MODE == kModeApply) {
    io.out[i] = fx ? io.u[i] : kv;
  } else if (MODE == kModeResid) {
    io.out[i] = fx ? T(0) : in.b - kv;
  } else if (MODE == kModeJacobi) {
    io.out[i] = fx ? T(0) : own + io.omega * in.dinv * (in.b - kv);
  } else if (MODE == kModeCgQ) {
    const T q = fx ? T(0) : kv;
    io.out[i] = q;
    part += (double)own * (double)q;
  } else if (MODE == kModeChebFirst) {
    const T dd = fx ? T(0) : (T)io.coef[0] * in.dinv * (in.b - kv);
    io.d[i] = dd;
    io.out[i] = own + dd;
  } else if (MODE == kModeChebStep) {
    const T dd = fx ? T(0) : (T)io.coef[2 * io.step] * in.d + (T)io.coef[2 * io.step + 1] * in.dinv * (in.b - kv);
    io.d[i] = dd;
    io.out[i] = own + dd;
  } else if (MODE == kModeChebStepDot) {
    T dd;
    if (io.step == 0) dd = fx ? T(0) : (T)io.coef[0] * in.dinv * (in.b - kv);
    else dd = fx ? T(0) : (T)io.coef[2 * io.step] * in.d + (T)io.coef[2 * io.step + 1] * in.dinv * (in.b - kv);
    io.d[i] = dd;
    const T z = own + dd;
    io.out[i] = z;
    part += (double)in.b * (double)z;
  } else {  // kModeDinvApply
    io.out[i] = fx ? T(0) : in.dinv * kv;
  }
}

// Diagonal of the fine operator: D[n,c] = sum_e E_e KE[3a+c][3a+c]; 1 on fixed DOFs.
// Writes its inverse.
template <typename T, class ESrc>
__global__ void fine_diag_inv_kernel(Grid g, const __grid_constant__ KEP<double> ke, ESrc esrc,
                                     const uint8_t* __restrict__ fix, T* dinv) {
  const int NX = g.nx + 1, NY = g.ny + 1;
  const long long nn = g.nnode();
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn; n += (long long)gridDim.x * blockDim.x) {
    const int iy = (int)(n % NY);
    const long long r = n / NY;
    const int ix = (int)(r % NX), iz = (int)(r / NX);
    double d[3] = {0, 0, 0};
#pragma unroll
    for (int ez = -1; ez <= 0; ++ez)
#pragma unroll
      for (int ex = -1; ex <= 0; ++ex)
#pragma unroll
        for (int ey = -1; ey <= 0; ++ey) {
          const int x = ix + ex, y = iy + ey, z = iz + ez;
          if (x < 0 || x >= g.nx || y < 0 || y >= g.ny || z < 0 || z >= g.nz) continue;
          const double E = (double)esrc(g.eidx(x, y, z));
          const int a = corner_index(-ex, -ey, -ez);
#pragma unroll
          for (int c = 0; c < 3; ++c) d[c] += E * ke.k[(3 * a + c) * 24 + 3 * a + c];
        }
    const int f = fix[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) dinv[3 * n + c] = ((f >> c) & 1) || !(d[c] > 0.0) ? T(0) : (T)(1.0 / d[c]);
  }
}

// ----------------------------------------------------------------------------
// 27-point block-stencil levels
// ----------------------------------------------------------------------------
// coefficient index k = (jrel * 3 + c) * 3 + d, jrel = (dz+1)*9 + (dx+1)*3 + (dy+1);
// storage A[k * nn + node].
__host__ __device__ constexpr int stencil_k(int jrel, int c, int d) { return (jrel * 3 + c) * 3 + d; }
__host__ __device__ constexpr int jrel_of(int dx, int dy, int dz) { return (dz + 1) * 9 + (dx + 1) * 3 + (dy + 1); }

// Apply layout ("packed"): S[(jrel * 3 + d) * ndof + 3 n + c] = A[(n,c),(m,d)]
// with m = n + offset(jrel), set to zero wherever DOF (n,c) or (m,d) is fixed
// or m lies outside the grid.  One thread owns one DOF, so every coefficient
// load of a warp is one contiguous run, and the masking needs no mask loads
// for the neighbours.
template <typename T>
__global__ void stencil_pack_kernel(Grid g, const double* __restrict__ A, const uint8_t* __restrict__ fix, T* S) {
  const int NX = g.nx + 1, NY = g.ny + 1, NZ = g.nz + 1;
  const long long nn = g.nnode(), ndof = 3 * nn;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ndof; i += (long long)gridDim.x * blockDim.x) {
    const long long n = i / 3;
    const int c = (int)(i - 3 * n);
    const int iy = (int)(n % NY);
    const long long r = n / NY;
    const int ix = (int)(r % NX), iz = (int)(r / NX);
    const bool fi = (fix[n] >> c) & 1;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy) {
          const int x = ix + dx, y = iy + dy, z = iz + dz;
          const bool in = x >= 0 && x < NX && y >= 0 && y < NY && z >= 0 && z < NZ;
          const int fm = in ? fix[g.nidx(x, y, z)] : 7;
          const int jr = jrel_of(dx, dy, dz);
          for (int d = 0; d < 3; ++d) {
            const double v = (fi || ((fm >> d) & 1)) ? 0.0 : A[(long long)stencil_k(jr, c, d) * nn + n];
            S[(long long)(jr * 3 + d) * ndof + i] = (T)v;
          }
        }
  }
}

// Packed layout with bf16 coefficients (the mixed form's level-1 option):
// symmetric by construction, each coupling the mean of its two FP64 copies
// rounded once, so the operator the FP32 smoother sees stays symmetric.
template <typename TS>
__global__ void stencil_pack_sym_kernel(Grid g, const double* __restrict__ A, const uint8_t* __restrict__ fix,
                                        TS* S) {
  const int NX = g.nx + 1, NY = g.ny + 1, NZ = g.nz + 1;
  const long long nn = g.nnode(), ndof = 3 * nn;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ndof; i += (long long)gridDim.x * blockDim.x) {
    const long long n = i / 3;
    const int c = (int)(i - 3 * n);
    const int iy = (int)(n % NY);
    const long long r = n / NY;
    const int ix = (int)(r % NX), iz = (int)(r / NX);
    const bool fi = (fix[n] >> c) & 1;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy) {
          const int x = ix + dx, y = iy + dy, z = iz + dz;
          const bool in = x >= 0 && x < NX && y >= 0 && y < NY && z >= 0 && z < NZ;
          const long long m = in ? g.nidx(x, y, z) : n;
          const int fm = in ? fix[m] : 7;
          const int jr = jrel_of(dx, dy, dz);
          for (int d = 0; d < 3; ++d) {
            const double v = (fi || ((fm >> d) & 1))
                                 ? 0.0
                                 : 0.5 * (A[(long long)stencil_k(jr, c, d) * nn + n] +
                                          A[(long long)stencil_k(26 - jr, d, c) * nn + m]);
            S[(long long)(jr * 3 + d) * ndof + i] = TS(v);
          }
        }
  }
}

template <typename T, typename TS = T>
struct StencilParams {
  Grid g;
  const TS* S;  // packed layout
  const uint8_t* fix;
  OpIO<T> io;
};

// Load policies of the operator device functions: LdRO through the read-only
// path (data no kernel writes during the launch), LdL2 at L2 (data written
// earlier in the same launch by other blocks), LdPlain for shared memory.
struct LdRO {
  template <typename V>
  __device__ __forceinline__ V operator()(const V* p) const { return __ldg(p); }
};
struct LdL2 {
  template <typename V>
  __device__ __forceinline__ V operator()(const V* p) const { return __ldcg(p); }
};
struct LdPlain {
  template <typename V>
  __device__ __forceinline__ V operator()(const V* p) const { return *p; }
};

template <typename T, class Ld = LdRO>
__device__ __forceinline__ T ld_coef(const T* p) { return Ld()(p); }
template <typename T, class Ld = LdRO>
__device__ __forceinline__ T ld_coef(const __nv_bfloat16* p) { return (T)__bfloat162float(Ld()(p)); }

// One DOF per thread: 81 coalesced coefficient loads and 81 neighbour loads,
// all independent (offsets past the grid are clamped to the node itself and
// meet a zero coefficient), so a thread waits for memory about once.  Coarse
// levels hold far fewer than 2^31 DOFs: 32-bit index arithmetic.
// Row i of the packed stencil times u (K u at DOF i; fixed rows and columns are
// zero in the packed layout).
template <typename T, typename TS = T, class Ld = LdRO>
__device__ __forceinline__ T stencil_row(const Grid& g, const TS* __restrict__ S, const T* __restrict__ u, int i) {
  const Ld ld;
  const int NX = g.nx + 1, NY = g.ny + 1, NZ = g.nz + 1;
  const int NXY = NX * NY;
  const int ndof = 3 * NXY * NZ;
  const int n = i / 3;
  const int iy = n % NY, r = n / NY;
  const int ix = r % NX, iz = r / NX;
  const int oy0 = iy > 0 ? -1 : 0, oy2 = iy < NY - 1 ? 1 : 0;
  const int ox0 = ix > 0 ? -NY : 0, ox2 = ix < NX - 1 ? NY : 0;
  const int oz0 = iz > 0 ? -NXY : 0, oz2 = iz < NZ - 1 ? NXY : 0;
  T kv = T(0);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int oz = a == 0 ? oz0 : (a == 1 ? 0 : oz2);
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const int ox = b == 0 ? ox0 : (b == 1 ? 0 : ox2);
#pragma unroll
      for (int e = 0; e < 3; ++e) {
        const int oy = e == 0 ? oy0 : (e == 1 ? 0 : oy2);
        const int m3 = 3 * (n + oz + ox + oy);
        const TS* s = S + (size_t)((a * 9 + b * 3 + e) * 3) * ndof + i;
        kv = fma(ld_coef<T, Ld>(s), ld(&u[m3]), kv);
        kv = fma(ld_coef<T, Ld>(s + ndof), ld(&u[m3 + 1]), kv);
        kv = fma(ld_coef<T, Ld>(s + 2 * (size_t)ndof), ld(&u[m3 + 2]), kv);
      }
    }
  }
  return kv;
}

template <typename T, int MODE, typename TS = T>
__global__ void __launch_bounds__(256) stencil_apply_kernel(const __grid_constant__ StencilParams<T, TS> p) {
  pdl_entry();
  if (op_skip(p.io)) return;
  __shared__ double red[32];
  const Grid g = p.g;
  const int ndof = 3 * (g.nx + 1) * (g.ny + 1) * (g.nz + 1);
  const T* __restrict__ u = p.io.u;
  double part = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ndof; i += gridDim.x * blockDim.x) {
    const int n = i / 3, c = i - 3 * n;
    const T kv = stencil_row<T, TS>(g, p.S, u, i);
    const bool fx = (p.fix[n] >> c) & 1;
    op_epilogue<T, MODE>(p.io, i, fx, kv, fx ? T(0) : u[i], epi_load<T, MODE>(p.io, i), part);
  }
  if (mode_reduces<MODE>()) {
    part = block_sum(part, red);
    if (threadIdx.x == 0) p.io.partials[blockIdx.x] = part;
    if (p.io.fin_count) last_block_finalize(p.io.partials, gridDim.x, p.io.fin_count, p.io.fin, p.io.fin_op, red);
  }
}

// The same operator with four lanes per DOF, for the small coarse levels,
// where a launch holds too few threads to keep the memory system busy and each
// thread's 162 loads are the critical path: lane q of a group of four
// multiplies neighbours 7q .. 7q+6 of the 27 (in stencil_row's z, x, y order),
// the group adds its partial sums with two xor shuffles and its first lane
// runs the epilogue.  The loop bound is uniform over each block, so every lane
// reaches the shuffles.
template <typename T, typename TS>
__device__ __forceinline__ T stencil_row_part(const Grid& g, const TS* __restrict__ S, const T* __restrict__ u, int i,
                                              int q) {
  const int NX = g.nx + 1, NY = g.ny + 1, NZ = g.nz + 1;
  const int NXY = NX * NY;
  const int ndof = 3 * NXY * NZ;
  const int n = i / 3;
  const int iy = n % NY, r = n / NY;
  const int ix = r % NX, iz = r / NX;
  const int oy0 = iy > 0 ? -1 : 0, oy2 = iy < NY - 1 ? 1 : 0;
  const int ox0 = ix > 0 ? -NY : 0, ox2 = ix < NX - 1 ? NY : 0;
  const int oz0 = iz > 0 ? -NXY : 0, oz2 = iz < NZ - 1 ? NXY : 0;
  T kv = T(0);
#pragma unroll
  for (int jj = 0; jj < 7; ++jj) {
    const int j = 7 * q + jj;
    if (j < 27) {
      const int a = j / 9, b = (j / 3) % 3, e = j % 3;
      const int oz = a == 0 ? oz0 : (a == 1 ? 0 : oz2);
      const int ox = b == 0 ? ox0 : (b == 1 ? 0 : ox2);
      const int oy = e == 0 ? oy0 : (e == 1 ? 0 : oy2);
      const int m3 = 3 * (n + oz + ox + oy);
      const TS* s = S + (size_t)(j * 3) * ndof + i;
      kv = fma(ld_coef<T>(s), __ldg(&u[m3]), kv);
      kv = fma(ld_coef<T>(s + ndof), __ldg(&u[m3 + 1]), kv);
      kv = fma(ld_coef<T>(s + 2 * (size_t)ndof), __ldg(&u[m3 + 2]), kv);
    }
  }
  return kv;
}

template <typename T, int MODE, typename TS = T>
__global__ void __launch_bounds__(256) stencil_apply4_kernel(const __grid_constant__ StencilParams<T, TS> p) {
  pdl_entry();
  if (op_skip(p.io)) return;
  __shared__ double red[32];
  const Grid g = p.g;
  const int ndof = 3 * (g.nx + 1) * (g.ny + 1) * (g.nz + 1);
  const T* __restrict__ u = p.io.u;
  const int q = threadIdx.x & 3;
  double part = 0.0;
  for (int base = blockIdx.x * blockDim.x; base < 4 * ndof; base += gridDim.x * blockDim.x) {
    const int i = (base + threadIdx.x) >> 2;
    const bool live = i < ndof;
    EpiIn<T> in;
    if (live && q == 0) in = epi_load<T, MODE>(p.io, i);
    T kv = live ? stencil_row_part<T, TS>(g, p.S, u, i, q) : T(0);
    kv += __shfl_xor_sync(0xffffffffu, kv, 1);
    kv += __shfl_xor_sync(0xffffffffu, kv, 2);
    if (live && q == 0) {
      const int n = i / 3, c = i - 3 * n;
      const bool fx = (p.fix[n] >> c) & 1;
      op_epilogue<T, MODE>(p.io, i, fx, kv, fx ? T(0) : u[i], in, part);
    }
  }
  if (mode_reduces<MODE>()) {
    part = block_sum(part, red);
    if (threadIdx.x == 0) p.io.partials[blockIdx.x] = part;
    if (p.io.fin_count) last_block_finalize(p.io.partials, gridDim.x, p.io.fin_count, p.io.fin, p.io.fin_op, red);
  }
}

template <typename T>
__global__ void stencil_diag_inv_kernel(Grid g, const double* __restrict__ A, const uint8_t* __restrict__ fix,
                                        T* dinv) {
  const long long nn = g.nnode();
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn; n += (long long)gridDim.x * blockDim.x) {
    const int f = fix[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double d = A[(long long)stencil_k(13, c, c) * nn + n];
      dinv[3 * n + c] = (((f >> c) & 1) || !(d > 0.0)) ? T(0) : (T)(1.0 / d);
    }
  }
}

// First smoothing step from a zero guess: x = w dinv b, with w = omega or (coef
// given) the Chebyshev c0; d (if given) receives the same step.
template <typename T>
__global__ void smooth_zero_kernel(long long ndof, const T* __restrict__ b, const T* __restrict__ dinv, T omega,
                                   const double* coef, T* x, T* d, const int* done) {
  pdl_entry();
  if (done && *(volatile const int*)done) return;
  const T w = coef ? (T)coef[0] : omega;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ndof; i += (long long)gridDim.x * blockDim.x) {
    const T v = w * dinv[i] * b[i];
    x[i] = v;
    if (d) d[i] = v;
  }
}

// ----------------------------------------------------------------------------
// grid transfer (trilinear, vertex-centred coarsening by 2)
// ----------------------------------------------------------------------------
// coarse element grid of a fine element grid
__host__ __device__ inline Grid coarse_grid(const Grid& f) {
  return Grid{(f.nx + 1) / 2, (f.ny + 1) / 2, (f.nz + 1) / 2};
}

// Grid transfers run one thread per node of an (x, y) plane, blockIdx.y = z
// (one integer division per thread), and handle the node's three components.
inline dim3 plane_grid(int nxy, int nz) { return dim3((unsigned)((nxy + 255) / 256), (unsigned)nz); }

// b_c[I] = sum_i P[i,I] r_f[i], 0 on fixed coarse DOFs.  The 27 fine
// neighbours are read unconditionally (offsets past the fine grid are clamped
// and weighted 0), so the loads are independent.  Grid: plane_grid(CX*CY, CZ).
template <typename T, class Ld = LdRO>
__device__ __forceinline__ void restrict_node(const Grid& gf, const Grid& gc, const T* __restrict__ rf,
                                              const uint8_t* __restrict__ fixc, T* bc, int Ix, int Iy, int Iz) {
  const Ld ld;
  const int FX = gf.nx + 1, FY = gf.ny + 1, FZ = gf.nz + 1;
  const int CX = gc.nx + 1, CY = gc.ny + 1;
  const int FXY = FX * FY;
  T s0 = T(0), s1 = T(0), s2 = T(0);
#pragma unroll
  for (int dz = -1; dz <= 1; ++dz) {
    const int z = 2 * Iz + dz;
    const bool vz = z >= 0 && z < FZ;
#pragma unroll
    for (int dx = -1; dx <= 1; ++dx) {
      const int x = 2 * Ix + dx;
      const bool vx = x >= 0 && x < FX;
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy) {
        const int y = 2 * Iy + dy;
        const bool v = vz && vx && y >= 0 && y < FY;
        const T w = v ? T((dx ? 0.5 : 1.0) * (dy ? 0.5 : 1.0) * (dz ? 0.5 : 1.0)) : T(0);
        const T* src = rf + 3 * (v ? y + FY * x + FXY * z : 0);
        s0 = fma(w, ld(src), s0);
        s1 = fma(w, ld(src + 1), s1);
        s2 = fma(w, ld(src + 2), s2);
      }
    }
  }
  const long long n = Iy + (long long)CY * (Ix + (long long)CX * Iz);
  const int f = fixc[n];
  T* dst = bc + 3 * n;
  dst[0] = (f & 1) ? T(0) : s0;
  dst[1] = (f & 2) ? T(0) : s1;
  dst[2] = (f & 4) ? T(0) : s2;
}

// First smoothing step of the coarse level from a zero guess, fused into the
// restriction (it is pointwise): x0 = w dinv b with w = omega or (coef given)
// the Chebyshev c0, and d = x0 when d is given.  x0 == nullptr: none.
template <typename T>
struct CoarseFirstStep {
  const T* dinv = nullptr;
  const double* coef = nullptr;
  T omega = T(0);
  T* x0 = nullptr;
  T* d = nullptr;
};

template <typename T>
__global__ void __launch_bounds__(256) restrict_kernel(Grid gf, Grid gc, const T* __restrict__ rf,
                                                       const uint8_t* __restrict__ fixc, T* bc, const int* done,
                                                       CoarseFirstStep<T> fs) {
  pdl_entry();
  if (done && *(volatile const int*)done) return;
  const int CY = gc.ny + 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (gc.nx + 1) * CY) return;
  const int Ix = t / CY, Iy = t - Ix * CY;
  restrict_node<T>(gf, gc, rf, fixc, bc, Ix, Iy, blockIdx.y);
  if (fs.x0) {
    const T w = fs.coef ? (T)fs.coef[0] : fs.omega;
    const long long n = Iy + (long long)CY * (Ix + (long long)(gc.nx + 1) * blockIdx.y);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const long long i = 3 * n + c;
      const T v = w * fs.dinv[i] * bc[i];
      fs.x0[i] = v;
      if (fs.d) fs.d[i] = v;
    }
  }
}

// Residual and restriction in one launch, for small levels: one block per
// coarse node, thread q < 81 of it computes the residual of fine DOF q of the
// node's 3 x 3 x 3 fine neighbourhood (node q / 3 in the (z, x, y) order of
// restrict_node, component q % 3) from the fine stencil, weighted by the
// trilinear restriction weight; the block sums the 27 weighted residuals of
// each component in a fixed order.  Each fine residual is computed by up to 8
// coarse nodes' blocks: on a level of a few thousand DOFs that costs less than
// the launch it saves.  The coarse level's first smoothing step rides along as
// in restrict_kernel.
constexpr int kRestrictResidThreads = 96;

template <typename T, typename TS>
__global__ void __launch_bounds__(kRestrictResidThreads) restrict_resid_kernel(
    const __grid_constant__ StencilParams<T, TS> p, Grid gc, const uint8_t* __restrict__ fixc, T* bc,
    CoarseFirstStep<T> fs) {
  pdl_entry();
  if (op_skip(p.io)) return;
  __shared__ T part[81];
  const Grid& gf = p.g;
  const int FX = gf.nx + 1, FY = gf.ny + 1, FZ = gf.nz + 1;
  const int CX = gc.nx + 1, CY = gc.ny + 1;
  const int N = blockIdx.x;
  const int Iy = N % CY, rN = N / CY;
  const int Ix = rN % CX, Iz = rN / CX;
  const int q = threadIdx.x;
  if (q < 81) {
    const int j = q / 3, c = q - 3 * j;
    const int dz = j / 9 - 1, dx = (j / 3) % 3 - 1, dy = j % 3 - 1;
    const int x = 2 * Ix + dx, y = 2 * Iy + dy, z = 2 * Iz + dz;
    T v = T(0);
    if (x >= 0 && x < FX && y >= 0 && y < FY && z >= 0 && z < FZ) {
      const int n = y + FY * (x + FX * z);
      const int i = 3 * n + c;
      if (!((p.fix[n] >> c) & 1)) {
        const T w = T((dx ? 0.5 : 1.0) * (dy ? 0.5 : 1.0) * (dz ? 0.5 : 1.0));
        v = w * (p.io.b[i] - stencil_row<T, TS>(gf, p.S, p.io.u, i));
      }
    }
    part[q] = v;
  }
  __syncthreads();
  if (q < 3) {
    T sum = T(0);
    for (int j = 0; j < 27; ++j) sum += part[3 * j + q];
    const int i = 3 * N + q;
    const T bv = ((fixc[N] >> q) & 1) ? T(0) : sum;
    bc[i] = bv;
    if (fs.x0) {
      const T w = fs.coef ? (T)fs.coef[0] : fs.omega;
      const T v0 = w * fs.dinv[i] * bv;
      fs.x0[i] = v0;
      if (fs.d) fs.d[i] = v0;
    }
  }
}

// x_f[i] += sum_I P[i,I] x_c[I] on free fine DOFs.  A fine node takes 1, 2, 4
// or 8 coarse nodes (weights 1 or 1/2 per axis), read as a fixed 2x2x2 block
// with zero weights for the absent ones.  Grid: plane_grid(FX*FY, FZ).
template <typename T, class Ld = LdRO>
__device__ __forceinline__ void prolong_node(const Grid& gf, const Grid& gc, const T* __restrict__ xc,
                                             const uint8_t* __restrict__ fixf, T* xf, int ix, int iy, int iz) {
  const Ld ld;
  const int FX = gf.nx + 1, FY = gf.ny + 1;
  const int CX = gc.nx + 1, CY = gc.ny + 1;
  const long long n = iy + (long long)FY * (ix + (long long)FX * iz);
  const int f = fixf[n];
  if (f == 7) return;
  const int oy = iy & 1, ox = ix & 1, oz = iz & 1;
  const int CXY = CX * CY;
  const int base = (iy >> 1) + CY * (ix >> 1) + CXY * (iz >> 1);
  const T h = T(0.5);
  T s0 = T(0), s1 = T(0), s2 = T(0);
#pragma unroll
  for (int a = 0; a < 2; ++a) {
    const T wz = oz ? h : (a ? T(0) : T(1));
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const T wx = ox ? h : (b ? T(0) : T(1));
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const T wy = oy ? h : (e ? T(0) : T(1));
        const T w = wz * wx * wy;
        const T* src = xc + 3 * (base + (e & oy) + CY * (b & ox) + CXY * (a & oz));
        s0 = fma(w, ld(src), s0);
        s1 = fma(w, ld(src + 1), s1);
        s2 = fma(w, ld(src + 2), s2);
      }
    }
  }
  T* dst = xf + 3 * n;
  if (!(f & 1)) dst[0] += s0;
  if (!(f & 2)) dst[1] += s1;
  if (!(f & 4)) dst[2] += s2;
}

template <typename T>
__global__ void __launch_bounds__(256) prolong_add_kernel(Grid gf, Grid gc, const T* __restrict__ xc,
                                                          const uint8_t* __restrict__ fixf, T* xf, const int* done) {
  pdl_entry();
  if (done && *(volatile const int*)done) return;
  const int FY = gf.ny + 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (gf.nx + 1) * FY) return;
  const int ix = t / FY;
  prolong_node<T>(gf, gc, xc, fixf, xf, ix, t - ix * FY, blockIdx.y);
}

}  // namespace tp3d
