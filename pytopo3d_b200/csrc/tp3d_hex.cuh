// Matrix-free trilinear-hexahedron elasticity operator and multigrid kernels.
//
// Replaces the reference's per-iteration CSR assembly (kron + add.at + the
// K[free][:,free] slice, pytopo3d/core/optimizer.py:584-591) and the sparse
// direct / CG solve (pytopo3d/utils/solver.py:15-73).
//
// Fine level: y = Z K(E) Z u + (I - Z) u, applied node by node from the 24x24
// element stiffness KE (kernel-parameter space, i.e. the constant bank, so
// every FMA takes its coefficient as an immediate-bank operand) and the
// element moduli E.  Z masks fixed DOFs.  A block owns a TY x TX column of
// nodes and marches along z; each step stages one new node plane of u (tile +
// 1 halo) and one element slab of E in shared memory.  Per node the 27
// neighbours are read once and fed into 8 per-element accumulators (576 FMAs
// per node, 24 independent FMA chains).
//
// Coarse levels: Galerkin operators P^T A P of the unmasked stiffness with
// trilinear P, stored as 27-point 3x3-block stencils (243 coefficients per
// node, structure-of-arrays), fixed DOFs by injection.
#pragma once

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
};

template <typename T>
__device__ __forceinline__ bool op_skip(const OpIO<T>& io) {
  return (io.done && *(volatile const int*)io.done) || (io.gate && *(volatile const int*)io.gate == 0);
}

// Per-DOF epilogue; `own` is this DOF's input value (0 on fixed DOFs).
template <typename T, int MODE>
__device__ __forceinline__ void op_epilogue(const OpIO<T>& io, long long i, bool fx, T kv, T own, double& part) {
  if (MODE == kModeApply) {
    io.out[i] = fx ? io.u[i] : kv;
  } else if (MODE == kModeResid) {
    io.out[i] = fx ? T(0) : io.b[i] - kv;
  } else if (MODE == kModeJacobi) {
    io.out[i] = fx ? T(0) : own + io.omega * io.dinv[i] * (io.b[i] - kv);
  } else if (MODE == kModeCgQ) {
    const T q = fx ? T(0) : kv;
    io.out[i] = q;
    part += (double)own * (double)q;
  } else if (MODE == kModeChebFirst) {
    const T dd = fx ? T(0) : (T)io.coef[0] * io.dinv[i] * (io.b[i] - kv);
    io.d[i] = dd;
    io.out[i] = own + dd;
  } else if (MODE == kModeChebStep) {
    const T dd = fx ? T(0)
                    : (T)io.coef[2 * io.step] * io.d[i] + (T)io.coef[2 * io.step + 1] * io.dinv[i] * (io.b[i] - kv);
    io.d[i] = dd;
    io.out[i] = own + dd;
  } else {  // kModeDinvApply
    io.out[i] = fx ? T(0) : io.dinv[i] * kv;
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

template <typename T>
struct StencilParams {
  Grid g;
  const T* A;
  const uint8_t* fix;
  OpIO<T> io;
};

template <typename T, int MODE>
__global__ void __launch_bounds__(256) stencil_apply_kernel(const __grid_constant__ StencilParams<T> p) {
  if (op_skip(p.io)) return;
  __shared__ double red[32];
  const Grid g = p.g;
  const int NX = g.nx + 1, NY = g.ny + 1, NZ = g.nz + 1;
  const long long nn = g.nnode();
  const T* __restrict__ A = p.A;
  const T* __restrict__ u = p.io.u;
  double part = 0.0;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn; n += (long long)gridDim.x * blockDim.x) {
    const int iy = (int)(n % NY);
    const long long r = n / NY;
    const int ix = (int)(r % NX), iz = (int)(r / NX);
    T kv[3] = {T(0), T(0), T(0)};
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
      for (int dx = -1; dx <= 1; ++dx)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy) {
          const int x = ix + dx, y = iy + dy, z = iz + dz;
          if (x < 0 || x >= NX || y < 0 || y >= NY || z < 0 || z >= NZ) continue;
          const long long m = g.nidx(x, y, z);
          const int fm = p.fix[m];
          const int jr = jrel_of(dx, dy, dz);
          T um[3];
#pragma unroll
          for (int d = 0; d < 3; ++d) um[d] = ((fm >> d) & 1) ? T(0) : __ldg(&u[3 * m + d]);
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int d = 0; d < 3; ++d) kv[c] = fma(__ldg(&A[(long long)stencil_k(jr, c, d) * nn + n]), um[d], kv[c]);
        }
    const int f = p.fix[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const bool fx = (f >> c) & 1;
      op_epilogue<T, MODE>(p.io, 3 * n + c, fx, kv[c], fx ? T(0) : u[3 * n + c], part);
    }
  }
  if (MODE == kModeCgQ) {
    part = block_sum(part, red);
    if (threadIdx.x == 0) p.io.partials[blockIdx.x] = part;
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

// b_c[I] = sum_i P[i,I] r_f[i], 0 on fixed coarse DOFs.
template <typename T>
__global__ void restrict_kernel(Grid gf, Grid gc, const T* __restrict__ rf, const uint8_t* __restrict__ fixc, T* bc,
                                const int* done) {
  if (done && *(volatile const int*)done) return;
  const int FX = gf.nx + 1, FY = gf.ny + 1, FZ = gf.nz + 1;
  const int CX = gc.nx + 1, CY = gc.ny + 1;
  const long long nn = gc.nnode();
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn; n += (long long)gridDim.x * blockDim.x) {
    const int Iy = (int)(n % CY);
    const long long r = n / CY;
    const int Ix = (int)(r % CX), Iz = (int)(r / CX);
    T s[3] = {T(0), T(0), T(0)};
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
      for (int dx = -1; dx <= 1; ++dx)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy) {
          const int x = 2 * Ix + dx, y = 2 * Iy + dy, z = 2 * Iz + dz;
          if (x < 0 || x >= FX || y < 0 || y >= FY || z < 0 || z >= FZ) continue;
          const T w = T((dx ? 0.5 : 1.0) * (dy ? 0.5 : 1.0) * (dz ? 0.5 : 1.0));
          const long long m = gf.nidx(x, y, z);
#pragma unroll
          for (int c = 0; c < 3; ++c) s[c] = fma(w, rf[3 * m + c], s[c]);
        }
    const int f = fixc[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) bc[3 * n + c] = ((f >> c) & 1) ? T(0) : s[c];
  }
}

// x_f[i] += sum_I P[i,I] x_c[I] on free fine DOFs.
template <typename T>
__global__ void prolong_add_kernel(Grid gf, Grid gc, const T* __restrict__ xc, const uint8_t* __restrict__ fixf,
                                   T* xf, const int* done) {
  if (done && *(volatile const int*)done) return;
  const int FX = gf.nx + 1, FY = gf.ny + 1;
  const long long nn = gf.nnode();
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn; n += (long long)gridDim.x * blockDim.x) {
    const int iy = (int)(n % FY);
    const long long r = n / FY;
    const int ix = (int)(r % FX), iz = (int)(r / FX);
    T s[3] = {T(0), T(0), T(0)};
    const int nxp = (ix & 1) ? 2 : 1, nyp = (iy & 1) ? 2 : 1, nzp = (iz & 1) ? 2 : 1;
    const T wx = (ix & 1) ? T(0.5) : T(1), wy = (iy & 1) ? T(0.5) : T(1), wz = (iz & 1) ? T(0.5) : T(1);
    for (int a = 0; a < nzp; ++a)
      for (int b = 0; b < nxp; ++b)
        for (int c2 = 0; c2 < nyp; ++c2) {
          const int Ix = (ix >> 1) + b, Iy = (iy >> 1) + c2, Iz = (iz >> 1) + a;
          const long long m = gc.nidx(Ix, Iy, Iz);
          const T w = wx * wy * wz;
#pragma unroll
          for (int c = 0; c < 3; ++c) s[c] = fma(w, xc[3 * m + c], s[c]);
        }
    const int f = fixf[n];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      if (!((f >> c) & 1)) xf[3 * n + c] += s[c];
  }
}

}  // namespace tp3d
