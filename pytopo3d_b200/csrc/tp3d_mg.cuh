// Multigrid hierarchy construction: Galerkin coarse operators, coarse masks,
// coarsest dense inverse.
//
// Level 1 comes straight from the fine moduli: the coarse element matrix of a
// 2x2x2 block of fine elements is sum_s E_s KE1[s] with KE1[s] = P_s^T KE P_s
// (P_s: trilinear interpolation from the coarse element's corners to fine
// sub-element s), which equals P^T K P exactly for nested trilinear spaces.
// Deeper levels use the stencil form of P^T A P.  Threads are laid out so
// that one warp handles 32 coarse nodes for one (row component c, z-offset
// dzr) pair: every coefficient-table load is warp-uniform (a broadcast) and a
// thread carries 27 accumulators.
#pragma once

#include "tp3d_hex.cuh"

namespace tp3d {

constexpr int kBuildThreads = 9 * 32;

__host__ __device__ constexpr double hat(int d) { return d == 0 ? 1.0 : ((d == 1 || d == -1) ? 0.5 : 0.0); }

// ---- level 1 from fine element moduli ----
template <int DZR>
__device__ __forceinline__ void build_l1_rows(const Grid& gf, const Grid& gc, const double* __restrict__ E,
                                              const double* __restrict__ KE1, int Ix, int Iy, int Iz, int c,
                                              double acc[9][3]) {
#pragma unroll
  for (int ez = -1; ez <= 0; ++ez) {
    const int oz_need = DZR - ez;
    if (oz_need < 0 || oz_need > 1) continue;
    const int ecz = Iz + ez;
    if (ecz < 0 || ecz >= gc.nz) continue;
#pragma unroll
    for (int ex = -1; ex <= 0; ++ex) {
      const int ecx = Ix + ex;
      if (ecx < 0 || ecx >= gc.nx) continue;
#pragma unroll
      for (int ey = -1; ey <= 0; ++ey) {
        const int ecy = Iy + ey;
        if (ecy < 0 || ecy >= gc.ny) continue;
        const int a = corner_index(-ex, -ey, -ez);
#pragma unroll
        for (int s = 0; s < 8; ++s) {
          const int fx = 2 * ecx + corner_ox(s), fy = 2 * ecy + corner_oy(s), fz = 2 * ecz + corner_oz(s);
          if (fx >= gf.nx || fy >= gf.ny || fz >= gf.nz) continue;
          const double Es = __ldg(&E[gf.eidx(fx, fy, fz)]);
          const double* row = KE1 + (size_t)s * 576 + (3 * a + c) * 24;
#pragma unroll
          for (int b = 0; b < 8; ++b) {
            if (corner_oz(b) != oz_need) continue;
            const int jx = ex + corner_ox(b), jy = ey + corner_oy(b);
            const int slot = (jx + 1) * 3 + (jy + 1);
#pragma unroll
            for (int d = 0; d < 3; ++d) acc[slot][d] = fma(Es, __ldg(&row[3 * b + d]), acc[slot][d]);
          }
        }
      }
    }
  }
}

__global__ void __launch_bounds__(kBuildThreads) build_level1_kernel(Grid gf, Grid gc, const double* __restrict__ E,
                                                                     const double* __restrict__ KE1, double* A) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = w / 3, dzr = w % 3 - 1;
  const long long nn = gc.nnode();
  const long long n = (long long)blockIdx.x * 32 + lane;
  if (n >= nn) return;
  const int CY = gc.ny + 1, CX = gc.nx + 1;
  const int Iy = (int)(n % CY);
  const long long r = n / CY;
  const int Ix = (int)(r % CX), Iz = (int)(r / CX);
  double acc[9][3];
#pragma unroll
  for (int i = 0; i < 9; ++i)
#pragma unroll
    for (int d = 0; d < 3; ++d) acc[i][d] = 0.0;
  if (dzr == -1) build_l1_rows<-1>(gf, gc, E, KE1, Ix, Iy, Iz, c, acc);
  else if (dzr == 0) build_l1_rows<0>(gf, gc, E, KE1, Ix, Iy, Iz, c, acc);
  else build_l1_rows<1>(gf, gc, E, KE1, Ix, Iy, Iz, c, acc);
#pragma unroll
  for (int jx = -1; jx <= 1; ++jx)
#pragma unroll
    for (int jy = -1; jy <= 1; ++jy)
#pragma unroll
      for (int d = 0; d < 3; ++d)
        A[(long long)stencil_k(jrel_of(jx, jy, dzr), c, d) * nn + n] = acc[(jx + 1) * 3 + (jy + 1)][d];
}

// ---- stencil Galerkin product A_c = P^T A_f P ----
template <int DZR>
__device__ __forceinline__ void rap_rows(const Grid& gf, const double* __restrict__ Af, int Ix, int Iy, int Iz,
                                         int c, double acc[9][3]) {
  const int FX = gf.nx + 1, FY = gf.ny + 1, FZ = gf.nz + 1;
  const long long nnf = gf.nnode();
#pragma unroll
  for (int diz = -1; diz <= 1; ++diz) {
    const int iz = 2 * Iz + diz;
    if (iz < 0 || iz >= FZ) continue;
#pragma unroll
    for (int djz = -1; djz <= 1; ++djz) {
      const int jjz = diz + djz;  // fine offset of j from 2I along z, in [-2, 2]
      // coarse offsets Jz with |jjz - 2 Jz| <= 1 must include DZR
      const double wz = hat(jjz - 2 * DZR);
      if (wz == 0.0) continue;
      if (iz + djz < 0 || iz + djz >= FZ) continue;
#pragma unroll
      for (int dix = -1; dix <= 1; ++dix) {
        const int ix = 2 * Ix + dix;
        if (ix < 0 || ix >= FX) continue;
#pragma unroll
        for (int diy = -1; diy <= 1; ++diy) {
          const int iy = 2 * Iy + diy;
          if (iy < 0 || iy >= FY) continue;
          const long long i = gf.nidx(ix, iy, iz);
          const double wi = hat(dix) * hat(diy) * hat(diz);
#pragma unroll
          for (int djx = -1; djx <= 1; ++djx) {
            if (ix + djx < 0 || ix + djx >= FX) continue;
#pragma unroll
            for (int djy = -1; djy <= 1; ++djy) {
              if (iy + djy < 0 || iy + djy >= FY) continue;
              const int jr = jrel_of(djx, djy, djz);
              double a3[3];
#pragma unroll
              for (int d = 0; d < 3; ++d) a3[d] = wi * wz * __ldg(&Af[(long long)stencil_k(jr, c, d) * nnf + i]);
              const int jjx = dix + djx, jjy = diy + djy;
#pragma unroll
              for (int Jx = -1; Jx <= 1; ++Jx) {
                const double wx = hat(jjx - 2 * Jx);
                if (wx == 0.0) continue;
#pragma unroll
                for (int Jy = -1; Jy <= 1; ++Jy) {
                  const double wy = hat(jjy - 2 * Jy);
                  if (wy == 0.0) continue;
                  const int slot = (Jx + 1) * 3 + (Jy + 1);
#pragma unroll
                  for (int d = 0; d < 3; ++d) acc[slot][d] = fma(wx * wy, a3[d], acc[slot][d]);
                }
              }
            }
          }
        }
      }
    }
  }
}

__global__ void __launch_bounds__(kBuildThreads) rap_kernel(Grid gf, Grid gc, const double* __restrict__ Af,
                                                            double* Ac) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = w / 3, dzr = w % 3 - 1;
  const long long nn = gc.nnode();
  const long long n = (long long)blockIdx.x * 32 + lane;
  if (n >= nn) return;
  const int CY = gc.ny + 1, CX = gc.nx + 1;
  const int Iy = (int)(n % CY);
  const long long r = n / CY;
  const int Ix = (int)(r % CX), Iz = (int)(r / CX);
  double acc[9][3];
#pragma unroll
  for (int i = 0; i < 9; ++i)
#pragma unroll
    for (int d = 0; d < 3; ++d) acc[i][d] = 0.0;
  if (dzr == -1) rap_rows<-1>(gf, Af, Ix, Iy, Iz, c, acc);
  else if (dzr == 0) rap_rows<0>(gf, Af, Ix, Iy, Iz, c, acc);
  else rap_rows<1>(gf, Af, Ix, Iy, Iz, c, acc);
#pragma unroll
  for (int jx = -1; jx <= 1; ++jx)
#pragma unroll
    for (int jy = -1; jy <= 1; ++jy)
#pragma unroll
      for (int d = 0; d < 3; ++d)
        Ac[(long long)stencil_k(jrel_of(jx, jy, dzr), c, d) * nn + n] = acc[(jx + 1) * 3 + (jy + 1)][d];
}

// ---- coarse fixed-DOF masks ----
// Injection: a coarse node takes the mask of the fine node it sits on (the
// last fine node when it lies past an odd fine edge).  Dilation (fallback used
// when injection fixes nothing): OR over the fine nodes within one fine step.
__global__ void coarse_mask_kernel(Grid gf, Grid gc, const uint8_t* __restrict__ ff, uint8_t* fc, int dilate,
                                   unsigned int* count) {
  const int FX = gf.nx + 1, FY = gf.ny + 1, FZ = gf.nz + 1;
  const int CX = gc.nx + 1, CY = gc.ny + 1;
  const long long nn = gc.nnode();
  unsigned int local = 0;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn; n += (long long)gridDim.x * blockDim.x) {
    const int Iy = (int)(n % CY);
    const long long r = n / CY;
    const int Ix = (int)(r % CX), Iz = (int)(r / CX);
    int m = 0;
    if (!dilate) {
      m = ff[gf.nidx(min(2 * Ix, FX - 1), min(2 * Iy, FY - 1), min(2 * Iz, FZ - 1))];
    } else {
      for (int dz = -1; dz <= 1; ++dz)
        for (int dx = -1; dx <= 1; ++dx)
          for (int dy = -1; dy <= 1; ++dy) {
            const int x = 2 * Ix + dx, y = 2 * Iy + dy, z = 2 * Iz + dz;
            if (x < 0 || x >= FX || y < 0 || y >= FY || z < 0 || z >= FZ) continue;
            m |= ff[gf.nidx(x, y, z)];
          }
    }
    fc[n] = (uint8_t)m;
    local += (m != 0);
  }
  if (local) atomicAdd(count, local);
}

// per-DOF uint8 mask -> per-node bits
__global__ void pack_mask_kernel(long long nn, const uint8_t* __restrict__ dofmask, uint8_t* nodebits,
                                 unsigned int* count) {
  unsigned int local = 0;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn; n += (long long)gridDim.x * blockDim.x) {
    const int m = (dofmask[3 * n] ? 1 : 0) | (dofmask[3 * n + 1] ? 2 : 0) | (dofmask[3 * n + 2] ? 4 : 0);
    nodebits[n] = (uint8_t)m;
    local += (m != 0);
  }
  if (local) atomicAdd(count, local);
}

// ---- coarsest level: dense masked operator, Cholesky, explicit inverse ----
__global__ void dense_from_stencil_kernel(Grid g, const double* __restrict__ A, const uint8_t* __restrict__ fix,
                                          double* D) {
  const int NX = g.nx + 1, NY = g.ny + 1, NZ = g.nz + 1;
  const long long nn = g.nnode();
  const long long n3 = 3 * nn;
  // D is zeroed by the caller
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nn; n += (long long)gridDim.x * blockDim.x) {
    const int iy = (int)(n % NY);
    const long long r = n / NY;
    const int ix = (int)(r % NX), iz = (int)(r / NX);
    const int fi = fix[n];
    for (int dz = -1; dz <= 1; ++dz)
      for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy) {
          const int x = ix + dx, y = iy + dy, z = iz + dz;
          if (x < 0 || x >= NX || y < 0 || y >= NY || z < 0 || z >= NZ) continue;
          const long long m = g.nidx(x, y, z);
          const int fm = fix[m];
          for (int c = 0; c < 3; ++c)
            for (int d = 0; d < 3; ++d) {
              double v = A[(long long)stencil_k(jrel_of(dx, dy, dz), c, d) * nn + n];
              if (((fi >> c) & 1) || ((fm >> d) & 1)) v = 0.0;
              D[(3 * n + c) * n3 + 3 * m + d] = v;
            }
        }
    for (int c = 0; c < 3; ++c)
      if ((fi >> c) & 1) D[(3 * n + c) * n3 + 3 * n + c] = 1.0;
  }
}

// In-place Gauss-Jordan inverse of the SPD matrix D (n x n, row-major) into
// Inv, one block, no pivoting (SPD pivots stay positive in exact arithmetic).
// When `in_smem`, the matrix lives in dynamic shared memory (n <= 160).
// *status = 0 ok, k+1 if pivot k was not positive.
__global__ void __launch_bounds__(1024) dense_gj_inverse_kernel(int n, const double* __restrict__ D, double* Inv,
                                                                int in_smem, int* status) {
  extern __shared__ double sA[];
  double* A = in_smem ? sA : Inv;
  __shared__ int bad;
  __shared__ double piv;
  const long long nn = (long long)n * n;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  for (long long t = threadIdx.x; t < nn; t += blockDim.x) A[t] = D[t];
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    if (threadIdx.x == 0) {
      const double p = A[(size_t)k * n + k];
      if (!(p > 0.0) && !bad) bad = k + 1;
      piv = 1.0 / (p > 0.0 ? p : 1e-300);
    }
    __syncthreads();
    const double pk = piv;
    // entries off row k and column k, from the old row/column: a warp per row
    for (int i = warp; i < n; i += nwarps) {
      if (i == k) continue;
      double* Ai = A + (size_t)i * n;
      const double f = Ai[k] * pk;
      const double* Ak = A + (size_t)k * n;
      for (int j = lane; j < n; j += 32)
        if (j != k) Ai[j] -= f * Ak[j];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
      if (t != k) {
        A[(size_t)t * n + k] *= -pk;  // column k
        A[(size_t)k * n + t] *= pk;   // row k
      }
    }
    if (threadIdx.x == 0) A[(size_t)k * n + k] = pk;
    __syncthreads();
  }
  if (in_smem)
    for (long long t = threadIdx.x; t < nn; t += blockDim.x) Inv[t] = A[t];
  if (threadIdx.x == 0) *status = bad;
}

template <typename T>
__global__ void dense_matvec_kernel(int n, const T* __restrict__ Inv, const T* __restrict__ b, T* x, const int* done) {
  if (done && *(volatile const int*)done) return;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int i = warp; i < n; i += nwarps) {
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s += (double)Inv[(size_t)i * n + j] * (double)b[j];
    s = warp_sum(s);
    if (lane == 0) x[i] = (T)s;
  }
}

}  // namespace tp3d
