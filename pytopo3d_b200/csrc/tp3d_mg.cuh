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

#include "tp3d_coarse_nm.cuh"
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

// The value of the apply layouts for entry (jx, jy, d) of the rows this thread
// built (node n, row component c, z-plane iz + dzr): zero on fixed rows /
// columns and for neighbours past the grid.
__device__ __forceinline__ double masked_row_entry(const Grid& g, const uint8_t* __restrict__ fix, bool fixed_row,
                                                   int ix, int iy, int z, int jx, int jy, int d,
                                                   const double (&acc)[9][3]) {
  const int NX = g.nx + 1, NY = g.ny + 1, NZ = g.nz + 1;
  const int x = ix + jx, y = iy + jy;
  const bool in = x >= 0 && x < NX && y >= 0 && y < NY && z >= 0 && z < NZ;
  const int fm = in ? fix[g.nidx(x, y, z)] : 7;
  return (fixed_row || ((fm >> d) & 1)) ? 0.0 : acc[(jx + 1) * 3 + (jy + 1)][d];
}

// The rows this thread built (node n, row component c, z-offset dzr), also
// in the apply layout of stencil_pack_kernel.
template <typename TP>
__device__ __forceinline__ void store_packed_rows(const Grid& g, const uint8_t* __restrict__ fix, long long n, int ix,
                                                  int iy, int iz, int c, int dzr, const double (&acc)[9][3],
                                                  TP* P) {
  const long long ndof = 3 * g.nnode();
  const bool fi = (fix[n] >> c) & 1;
#pragma unroll
  for (int jx = -1; jx <= 1; ++jx)
#pragma unroll
    for (int jy = -1; jy <= 1; ++jy) {
      const int jr = jrel_of(jx, jy, dzr);
#pragma unroll
      for (int d = 0; d < 3; ++d)
        P[(long long)(jr * 3 + d) * ndof + 3 * n + c] =
            (TP)masked_row_entry(g, fix, fi, ix, iy, iz + dzr, jx, jy, d, acc);
    }
}

// Node-major bf16 rows (nm3_apply_kernel's layout) of a builder block's 32
// nodes n0 .. n0 + 31: every warp of the block (row component c, z-offset dzr)
// puts its masked entries into a shared copy of the 32 rows (pad entries
// zero), then the block writes the rows, which are contiguous in N, with
// 16-byte stores.  Every thread of the block calls it.
__device__ __forceinline__ void write_node_major_rows(const Grid& g, const uint8_t* __restrict__ fix, long long n0,
                                                      bool live, int lane, int ix, int iy, int iz, int c, int dzr,
                                                      const double (&acc)[9][3], __nv_bfloat16* N) {
  __shared__ __align__(16) __nv_bfloat16 stage[32 * kNM3Row];
  uint4* st4 = reinterpret_cast<uint4*>(stage);
  constexpr int kChunksPerNode = kNM3Row * 2 / 16;  // 33
  for (int i = threadIdx.x; i < 32 * kChunksPerNode; i += blockDim.x) st4[i] = make_uint4(0u, 0u, 0u, 0u);
  __syncthreads();
  if (live) {
    const bool fi = (fix[n0 + lane] >> c) & 1;
#pragma unroll
    for (int jx = -1; jx <= 1; ++jx)
#pragma unroll
      for (int jy = -1; jy <= 1; ++jy)
#pragma unroll
        for (int d = 0; d < 3; ++d)
          stage[nm3_index(lane, dzr + 1, jx + 1, jy + 1, c, d)] =
              __double2bfloat16(masked_row_entry(g, fix, fi, ix, iy, iz + dzr, jx, jy, d, acc));
  }
  __syncthreads();
  const long long nvalid = min(32LL, g.nnode() - n0);
  uint4* dst = reinterpret_cast<uint4*>(N + n0 * kNM3Row);
  for (int i = threadIdx.x; i < nvalid * kChunksPerNode; i += blockDim.x) dst[i] = st4[i];
}

// With P / N given, also writes the apply layouts (see store_packed_rows).
template <typename TP>
__global__ void __launch_bounds__(kBuildThreads) build_level1_kernel(Grid gf, Grid gc, const double* __restrict__ E,
                                                                     const double* __restrict__ KE1, double* A,
                                                                     const uint8_t* __restrict__ fixc, TP* P,
                                                                     TP* N) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = w / 3, dzr = w % 3 - 1;
  const long long nn = gc.nnode();
  const long long n0 = (long long)blockIdx.x * 32, n = n0 + lane;
  const bool live = n < nn;  // no early return: the node-major writer takes block barriers
  const int CY = gc.ny + 1, CX = gc.nx + 1;
  const int Iy = (int)(n % CY);
  const long long r = n / CY;
  const int Ix = (int)(r % CX), Iz = (int)(r / CX);
  double acc[9][3];
#pragma unroll
  for (int i = 0; i < 9; ++i)
#pragma unroll
    for (int d = 0; d < 3; ++d) acc[i][d] = 0.0;
  if (live) {
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
    if (P) store_packed_rows<TP>(gc, fixc, n, Ix, Iy, Iz, c, dzr, acc, P);
  }
  if constexpr (sizeof(TP) == 2)
    if (N) write_node_major_rows(gc, fixc, n0, live, lane, Ix, Iy, Iz, c, dzr, acc, N);
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

// ---- element-wise Galerkin products for levels >= 2 ----
// With nested trilinear spaces every fine element maps into exactly one
// coarse element of each level, so the level-L operator is the assembly of
// level-L element matrices: for level 2, K2[C] = sum_f E_f Q_f^T KE Q_f over
// the 4x4x4 fine elements f of C (tables KE2[f] = Q_f^T KE Q_f, f = fx + 4 fy +
// 16 fz); for deeper levels K_L[C] = sum_s P_s^T K_{L-1}[C_s] P_s over the 8
// sub-elements, P_s the trilinear interpolation to sub-element s.  Element
// matrices are stored [element][24][24], element index as Grid::eidx.

// Level-2 element matrices from the fine moduli; one block (576 threads, one
// matrix entry each) per level-2 element.
__global__ void __launch_bounds__(576) elem2_from_fine_kernel(Grid gf, Grid g2, const double* __restrict__ E,
                                                              const double* __restrict__ KE2, double* K2) {
  __shared__ double sE[64];
  const int C = blockIdx.x;
  const int cy = C % g2.ny, r = C / g2.ny;
  const int cx = r % g2.nx, cz = r / g2.nx;
  if (threadIdx.x < 64) {
    const int x = 4 * cx + (threadIdx.x & 3), y = 4 * cy + ((threadIdx.x >> 2) & 3), z = 4 * cz + (threadIdx.x >> 4);
    sE[threadIdx.x] = (x < gf.nx && y < gf.ny && z < gf.nz) ? __ldg(&E[gf.eidx(x, y, z)]) : 0.0;
  }
  __syncthreads();
  double acc = 0.0;
#pragma unroll 8
  for (int f = 0; f < 64; ++f) acc = fma(sE[f], __ldg(&KE2[f * 576 + threadIdx.x]), acc);
  K2[(size_t)C * 576 + threadIdx.x] = acc;
}

// Trilinear weight of coarse corner b at corner a of sub-element s.
__device__ __forceinline__ double sub_weight(int s, int a, int b) {
  const int px = corner_ox(s) + corner_ox(a) - 2 * corner_ox(b);
  const int py = corner_oy(s) + corner_oy(a) - 2 * corner_oy(b);
  const int pz = corner_oz(s) + corner_oz(a) - 2 * corner_oz(b);
  return (px == 0 ? 1.0 : (px == 1 || px == -1 ? 0.5 : 0.0)) * (py == 0 ? 1.0 : (py == 1 || py == -1 ? 0.5 : 0.0)) *
         (pz == 0 ? 1.0 : (pz == 1 || pz == -1 ? 0.5 : 0.0));
}

// Level-L element matrices from level L-1; one block (576 threads) per
// level-L element.  Per sub-element: T = K_s (W_s x I3), then out += (W_s x I3)^T T.
__global__ void __launch_bounds__(576) elem_coarsen_kernel(Grid gf, Grid gc, const double* __restrict__ Kf,
                                                           double* Kc) {
  __shared__ double sK[576], sT[576], sW[64];
  const int C = blockIdx.x;
  const int cy = C % gc.ny, r = C / gc.ny;
  const int cx = r % gc.nx, cz = r / gc.nx;
  const int t = threadIdx.x;
  const int row = t / 24, col = t - 24 * row;  // output entry (row, col)
  const int ra = row / 3, rc = row - 3 * ra, cb = col / 3, cd = col - 3 * cb;
  double acc = 0.0;
  for (int s = 0; s < 8; ++s) {
    const int fx = 2 * cx + corner_ox(s), fy = 2 * cy + corner_oy(s), fz = 2 * cz + corner_oz(s);
    if (fx >= gf.nx || fy >= gf.ny || fz >= gf.nz) continue;  // uniform over the block
    __syncthreads();
    sK[t] = __ldg(&Kf[(size_t)gf.eidx(fx, fy, fz) * 576 + t]);
    if (t < 64) sW[t] = sub_weight(s, t >> 3, t & 7);  // sW[a * 8 + b]
    __syncthreads();
    // T[3a+c][3B+d] = sum_b' K_s[3a+c][3b'+d] W[b'][B]   (this thread: a = ra, c = rc, B = cb, d = cd)
    double tv = 0.0;
#pragma unroll
    for (int b = 0; b < 8; ++b) tv = fma(sK[row * 24 + 3 * b + cd], sW[b * 8 + cb], tv);
    sT[t] = tv;
    __syncthreads();
    // out[3A+c][3B+d] += sum_a W[a][A] T[3a+c][3B+d]   (A = ra)
#pragma unroll
    for (int a = 0; a < 8; ++a) acc = fma(sW[a * 8 + ra], sT[(3 * a + rc) * 24 + col], acc);
  }
  Kc[(size_t)C * 576 + t] = acc;
}

// Stencil (27-point 3x3 blocks, layout of stencil_k) of level g assembled
// from its element matrices.  Threads as in the other builders: a warp per 32
// nodes for one (row component c, z-offset dzr).
template <typename TP>
__global__ void __launch_bounds__(kBuildThreads) stencil_from_elems_kernel(Grid g, const double* __restrict__ Ke,
                                                                           double* A, const uint8_t* __restrict__ fix,
                                                                           TP* P, TP* N) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = w / 3, dzr = w % 3 - 1;
  const long long nn = g.nnode();
  const long long n0 = (long long)blockIdx.x * 32, n = n0 + lane;
  const bool live = n < nn;  // no early return: the node-major writer takes block barriers
  const int NY = g.ny + 1, NX = g.nx + 1;
  const int iy = (int)(n % NY);
  const long long r = n / NY;
  const int ix = (int)(r % NX), iz = (int)(r / NX);
  double acc[9][3];
#pragma unroll
  for (int i = 0; i < 9; ++i)
#pragma unroll
    for (int d = 0; d < 3; ++d) acc[i][d] = 0.0;
  if (live) {
#pragma unroll
    for (int ez = -1; ez <= 0; ++ez) {
      const int zc = iz + ez;
      if (zc < 0 || zc >= g.nz) continue;
#pragma unroll
      for (int ex = -1; ex <= 0; ++ex) {
        const int xc = ix + ex;
        if (xc < 0 || xc >= g.nx) continue;
#pragma unroll
        for (int ey = -1; ey <= 0; ++ey) {
          const int yc = iy + ey;
          if (yc < 0 || yc >= g.ny) continue;
          const int a = corner_index(-ex, -ey, -ez);
          const double* rowp = Ke + (size_t)g.eidx(xc, yc, zc) * 576 + (3 * a + c) * 24;
#pragma unroll
          for (int b = 0; b < 8; ++b) {
            if (ez + corner_oz(b) != dzr) continue;
            const int jx = ex + corner_ox(b), jy = ey + corner_oy(b);
            const int slot = (jx + 1) * 3 + (jy + 1);
#pragma unroll
            for (int d = 0; d < 3; ++d) acc[slot][d] += __ldg(&rowp[3 * b + d]);
          }
        }
      }
    }
#pragma unroll
    for (int jx = -1; jx <= 1; ++jx)
#pragma unroll
      for (int jy = -1; jy <= 1; ++jy)
#pragma unroll
        for (int d = 0; d < 3; ++d)
          A[(long long)stencil_k(jrel_of(jx, jy, dzr), c, d) * nn + n] = acc[(jx + 1) * 3 + (jy + 1)][d];
    if (P) store_packed_rows<TP>(g, fix, n, ix, iy, iz, c, dzr, acc, P);
  }
  if constexpr (sizeof(TP) == 2)
    if (N) write_node_major_rows(g, fix, n0, live, lane, ix, iy, iz, c, dzr, acc, N);
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

// Dense inverse of the coarsest operator, entirely on the device (no host
// round trip per set-up).  Gauss-Jordan without pivoting (SPD pivots stay
// positive in exact arithmetic); if a pivot is not positive, the elimination
// restarts from D with the diagonal raised by 1e-12, 1e-9, then 1e-6 times its
// mean magnitude; if all of those fail too, Inv is the inverse diagonal of D.
// *status = the number of shifted attempts used (0..3), or kGjFallback.
constexpr int kGjAttempts = 4;
constexpr int kGjFallback = 4;

__device__ __forceinline__ double gj_shift(const double* __restrict__ D, int n, int attempt) {
  if (attempt == 0) return 0.0;
  double m = 0.0;
  for (int i = 0; i < n; ++i) m += fabs(D[(size_t)i * n + i]);
  m = fmax(m / n, 1e-300);
  return (attempt == 1 ? 1e-12 : (attempt == 2 ? 1e-9 : 1e-6)) * m;
}

__device__ __forceinline__ void gj_diag_fallback(const double* __restrict__ D, int n, double* Inv) {
  for (long long t = threadIdx.x; t < (long long)n * n; t += blockDim.x) {
    const int i = (int)(t / n), j = (int)(t % n);
    const double d = D[(size_t)i * n + i];
    Inv[t] = (i == j && d > 0.0) ? 1.0 / d : 0.0;
  }
}

// One block.  When `in_smem`, the working matrix lives in dynamic shared
// memory (n <= 160), else in Inv.  Each pivot step copies row k and column k
// aside, then updates every entry in one pass over the matrix, a warp per row
// (two barriers per step).
__global__ void __launch_bounds__(1024) dense_gj_inverse_kernel(int n, const double* __restrict__ D, double* Inv,
                                                                int in_smem, int* status) {
  extern __shared__ double sA[];  // [n * n if in_smem] [row k: n] [column k: n]
  const long long nn = (long long)n * n;
  double* A = in_smem ? sA : Inv;
  double* rowk = sA + (in_smem ? nn : 0);
  double* colk = rowk + n;
  __shared__ int bad;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  int attempt = 0;
  for (; attempt < kGjAttempts; ++attempt) {
    const double shift = gj_shift(D, n, attempt);
    for (long long t = threadIdx.x; t < nn; t += blockDim.x) A[t] = D[t] + ((t % (n + 1)) == 0 ? shift : 0.0);
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    for (int k = 0; k < n; ++k) {
      for (int t = threadIdx.x; t < n; t += blockDim.x) {
        rowk[t] = A[(size_t)k * n + t];
        colk[t] = A[(size_t)t * n + k];
      }
      __syncthreads();
      const double p = rowk[k];
      if (threadIdx.x == 0 && !(p > 0.0) && !bad) bad = k + 1;
      const double pk = 1.0 / (p > 0.0 ? p : 1e-300);
      // a warp per row, lanes along the row
      for (int i = warp; i < n; i += nwarps) {
        double* Ai = A + (size_t)i * n;
        const double f = colk[i] * pk;
        if (i == k) {
          for (int j = lane; j < n; j += 32) Ai[j] = (j == k) ? pk : rowk[j] * pk;
        } else {
          for (int j = lane; j < n; j += 32) Ai[j] = (j == k) ? -f : Ai[j] - f * rowk[j];
        }
      }
      __syncthreads();
    }
    const int failed = bad;
    __syncthreads();  // every thread has read `bad` before thread 0 resets it
    if (!failed) break;
  }
  if (attempt == kGjAttempts) {
    gj_diag_fallback(D, n, Inv);
  } else if (in_smem) {
    for (long long t = threadIdx.x; t < nn; t += blockDim.x) Inv[t] = A[t];
  }
  if (threadIdx.x == 0) *status = attempt == kGjAttempts ? kGjFallback : attempt;
}

// Gauss-Jordan inverse of a small SPD matrix (n <= 160) held in registers: one
// block of 16 x 32 threads, thread (w, l) owns the 10 x 5 entries (w + 16 r,
// l + 32 c).  Per pivot step the owners of row k and column k publish them in
// shared memory (double-buffered, one barrier per step) and every thread
// updates its entries in registers.  Same arithmetic, attempts and status as
// dense_gj_inverse_kernel.
constexpr int kGjRegMaxN = 160;

__global__ void __launch_bounds__(512, 1) dense_gj_inverse_reg_kernel(int n, const double* __restrict__ D, double* Inv,
                                                                      int* status) {
  constexpr int R = 10, C = 5;
  __shared__ double rowk[2][kGjRegMaxN], colk[2][kGjRegMaxN];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  double a[R][C];
  int attempt = 0;
  for (; attempt < kGjAttempts; ++attempt) {
    const double shift = gj_shift(D, n, attempt);
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const int i = w + 16 * r, j = l + 32 * c;
        a[r][c] = (i < n && j < n) ? D[(size_t)i * n + j] + (i == j ? shift : 0.0) : 0.0;
      }
    int bad = 0;  // the same in every thread: each reads the pivot from shared memory
    for (int k = 0; k < n; ++k) {
      const int buf = k & 1;
      // owners of row k (warp k % 16, r = k / 16) and of column k (lane k % 32,
      // c = k / 32) publish them; selects keep every index compile-time
      if (w == (k & 15)) {
        const int kr = k >> 4;
#pragma unroll
        for (int c = 0; c < C; ++c) {
          double v = 0.0;
#pragma unroll
          for (int r = 0; r < R; ++r) v = (r == kr) ? a[r][c] : v;
          rowk[buf][l + 32 * c] = v;
        }
      }
      if (l == (k & 31)) {
        const int kc = k >> 5;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          double v = 0.0;
#pragma unroll
          for (int c = 0; c < C; ++c) v = (c == kc) ? a[r][c] : v;
          colk[buf][w + 16 * r] = v;
        }
      }
      __syncthreads();
      const double p = rowk[buf][k];
      if (!(p > 0.0) && !bad) bad = k + 1;
      const double pk = 1.0 / (p > 0.0 ? p : 1e-300);
      double g[C];
#pragma unroll
      for (int c = 0; c < C; ++c) g[c] = rowk[buf][l + 32 * c];
      // every entry: a_ij -= (a_ik / a_kk) a_kj (one FMA each); row k and
      // column k are then overwritten by their owners
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const double f = colk[buf][w + 16 * r] * pk;
#pragma unroll
        for (int c = 0; c < C; ++c) a[r][c] = a[r][c] - f * g[c];
      }
      if (w == (k & 15)) {  // row k: a_kj / a_kk
        const int kr = k >> 4;
#pragma unroll
        for (int r = 0; r < R; ++r)
          if (r == kr) {
#pragma unroll
            for (int c = 0; c < C; ++c) a[r][c] = g[c] * pk;
          }
      }
      if (l == (k & 31)) {  // column k: -a_ik / a_kk, and 1 / a_kk on the diagonal
        const int kc = k >> 5;
#pragma unroll
        for (int c = 0; c < C; ++c)
          if (c == kc) {
#pragma unroll
            for (int r = 0; r < R; ++r) a[r][c] = (w + 16 * r == k) ? pk : -(colk[buf][w + 16 * r] * pk);
          }
      }
    }
    __syncthreads();  // the last step's buffers are read before the next attempt writes them
    if (!bad) break;
  }
  if (attempt == kGjAttempts) {
    gj_diag_fallback(D, n, Inv);
  } else {
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const int i = w + 16 * r, j = l + 32 * c;
        if (i < n && j < n) Inv[(size_t)i * n + j] = a[r][c];
      }
  }
  if (threadIdx.x == 0) *status = attempt == kGjAttempts ? kGjFallback : attempt;
}

template <typename T>
__global__ void dense_matvec_kernel(int n, const T* __restrict__ Inv, const T* __restrict__ b, T* x, const int* done) {
  pdl_entry();
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
