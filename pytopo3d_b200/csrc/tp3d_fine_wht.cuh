// Fine-level operator y = Z K(E) Z u + (I - Z) u in the Walsh-Hadamard basis
// of the element's corners.
//
// The 8 corners of a brick element form the group {0,1}^3 under the three axis
// reflections, and the element stiffness of an axis-aligned orthotropic
// material (lk_H8, pytopo3d/utils/stiffness.py:12-130) commutes with them.
// Transforming the corner values of each displacement component with the
// 8-point Walsh-Hadamard transform u_hat(s, i) = sum_a (-1)^(s.a) u(a, i)
// therefore splits KE into eight 3x3 blocks: for every character t in {0,1}^3
// the block couples u_hat(t ^ e_i, i) for i = 0, 1, 2 (e_i the bit of axis i),
//   y = W^T M u_hat,   M_t[i][j] = (W KE W^T)[(t^e_i, i), (t^e_j, j)] / 64.
// For t = e_k the member (s = 0, i = k) is the rigid translation along k, so
// its row and column vanish.  Per element this is 57 multiply-adds instead of
// the 576 of the dense KE u_e, and the transforms themselves are separable:
//  * per node plane, each thread forms the 2D transform P[sx + 2 sy][c] of its
//    element column's four corners in the plane (three neighbours read from
//    shared memory);
//  * the element between planes z and z+1 takes u_hat(s + 4 sz) =
//    P_z[s] + (-1)^sz P_{z+1}[s]; P of plane z+1 is kept for the next element;
//  * the inverse splits the same way: the top-face half of element z-1 is kept
//    in registers and added to the bottom-face half of element z before the
//    2D inverse hands three of the four corner contributions to the
//    neighbouring threads through shared memory.
// A block owns a (TX + 2) x (TY + 2) patch of nodes (one node per thread, a
// one-node halo on the low and high sides) and marches along z over ZC node
// planes; it writes the TX x TY interior.  Per node and plane about 190
// floating-point operations, 12 shared stores, 18 shared loads and two barriers.
#pragma once

#include <type_traits>

#include "tp3d_fine.cuh"

namespace tp3d {

template <typename T>
struct WhtBlocks {
  T m[8][3][3];  // M_t[i][j] as above (1/64 folded in)
};

template <typename T, class ESrc>
struct WhtParams {
  WhtBlocks<T> mb;
  Grid g;           // element grid
  int TX, TY, PY;   // interior tile (nodes written); PY = TY + 2 threads per patch row
  int ZC;           // node planes per block
  int tiles_y, tiles_x;
  const uint8_t* fix;
  ESrc esrc;
  OpIO<T> io;
};

template <typename T>
__host__ __device__ constexpr size_t wht_smem_bytes(int nthr) {
  return (size_t)12 * nthr * sizeof(T);
}

template <typename T, class ESrc, int MODE, int NTHR, int MINB>
__global__ void __launch_bounds__(NTHR, MINB) wht_apply_kernel(const __grid_constant__ WhtParams<T, ESrc> p) {
  pdl_entry();
  if (op_skip(p.io)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* su = reinterpret_cast<T*>(smem_raw);  // [3][NTHR] masked u of each thread's node
  T* sc = su + 3 * NTHR;                   // [9][NTHR] corner (1,0), (0,1), (1,1) contributions
  __shared__ double red[32];

  const int NX = p.g.nx + 1, NY = p.g.ny + 1, NZ = p.g.nz + 1;
  const int PY = p.PY;
  const int by = blockIdx.x % p.tiles_y, bx = blockIdx.x / p.tiles_y;
  const int x0 = bx * p.TX, y0 = by * p.TY;
  const int zb = blockIdx.y * p.ZC, ze = min(zb + p.ZC, NZ);
  const int t = threadIdx.x;
  const int ly = t % PY, lx = t / PY;
  const int gx = x0 - 1 + lx, gy = y0 - 1 + ly;
  const bool inpatch = lx < p.TX + 2;
  const bool node_in = inpatch && gx >= 0 && gx < NX && gy >= 0 && gy < NY;
  const bool elem_cols = inpatch && lx <= p.TX && ly <= p.TY;  // threads whose element column is needed
  const bool elem_in = elem_cols && gx >= 0 && gx < p.g.nx && gy >= 0 && gy < p.g.ny;
  const bool writer = node_in && lx >= 1 && lx <= p.TX && ly >= 1 && ly <= p.TY;
  const long long pstride = (long long)NX * NY;
  const long long sstride = (long long)p.g.nx * p.g.ny;
  const long long nbase = node_in ? gy + (long long)NY * gx : 0;
  const long long ebase = elem_in ? gy + (long long)p.g.ny * gx : 0;
  const T* __restrict__ u = p.io.u;
  const uint8_t* __restrict__ fix = p.fix;

  // masked u of this thread's node on plane zp (0 outside the grid)
  auto load_u = [&](int zp, T (&v)[3]) {
    if (node_in && zp >= 0 && zp < NZ) {
      const long long n = nbase + zp * pstride;
      const T a = u[3 * n], b = u[3 * n + 1], c = u[3 * n + 2];
      const int f = fix[n];
      v[0] = (f & 1) ? T(0) : a;
      v[1] = (f & 2) ? T(0) : b;
      v[2] = (f & 4) ? T(0) : c;
    } else {
      v[0] = v[1] = v[2] = T(0);
    }
  };
  auto load_E = [&](int zs) -> T {
    return (elem_in && zs >= 0 && zs < p.g.nz) ? (T)p.esrc(ebase + zs * sstride) : T(0);
  };
  // 2D transform of this element column's corners on one plane.  Stores this
  // node's values, waits, then reads the (x+1, y), (x, y+1), (x+1, y+1) nodes.
  // The caller guarantees that every thread has finished reading su since the
  // previous call.
  auto plane_wht = [&](const T (&v)[3], T (&P)[4][3]) {
#pragma unroll
    for (int c = 0; c < 3; ++c) su[c * NTHR + t] = v[c];
    __syncthreads();
    if (elem_cols) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const T u00 = v[c], u01 = su[c * NTHR + t + 1];
        const T u10 = su[c * NTHR + t + PY], u11 = su[c * NTHR + t + PY + 1];
        const T a0 = u00 + u01, a1 = u00 - u01, b0 = u10 + u11, b1 = u10 - u11;
        P[0][c] = a0 + b0;  // (sx, sy) = (0, 0)
        P[1][c] = a0 - b0;  // (1, 0)
        P[2][c] = a1 + b1;  // (0, 1)
        P[3][c] = a1 - b1;  // (1, 1)
      }
    } else {
#pragma unroll
      for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int c = 0; c < 3; ++c) P[s][c] = T(0);
    }
  };
  // Element between the planes holding Plo and Phi with modulus E: adds the
  // bottom-face half of its transformed product to R (when BOTTOM) and writes
  // the top-face half to Qt.  Output (s, i) of block t = s ^ e_i goes to the
  // bottom face with sign +1 and to the top face with sign (-1)^sz.
  auto element = [&](const T (&Plo)[4][3], const T (&Phi)[4][3], T E, T (&R)[4][3], T (&Qt)[4][3], auto bottom) {
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int c = 0; c < 3; ++c) Qt[s][c] = T(0);
    const T mE = -E;
    // blocks t and t ^ 4 read the same P entries and complete the same R / Qt
    // entries, so taking them in pairs keeps few values live
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int tt = (k >> 1) | ((k & 1) << 2);
      T uh[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int s = tt ^ (1 << j);
        uh[j] = (s & 4) ? Plo[s & 3][j] - Phi[s & 3][j] : Plo[s & 3][j] + Phi[s & 3][j];
      }
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        if (tt == (1 << i)) continue;  // rigid translation: zero row
        T acc = T(0);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          if (tt == (1 << j)) continue;  // rigid translation: zero column
          acc = fma(p.mb.m[tt][i][j], uh[j], acc);
        }
        const int s = tt ^ (1 << i);
        if constexpr (decltype(bottom)::value) R[s & 3][i] = fma(E, acc, R[s & 3][i]);
        Qt[s & 3][i] = fma((s & 4) ? mE : E, acc, Qt[s & 3][i]);
      }
    }
  };

  // prologue: P of plane zb, and the top-face half of element zb - 1
  T P0[4][3], Qt[4][3], vcur[3], vn[3];
  {
    T v[3], Plo[4][3];
    load_u(zb - 1, v);
    load_u(zb, vcur);
    load_u(zb + 1, vn);
    const T E = load_E(zb - 1);
    plane_wht(v, Plo);
    __syncthreads();
    plane_wht(vcur, P0);
    element(Plo, P0, E, Qt, Qt, std::false_type{});
    __syncthreads();
  }
  T En = load_E(zb);
  double part = 0.0;

  for (int z = zb; z < ze; ++z) {
    // next plane and slab in flight during this plane's arithmetic
    T vn2[3];
    load_u(z + 2, vn2);
    const T En2 = load_E(z + 1);
    const long long n = nbase + z * pstride;
    T Pn[4][3];
    plane_wht(vn, Pn);
    T R[4][3], Qn[4][3];
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int c = 0; c < 3; ++c) R[s][c] = Qt[s][c];
    element(P0, Pn, En, R, Qn, std::true_type{});
    EpiIn<T> in[3];
    if (writer) {
#pragma unroll
      for (int c = 0; c < 3; ++c) in[c] = epi_load<T, MODE>(p.io, 3 * n + c);
    }
    // 2D inverse: corner contributions of this element column on plane z
    T own_c[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const T a0 = R[0][c] + R[1][c], a1 = R[0][c] - R[1][c];  // sx summed / differenced
      const T b0 = R[2][c] + R[3][c], b1 = R[2][c] - R[3][c];
      own_c[c] = a0 + b0;                 // corner (0, 0)
      sc[(0 * 3 + c) * NTHR + t] = a1 + b1;  // corner (1, 0)
      sc[(1 * 3 + c) * NTHR + t] = a0 - b0;  // corner (0, 1)
      sc[(2 * 3 + c) * NTHR + t] = a1 - b1;  // corner (1, 1)
    }
    __syncthreads();
    if (writer) {
      const int f = fix[n];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const T kv = own_c[c] + sc[(0 * 3 + c) * NTHR + t - PY] + sc[(1 * 3 + c) * NTHR + t - 1] +
                     sc[(2 * 3 + c) * NTHR + t - PY - 1];
        op_epilogue<T, MODE>(p.io, 3 * n + c, (f >> c) & 1, kv, vcur[c], in[c], part);
      }
    }
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        P0[s][c] = Pn[s][c];
        Qt[s][c] = Qn[s][c];
      }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      vcur[c] = vn[c];
      vn[c] = vn2[c];
    }
    En = En2;
  }
  if constexpr (mode_reduces<MODE>()) {
    part = block_sum(part, red);
    if (t == 0) p.io.partials[blockIdx.y * gridDim.x + blockIdx.x] = part;
    if (p.io.fin_count)
      last_block_finalize(p.io.partials, gridDim.x * gridDim.y, p.io.fin_count, p.io.fin, p.io.fin_op, red);
  }
}

}  // namespace tp3d

namespace tp3d {

// Block shapes offered for the Walsh-Hadamard operator (threads, minimum
// resident blocks per SM, and the kernel: the scalar two-barrier kernel, the
// one-barrier kernel of tp3d_fine_wht1.cuh, for FP32 also the packed two-plane
// kernel).  Explicit instantiations live in tp3d_fine_wht.cu; the solver times
// them on its own grid and keeps the fastest.  kWhtVariants is the most any
// precision offers (wht_variant_count).
constexpr int kWhtVariants = 8;

// Host view of one launch configuration.
struct WhtTile {
  int variant = 0, nthr = 512;
  int TX = 1, TY = 1, PY = 3, tiles_y = 1, tiles_x = 1, ZC = 1, zchunks = 1, occ = 1;
};

template <typename T, class ESrc>
int wht_variant_threads(int v);
template <typename T, class ESrc>
int wht_variant_count();
// false for shapes that the timed choice skips (taken only when asked for by name)
template <typename T, class ESrc>
bool wht_variant_timed(int v);
template <typename T, class ESrc>
int wht_occupancy(int v);
template <typename T, class ESrc>
int wht_launch(const WhtParams<T, ESrc>& p, int mode, int v, dim3 grid, cudaStream_t st, bool pdl = false);

// Walsh-Hadamard blocks of KE (see the top of this file); false when KE is not
// block diagonal in that basis to 1e-12 of its largest entry, or the
// translation rows are not zero, in which case the dense form is used.
bool wht_blocks_from_ke(const double* KE, double m[8][3][3]);

// Tile and z chunking for variant v on grid g (nsm SMs): the first of
// wht_tile_candidates.
template <typename T, class ESrc>
WhtTile wht_choose_tile(const Grid& g, int nsm, int v);
// Up to max_out tile shapes for variant v, the fewest blocks per node plane
// first, each with its modelled z chunking; returns how many were written.
template <typename T, class ESrc>
int wht_tile_candidates(const Grid& g, int nsm, int v, WhtTile* out, int max_out);

}  // namespace tp3d
