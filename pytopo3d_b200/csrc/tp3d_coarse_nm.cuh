// Coarse-level operator from a node-major bf16 stencil, three lanes per node.
//
// The coarse levels hold Galerkin stencils (27 neighbour nodes x 3 x 3
// coefficients per node; the multigrid that replaces the reference's direct
// solve, pytopo3d/utils/solver.py:15-73).  The packed layout (one coefficient
// plane per DOF, stencil_apply_kernel) costs each DOF 81 two-byte coefficient
// loads and 81 neighbour loads, and the three DOFs of a node load the same 81
// neighbour values.  Here the level's bf16 stencil is stored node-major in three
// z-plane segments of 88 entries (the 9 in-plane neighbours x 3 rows x 3
// columns, then 7 zeros; 528 bytes per node, every segment 16-byte aligned):
//  * lane a of a group of three (ten groups per warp, lanes 30 and 31 idle)
//    takes the neighbours on z-plane a: 11 16-byte coefficient loads and 27
//    neighbour loads, and the node's three partial rows;
//  * the group rotates its partial rows with two shuffles, so that lane a ends
//    with row a's sum over the three planes (own plane first), and runs the
//    epilogue of DOF 3n + a: the warp's loads and stores of the epilogue are
//    30 consecutive DOFs.
// The coefficients are the packed layout's bf16 values (fixed rows and columns
// and neighbours past the grid zero): the level builders write them node-major
// directly (store_packed_rows), and levels built otherwise (the stencil triple
// product) are permuted by nm3_pack_kernel.  The rows are summed in a
// different order, so results round differently from the packed kernel's.
#pragma once

#include "tp3d_hex.cuh"

namespace tp3d {

constexpr int kNM3Seg = 88;           // entries per z-plane segment (81 + 7 zeros)
constexpr int kNM3Row = 3 * kNM3Seg;  // entries per node (528 bytes)

// Entry of node n for the neighbour at z-plane a, x-offset b, y-offset e
// (each 0..2, offset + 1), row component c and column component d.
__host__ __device__ __forceinline__ long long nm3_index(long long n, int a, int b, int e, int c, int d) {
  return n * kNM3Row + a * kNM3Seg + ((3 * b + e) * 3 + c) * 3 + d;
}

// Node-major copy of a level's packed bf16 stencil S (entry (n, c, j, d) at
// S[(3 j + d) ndof + 3 n + c], j = 9 a + 3 b + e the neighbour in z, x, y order):
// SN[n kNM3Row + a kNM3Seg + ((3 b + e) 3 + c) 3 + d].
__global__ void nm3_pack_kernel(Grid g, const __nv_bfloat16* __restrict__ S, __nv_bfloat16* __restrict__ SN) {
  const long long nn = g.nnode(), ndof = 3 * nn;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < nn * kNM3Row;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long n = idx / kNM3Row;
    const int k = (int)(idx - n * kNM3Row);
    const int a = k / kNM3Seg, r = k - a * kNM3Seg;
    __nv_bfloat16 v = __float2bfloat16(0.0f);
    if (r < 81) {
      const int j = 9 * a + r / 9, c = (r / 3) % 3, d = r % 3;
      v = S[(3 * j + d) * ndof + 3 * n + c];
    }
    SN[idx] = v;
  }
}

template <typename T, int MODE>
__global__ void __launch_bounds__(256) nm3_apply_kernel(const __grid_constant__ StencilParams<T, __nv_bfloat16> p) {
  pdl_entry();
  if (op_skip(p.io)) return;
  __shared__ double red[32];
  const Grid g = p.g;
  const int NX = g.nx + 1, NY = g.ny + 1, NZ = g.nz + 1;
  const int NXY = NX * NY, nn = NXY * NZ;
  const int lane = threadIdx.x & 31;
  const int grp = lane / 3, a = lane - 3 * grp;  // node of the warp's ten, and this lane's z-plane / row
  const T* __restrict__ u = p.io.u;
  const int wpb = blockDim.x >> 5;
  double part = 0.0;
  // warp-uniform loop over groups of ten nodes (every lane reaches the shuffles)
  for (int w = blockIdx.x * wpb + (threadIdx.x >> 5); w * 10 < nn; w += gridDim.x * wpb) {
    const int n = 10 * w + grp;
    const bool live = lane < 30 && n < nn;
    const int i = 3 * n + a;
    EpiIn<T> in;
    if (live) in = epi_load<T, MODE>(p.io, i);
    T y[3] = {T(0), T(0), T(0)};
    if (live) {
      const int iy = n % NY, r = n / NY;
      const int ix = r % NX, iz = r / NX;
      const int oy0 = iy > 0 ? -1 : 0, oy2 = iy < NY - 1 ? 1 : 0;
      const int ox0 = ix > 0 ? -NY : 0, ox2 = ix < NX - 1 ? NY : 0;
      const int oz = a == 0 ? (iz > 0 ? -NXY : 0) : (a == 1 ? 0 : (iz < NZ - 1 ? NXY : 0));
      const uint4* row = reinterpret_cast<const uint4*>(p.S + (size_t)n * kNM3Row + a * kNM3Seg);
      uint4 cw[11];
#pragma unroll
      for (int q = 0; q < 11; ++q) cw[q] = __ldg(row + q);
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const int ox = b == 0 ? ox0 : (b == 1 ? 0 : ox2);
#pragma unroll
        for (int e = 0; e < 3; ++e) {
          const int oy = e == 0 ? oy0 : (e == 1 ? 0 : oy2);
          const int m3 = 3 * (n + oz + ox + oy);
          const T um[3] = {__ldg(&u[m3]), __ldg(&u[m3 + 1]), __ldg(&u[m3 + 2])};
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              const int k = ((3 * b + e) * 3 + c) * 3 + d;
              const uint4 q4 = cw[k >> 3];
              const unsigned wd = (k & 6) == 0 ? q4.x : ((k & 6) == 2 ? q4.y : ((k & 6) == 4 ? q4.z : q4.w));
              const unsigned bits = (k & 1) ? (wd & 0xffff0000u) : (wd << 16);
              y[c] = fma((T)__uint_as_float(bits), um[d], y[c]);
            }
        }
      }
    }
    // lane a keeps row a of its own plane and receives row a of planes a+1 and
    // a+2 (mod 3): in round t the lane of plane l sends its row (l - t) mod 3
    T kv = y[a];
#pragma unroll
    for (int t = 1; t < 3; ++t) {
      const int sidx = (a + 3 - t) % 3;
      const T send = sidx == 0 ? y[0] : (sidx == 1 ? y[1] : y[2]);
      const int src = 3 * grp + (a + t) % 3;
      kv += __shfl_sync(0xffffffffu, send, src);
    }
    if (live) {
      const bool fx = (p.fix[n] >> a) & 1;
      op_epilogue<T, MODE>(p.io, i, fx, kv, fx ? T(0) : u[i], in, part);
    }
  }
  if (mode_reduces<MODE>()) {
    part = block_sum(part, red);
    if (threadIdx.x == 0) p.io.partials[blockIdx.x] = part;
    if (p.io.fin_count) last_block_finalize(p.io.partials, gridDim.x, p.io.fin_count, p.io.fin, p.io.fin_op, red);
  }
}

}  // namespace tp3d
