// Fine-level operator in the Walsh-Hadamard corner basis, FP32, two node
// planes per step in packed FP32 arithmetic (Blackwell's paired FADD2 / FFMA2).
//
// Same operator as wht_apply_kernel (tp3d_fine_wht.cuh): the element stiffness
// of an axis-aligned orthotropic H8 element (lk_H8,
// pytopo3d/utils/stiffness.py:12-130) splits into eight 3x3 blocks in the basis
// u_hat(s, i) = sum_a (-1)^(s.a) u(a, i), and the transforms are separable.
// Here a block still owns a (TX + 2) x (TY + 2) patch of node columns, one
// thread per column, marching along z, but each step handles the node planes
// z and z + 1 together:
//  * every thread holds its column's values on planes z+1 and z+2 as float2
//    pairs; one shared-memory exchange and one barrier give the 2D transforms
//    of both planes, packed: P = (P_{z+1}, P_{z+2});
//  * the elements z and z+1 are one packed computation: their lower faces are
//    (P_z, P_{z+1}) (P_z carried from the previous step) and their upper faces
//    (P_{z+1}, P_{z+2}); every block product is one FFMA2 per entry;
//  * plane z receives the top half of element z-1 (carried) and the bottom
//    half of element z, plane z+1 the top half of element z and the bottom half
//    of element z+1: one packed add; the top half of element z+1 is carried;
//  * the 2D inverse and the exchange of the three neighbour corner
//    contributions run packed over both planes, with one more barrier.
// Per node and plane that is half the arithmetic instructions, half the
// shared-memory instructions and half the barriers of the scalar kernel.
// FADD2 / FFMA2 round each lane as FADD / FFMA do.
#pragma once

#include "tp3d_fine_wht.cuh"

namespace tp3d {

__device__ __forceinline__ float2 p_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 p_sub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 p_fma(float m, float2 u, float2 c) { return __ffma2_rn(make_float2(m, m), u, c); }
__device__ __forceinline__ float2 p_fma2(float2 a, float2 u, float2 c) { return __ffma2_rn(a, u, c); }
__device__ __forceinline__ float p_add(float a, float b) { return a + b; }
__device__ __forceinline__ float p_sub(float a, float b) { return a - b; }
__device__ __forceinline__ float p_fma(float m, float u, float c) { return fmaf(m, u, c); }
__device__ __forceinline__ float p_fma2(float a, float u, float c) { return fmaf(a, u, c); }
template <typename V>
__device__ __forceinline__ V p_zero();
template <>
__device__ __forceinline__ float p_zero<float>() { return 0.0f; }
template <>
__device__ __forceinline__ float2 p_zero<float2>() { return make_float2(0.0f, 0.0f); }

__host__ __device__ constexpr size_t wht2_smem_bytes(int nthr) { return (size_t)12 * nthr * sizeof(float2); }

// One element (or a packed pair of elements) in the transformed basis: lower
// face Plo, upper face Phi, moduli E (mE = -E).  Adds the bottom-face half of
// each block output to Rb and the top-face half to Qt (sign (-1)^sz).  Blocks
// t and t ^ 4 read the same entries, so they are taken in pairs.
template <typename V>
__device__ __forceinline__ void wht_element(const WhtBlocks<float>& mb, const V (&Plo)[4][3], const V (&Phi)[4][3],
                                            V E, V mE, V (&Rb)[4][3], V (&Qt)[4][3]) {
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int tt = (k >> 1) | ((k & 1) << 2);
    V uh[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const int s = tt ^ (1 << j);
      uh[j] = (s & 4) ? p_sub(Plo[s & 3][j], Phi[s & 3][j]) : p_add(Plo[s & 3][j], Phi[s & 3][j]);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      if (tt == (1 << i)) continue;  // rigid translation: zero row
      V acc = p_zero<V>();
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        if (tt == (1 << j)) continue;  // rigid translation: zero column
        acc = p_fma(mb.m[tt][i][j], uh[j], acc);
      }
      const int s = tt ^ (1 << i);
      Rb[s & 3][i] = p_fma2(E, acc, Rb[s & 3][i]);
      Qt[s & 3][i] = p_fma2((s & 4) ? mE : E, acc, Qt[s & 3][i]);
    }
  }
}

template <class ESrc, int MODE, int NTHR, int MINB>
__global__ void __launch_bounds__(NTHR, MINB) wht2_apply_kernel(const __grid_constant__ WhtParams<float, ESrc> p) {
  pdl_entry();
  if (op_skip(p.io)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* su = reinterpret_cast<float2*>(smem_raw);  // [3][NTHR] masked u of each column, planes (a, a+1)
  float2* sc = su + 3 * NTHR;                        // [9][NTHR] corner (1,0), (0,1), (1,1) contributions
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
  const float* __restrict__ u = p.io.u;
  const uint8_t* __restrict__ fix = p.fix;

  // masked u of this thread's node on plane zp (0 outside the grid)
  auto load_u = [&](int zp, float (&v)[3]) {
    if (node_in && zp >= 0 && zp < NZ) {
      const long long n = nbase + zp * pstride;
      const float a = u[3 * n], b = u[3 * n + 1], c = u[3 * n + 2];
      const int f = fix[n];
      v[0] = (f & 1) ? 0.0f : a;
      v[1] = (f & 2) ? 0.0f : b;
      v[2] = (f & 4) ? 0.0f : c;
    } else {
      v[0] = v[1] = v[2] = 0.0f;
    }
  };
  auto load_E = [&](int zs) -> float {
    return (elem_in && zs >= 0 && zs < p.g.nz) ? (float)p.esrc(ebase + zs * sstride) : 0.0f;
  };
  // Packed 2D transforms of this element column's corners on two planes: stores
  // this node's pair, waits, then reads the (x+1, y), (x, y+1), (x+1, y+1)
  // nodes' pairs.  The caller guarantees that every thread has finished reading
  // su since the previous call.
  auto plane_wht2 = [&](const float (&va)[3], const float (&vb)[3], float2 (&P)[4][3]) {
#pragma unroll
    for (int c = 0; c < 3; ++c) su[c * NTHR + t] = make_float2(va[c], vb[c]);
    __syncthreads();
    if (elem_cols) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float2 u00 = make_float2(va[c], vb[c]), u01 = su[c * NTHR + t + 1];
        const float2 u10 = su[c * NTHR + t + PY], u11 = su[c * NTHR + t + PY + 1];
        const float2 a0 = p_add(u00, u01), a1 = p_sub(u00, u01), b0 = p_add(u10, u11), b1 = p_sub(u10, u11);
        P[0][c] = p_add(a0, b0);  // (sx, sy) = (0, 0)
        P[1][c] = p_sub(a0, b0);  // (1, 0)
        P[2][c] = p_add(a1, b1);  // (0, 1)
        P[3][c] = p_sub(a1, b1);  // (1, 1)
      }
    } else {
#pragma unroll
      for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int c = 0; c < 3; ++c) P[s][c] = make_float2(0.0f, 0.0f);
    }
  };

  // prologue: P of plane zb and the top-face half of element zb - 1 (carried
  // into plane zb); own values of plane zb and the next two planes
  float Pz[4][3], Qc[4][3], vz[3], v1[3], v2[3];
  {
    float va[3];
    load_u(zb - 1, va);
    load_u(zb, vz);
    load_u(zb + 1, v1);
    load_u(zb + 2, v2);
    const float E = load_E(zb - 1);
    float2 PP[4][3];
    plane_wht2(va, vz, PP);
    float Plo[4][3], Rb[4][3];
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        Plo[s][c] = PP[s][c].x;
        Pz[s][c] = PP[s][c].y;
        Rb[s][c] = 0.0f;
        Qc[s][c] = 0.0f;
      }
    wht_element<float>(p.mb, Plo, Pz, E, -E, Rb, Qc);
    __syncthreads();
  }
  float2 Ep = make_float2(load_E(zb), load_E(zb + 1));
  double part = 0.0;

  for (int z = zb; z < ze; z += 2) {
    const bool second = z + 1 < ze;  // plane z + 1 belongs to this block
    // the next step's planes and elements in flight during this step's arithmetic
    float w1[3], w2[3];
    load_u(z + 3, w1);
    load_u(z + 4, w2);
    const float2 Ep2 = make_float2(load_E(z + 2), load_E(z + 3));
    const long long n0 = nbase + z * pstride, n1 = n0 + pstride;
    // packed transforms of planes z+1, z+2; elements z and z+1 as one pair.
    // Plane z receives the carried top of element z-1 and the bottom of element
    // z (lane x of Rb, which starts from the carry); plane z+1 the top of element
    // z (lane x of Qt) and the bottom of element z+1 (lane y of Rb); the top of
    // element z+1 (lane y of Qt) is carried.
    float2 Phi[4][3], Plo[4][3], Rb[4][3], Qt[4][3];
    plane_wht2(v1, v2, Phi);
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        Plo[s][c] = make_float2(Pz[s][c], Phi[s][c].x);
        Rb[s][c] = make_float2(Qc[s][c], 0.0f);
        Qt[s][c] = make_float2(0.0f, 0.0f);
      }
    wht_element<float2>(p.mb, Plo, Phi, Ep, make_float2(-Ep.x, -Ep.y), Rb, Qt);
    EpiIn<float> in0[3], in1[3];
    if (writer) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        in0[c] = epi_load<float, MODE>(p.io, 3 * n0 + c);
        if (second) in1[c] = epi_load<float, MODE>(p.io, 3 * n1 + c);
      }
    }
    float2 R[4][3];
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        R[s][c] = make_float2(Rb[s][c].x, Rb[s][c].y + Qt[s][c].x);
        Qc[s][c] = Qt[s][c].y;
        Pz[s][c] = Phi[s][c].y;
      }
    // packed 2D inverse: corner contributions of this element column on both planes
    float2 own_c[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float2 a0 = p_add(R[0][c], R[1][c]), a1 = p_sub(R[0][c], R[1][c]);
      const float2 b0 = p_add(R[2][c], R[3][c]), b1 = p_sub(R[2][c], R[3][c]);
      own_c[c] = p_add(a0, b0);                      // corner (0, 0)
      sc[(0 * 3 + c) * NTHR + t] = p_add(a1, b1);    // corner (1, 0)
      sc[(1 * 3 + c) * NTHR + t] = p_sub(a0, b0);    // corner (0, 1)
      sc[(2 * 3 + c) * NTHR + t] = p_sub(a1, b1);    // corner (1, 1)
    }
    __syncthreads();
    if (writer) {
      const int f0 = fix[n0];
      const int f1 = second ? fix[n1] : 7;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float2 kv = p_add(p_add(p_add(own_c[c], sc[(0 * 3 + c) * NTHR + t - PY]), sc[(1 * 3 + c) * NTHR + t - 1]),
                                sc[(2 * 3 + c) * NTHR + t - PY - 1]);
        op_epilogue<float, MODE>(p.io, 3 * n0 + c, (f0 >> c) & 1, kv.x, vz[c], in0[c], part);
        if (second) op_epilogue<float, MODE>(p.io, 3 * n1 + c, (f1 >> c) & 1, kv.y, v1[c], in1[c], part);
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      vz[c] = v2[c];
      v1[c] = w1[c];
      v2[c] = w2[c];
    }
    Ep = Ep2;
  }
  if constexpr (mode_reduces<MODE>()) {
    part = block_sum(part, red);
    if (t == 0) p.io.partials[blockIdx.y * gridDim.x + blockIdx.x] = part;
    if (p.io.fin_count)
      last_block_finalize(p.io.partials, gridDim.x * gridDim.y, p.io.fin_count, p.io.fin, p.io.fin_op, red);
  }
}

}  // namespace tp3d
