// Fine-level operator in the Walsh-Hadamard corner basis with one block
// barrier per node plane.
//
// Same operator, arithmetic and summation order as wht_apply_kernel
// (tp3d_fine_wht.cuh: the element stiffness of an axis-aligned orthotropic H8
// element, lk_H8 in pytopo3d/utils/stiffness.py:12-130, splits into eight 3x3
// blocks in the basis u_hat(s, i) = sum_a (-1)^(s.a) u(a, i)), so the two
// kernels give bit-identical results.  What differs is the exchange between
// the threads of a block:
//  * a node's masked u and its fixed-DOF bits form one 4-word shared record
//    (16 bytes in FP32), so a neighbour's three components are one vector
//    load instead of three scalar ones; the corner contributions of the
//    inverse transform are 4-word records too;
//  * node records rotate through three plane buffers and corner records
//    through two: step z stores its node record for plane z+1, waits once,
//    reads the corner contributions that step z-1 left for plane z-1 and its
//    own plane z-1 record and finishes plane z-1's epilogue, then reads the
//    plane z+1 neighbours, computes element z and leaves its corner
//    contributions for step z+1.  One barrier per plane instead of two, and
//    nothing of plane z-1 but its own corner is carried in registers;
//  * consecutive steps use two register sets alternately (the plane loop is
//    unrolled by two), so no values are moved between steps, and a plane's
//    u and fixed-DOF bits, loaded two planes ahead, are first used a whole
//    step later, when the node record is stored.
// The epilogue of plane z therefore runs one step later than in the
// two-barrier kernel; its inputs are requested before the barrier that
// precedes it.  The solver runs this kernel for the apply, residual, CG-product
// and power-iteration epilogues (tp3d_fine_wht.cu, wht1_mode): the Chebyshev
// steps' nine inputs per node make it spill under 64 registers.
#pragma once

#include "tp3d_fine_wht.cuh"

namespace tp3d {

// Shared 4-word records.  Node record: masked u and the fixed-DOF bits (as the
// fourth word's bit pattern); corner record: three components and a pad word.
template <typename T>
__device__ __forceinline__ void wht1_st4(T* base, int idx, const T (&v)[3], int f) {
  if constexpr (sizeof(T) == 4) {
    reinterpret_cast<float4*>(base)[idx] = make_float4(v[0], v[1], v[2], __int_as_float(f));
  } else {
    reinterpret_cast<double2*>(base)[2 * idx] = make_double2(v[0], v[1]);
    reinterpret_cast<double2*>(base)[2 * idx + 1] = make_double2(v[2], __longlong_as_double((long long)f));
  }
}
template <typename T>
__device__ __forceinline__ void wht1_ld3(const T* base, int idx, T (&v)[3]) {
  if constexpr (sizeof(T) == 4) {
    const float4 q = reinterpret_cast<const float4*>(base)[idx];
    v[0] = q.x;
    v[1] = q.y;
    v[2] = q.z;
  } else {
    const double2 q = reinterpret_cast<const double2*>(base)[2 * idx];
    v[0] = q.x;
    v[1] = q.y;
    v[2] = base[4 * idx + 2];
  }
}
template <typename T>
__device__ __forceinline__ int wht1_ld4(const T* base, int idx, T (&v)[3]) {
  if constexpr (sizeof(T) == 4) {
    const float4 q = reinterpret_cast<const float4*>(base)[idx];
    v[0] = q.x;
    v[1] = q.y;
    v[2] = q.z;
    return __float_as_int(q.w);
  } else {
    const double2 q = reinterpret_cast<const double2*>(base)[2 * idx];
    const double2 r = reinterpret_cast<const double2*>(base)[2 * idx + 1];
    v[0] = q.x;
    v[1] = q.y;
    v[2] = r.x;
    return (int)__double_as_longlong(r.y);
  }
}

// three buffers of node records + two buffers of three corner records, 4 words each
template <typename T>
__host__ __device__ constexpr size_t wht1_smem_bytes(int nthr) {
  return (size_t)(3 * 4 + 2 * 3 * 4) * nthr * sizeof(T);
}

template <typename T, class ESrc, int MODE, int NTHR, int MINB>
__global__ void __launch_bounds__(NTHR, MINB) wht1_apply_kernel(const __grid_constant__ WhtParams<T, ESrc> p) {
  pdl_entry();
  if (op_skip(p.io)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* su = reinterpret_cast<T*>(smem_raw);  // [3][NTHR] node records, plane k in buffer k % 3
  T* sc = su + 3 * 4 * NTHR;               // [2][3][NTHR] corner (1,0), (0,1), (1,1) records
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
  const bool elem_cols = inpatch && lx <= p.TX && ly <= p.TY;
  const bool elem_in = elem_cols && gx >= 0 && gx < p.g.nx && gy >= 0 && gy < p.g.ny;
  const bool writer = node_in && lx >= 1 && lx <= p.TX && ly >= 1 && ly <= p.TY;
  const long long pstride = (long long)NX * NY;
  const long long sstride = (long long)p.g.nx * p.g.ny;
  const long long nbase = node_in ? gy + (long long)NY * gx : 0;
  const long long ebase = elem_in ? gy + (long long)p.g.ny * gx : 0;
  const T* __restrict__ u = p.io.u;
  const uint8_t* __restrict__ fix = p.fix;
  constexpr int REC = 4 * NTHR;  // words per record buffer

  auto load_E = [&](int zs) -> T {
    return (elem_in && zs >= 0 && zs < p.g.nz) ? (T)p.esrc(ebase + zs * sstride) : T(0);
  };
  // 2D transform of this element column's corners on one plane from the node
  // records in buf (this node's own values in v)
  auto plane_wht = [&](const T* buf, const T (&v)[3], T (&P)[4][3]) {
    if (elem_cols) {
      T n01[3], n10[3], n11[3];
      wht1_ld3(buf, t + 1, n01);
      wht1_ld3(buf, t + PY, n10);
      wht1_ld3(buf, t + PY + 1, n11);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const T a0 = v[c] + n01[c], a1 = v[c] - n01[c], b0 = n10[c] + n11[c], b1 = n10[c] - n11[c];
        P[0][c] = a0 + b0;
        P[1][c] = a0 - b0;
        P[2][c] = a1 + b1;
        P[3][c] = a1 - b1;
      }
    } else {
#pragma unroll
      for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int c = 0; c < 3; ++c) P[s][c] = T(0);
    }
  };
  // element between the planes of Plo and Phi (see wht_apply_kernel)
  auto element = [&](const T (&Plo)[4][3], const T (&Phi)[4][3], T E, T (&R)[4][3], T (&Qt)[4][3], auto bottom) {
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int c = 0; c < 3; ++c) Qt[s][c] = T(0);
    const T mE = -E;
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
        if (tt == (1 << i)) continue;
        T acc = T(0);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          if (tt == (1 << j)) continue;
          acc = fma(p.mb.m[tt][i][j], uh[j], acc);
        }
        const int s = tt ^ (1 << i);
        if constexpr (decltype(bottom)::value) R[s & 3][i] = fma(E, acc, R[s & 3][i]);
        Qt[s & 3][i] = fma((s & 4) ? mE : E, acc, Qt[s & 3][i]);
      }
    }
  };
  double part = 0.0;
  // plane zp's output from its own corner oc, the three neighbour corners in
  // corner buffer cb and its own node record in node buffer nb
  auto finish = [&](const T* cb, const T* nb, int zp, const T (&oc)[3], const EpiIn<T> (&in)[3]) {
    T c10[3], c01[3], c11[3], vo[3];
    wht1_ld3(cb, t - PY, c10);
    wht1_ld3(cb + REC, t - 1, c01);
    wht1_ld3(cb + 2 * REC, t - PY - 1, c11);
    const int f = wht1_ld4(nb, t, vo);
    const long long n = nbase + zp * pstride;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const T kv = oc[c] + c10[c] + c01[c] + c11[c];
      op_epilogue<T, MODE>(p.io, 3 * n + c, (f >> c) & 1, kv, vo[c], in[c], part);
    }
  };
  auto epi_inputs = [&](int zp, EpiIn<T> (&in)[3]) {
    const long long n = nbase + zp * pstride;
#pragma unroll
    for (int c = 0; c < 3; ++c) in[c] = epi_load<T, MODE>(p.io, 3 * n + c);
  };

  // unmasked u of this thread's node on plane zp and its fixed-DOF bits (0
  // outside); masked only when the record is stored, a step later, so that the
  // loads stay in flight for a whole step
  auto load_raw = [&](int zp, T (&v)[3]) -> int {
    if (node_in && zp >= 0 && zp < NZ) {
      const long long n = nbase + zp * pstride;
      v[0] = u[3 * n];
      v[1] = u[3 * n + 1];
      v[2] = u[3 * n + 2];
      return fix[n];
    }
    v[0] = v[1] = v[2] = T(0);
    return 0;
  };
  auto mask = [](const T (&r)[3], int f, T (&v)[3]) {
    v[0] = (f & 1) ? T(0) : r[0];
    v[1] = (f & 2) ? T(0) : r[1];
    v[2] = (f & 4) ? T(0) : r[2];
  };

  // prologue: P of plane zb and the top-face half of element zb - 1
  int bm = (zb + 2) % 3, b0 = zb % 3, b1 = (zb + 1) % 3;  // node buffers of planes z-1, z, z+1
  // two register sets used alternately by consecutive steps (no rotation moves):
  // P and Qt of the current plane, the next plane's raw u, the modulus, the own corner
  T PA[4][3], PB[4][3], QA[4][3], QB[4][3], uA[3], uB[3], EA, EB, oA[3] = {T(0), T(0), T(0)}, oB[3];
  int fA, fB;
  {
    T r[3], v[3], vc[3], Plo[4][3];
    const int fm = load_raw(zb - 1, r);
    mask(r, fm, v);
    const int fc = load_raw(zb, r);
    mask(r, fc, vc);
    fA = load_raw(zb + 1, uA);
    const T E = load_E(zb - 1);
    wht1_st4(su + bm * REC, t, v, fm);
    wht1_st4(su + b0 * REC, t, vc, fc);
    __syncthreads();
    plane_wht(su + bm * REC, v, Plo);
    plane_wht(su + b0 * REC, vc, PA);
    element(Plo, PA, E, QA, QA, std::false_type{});
  }
  EA = load_E(zb);

  // one step: plane z's P in Pc, element z-1's top half in Qc, plane z+1's raw u
  // in uc / fc, element z's modulus in Ec, plane z-1's own corner in oc; fills
  // the other set for step z+1
  auto step = [&](int z, T (&Pc)[4][3], T (&Pn)[4][3], T (&Qc)[4][3], T (&Qn)[4][3], const T (&uc)[3], int fc,
                  T (&un)[3], int& fnx, T Ec, T& Enx, const T (&oc)[3], T (&on)[3]) {
    fnx = load_raw(z + 2, un);
    Enx = load_E(z + 1);
    const bool fin_prev = writer && z > zb;
    EpiIn<T> in[3];
    if (fin_prev) epi_inputs(z - 1, in);
    // plane z+1's buffer last held plane z-2, whose readers all passed the
    // previous barrier
    T vn[3];
    mask(uc, fc, vn);
    T* ubuf = su + b1 * REC;
    wht1_st4(ubuf, t, vn, fc);
    __syncthreads();
    // plane z-1 first, so that its inputs are dead before plane z+1's transform
    if (fin_prev) finish(sc + ((z - 1) & 1) * 3 * REC, su + bm * REC, z - 1, oc, in);
    plane_wht(ubuf, vn, Pn);
    T R[4][3];
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int c = 0; c < 3; ++c) R[s][c] = Qc[s][c];
    element(Pc, Pn, Ec, R, Qn, std::true_type{});
    // 2D inverse: this column's own corner kept, the other three left for the neighbours
    T* cb = sc + (z & 1) * 3 * REC;
    T c10[3], c01[3], c11[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const T a0 = R[0][c] + R[1][c], a1 = R[0][c] - R[1][c];
      const T q0 = R[2][c] + R[3][c], q1 = R[2][c] - R[3][c];
      on[c] = a0 + q0;
      c10[c] = a1 + q1;
      c01[c] = a0 - q0;
      c11[c] = a1 - q1;
    }
    wht1_st4(cb, t, c10, 0);
    wht1_st4(cb + REC, t, c01, 0);
    wht1_st4(cb + 2 * REC, t, c11, 0);
    bm = b0;
    b0 = b1;
    b1 = (b1 == 2) ? 0 : b1 + 1;
  };
  int z = zb;
  for (; z + 1 < ze; z += 2) {
    step(z, PA, PB, QA, QB, uA, fA, uB, fB, EA, EB, oA, oB);
    step(z + 1, PB, PA, QB, QA, uB, fB, uA, fA, EB, EA, oB, oA);
  }
  const bool odd = z < ze;
  if (odd) step(z, PA, PB, QA, QB, uA, fA, uB, fB, EA, EB, oA, oB);
  // the last plane's epilogue (its node record is in buffer bm after the rotation)
  {
    EpiIn<T> in[3];
    if (writer) epi_inputs(ze - 1, in);
    __syncthreads();
    if (writer) finish(sc + ((ze - 1) & 1) * 3 * REC, su + bm * REC, ze - 1, odd ? oB : oA, in);
  }
  if constexpr (mode_reduces<MODE>()) {
    part = block_sum(part, red);
    if (t == 0) p.io.partials[blockIdx.y * gridDim.x + blockIdx.x] = part;
    if (p.io.fin_count)
      last_block_finalize(p.io.partials, gridDim.x * gridDim.y, p.io.fin_count, p.io.fin, p.io.fin_op, red);
  }
}

}  // namespace tp3d
