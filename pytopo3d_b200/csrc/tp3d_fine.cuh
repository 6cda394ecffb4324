// Matrix-free fine-level operator y = Z K(E) Z u + (I - Z) u with fused epilogues.
//
// A block owns a TY x TX column of nodes (TY a compile-time tile height, TX
// chosen at run time) and marches along z over a chunk of ZC node planes,
// NZT planes per step:
//  * shared memory holds a ring of NZT + 2 node planes of u (tile + 1 halo,
//    structure-of-arrays per component) and NZT + 1 element slabs of E; the
//    plane and slab pitches are compile-time, so every neighbour offset is an
//    immediate and a thread only keeps one base address per plane;
//  * the planes and slabs of the next step are loaded from global memory into
//    registers before the current step's arithmetic and stored to shared
//    memory after it, so global latency hides behind the FMAs;
//  * for NZT = 2 the two nodes of a thread share the four staged planes: 36
//    neighbour positions are read once (54 shared loads per node instead of 81);
//  * per node the 27 neighbours feed 8 per-element accumulators (576 FMAs, 24
//    independent chains per node); KE sits in kernel-parameter space, so every
//    FMA takes its coefficient from the constant bank.
// The epilogue (apply, residual, Chebyshev / Jacobi step, CG product with a
// block partial of p.q, power-iteration step) is chosen at run time.
#pragma once

#include "tp3d_hex.cuh"
#include "tp3d_ke_classes.h"

namespace tp3d {

template <typename T, class ESrc>
struct FineParams {
  KEP<T> ke;
  T kcls[kKEClasses];   // class values of ke (cubic-symmetric materials)
  Grid g;               // element grid
  int TX, ZC;           // tile width along x (runtime), z chunk (multiple of NZT)
  int tiles_y, tiles_x;
  int mode;             // ApplyMode
  const uint8_t* fix;   // per node, bit c = DOF c fixed
  ESrc esrc;
  OpIO<T> io;
};

template <int TY>
struct FineTile {
  static constexpr int PY = TY + 2;          // node-plane row pitch
  static constexpr int PXM = 256 / TY + 2;   // rows reserved per plane
  static constexpr int PP = PY * PXM;        // per-component plane pitch
  static constexpr int EY = TY + 1;          // element-slab row pitch
  static constexpr int EXM = 256 / TY + 1;
  static constexpr int EP = EY * EXM;
};

template <typename T, int TY, int NZT>
__host__ __device__ constexpr size_t fine_smem_bytes() {
  return (size_t)((NZT + 2) * 3 * FineTile<TY>::PP + (NZT + 1) * FineTile<TY>::EP) * sizeof(T);
}

template <typename T>
__device__ __forceinline__ EpiIn<T> fine_epi_load(int mode, const OpIO<T>& io, long long i) {
  switch (mode) {
    case kModeResid: return epi_load<T, kModeResid>(io, i);
    case kModeJacobi: return epi_load<T, kModeJacobi>(io, i);
    case kModeChebFirst: return epi_load<T, kModeChebFirst>(io, i);
    case kModeChebStep: return epi_load<T, kModeChebStep>(io, i);
    case kModeDinvApply: return epi_load<T, kModeDinvApply>(io, i);
    case kModeChebStepDot: return epi_load<T, kModeChebStepDot>(io, i);
    default: return EpiIn<T>{};
  }
}

template <typename T>
__device__ __forceinline__ void fine_epilogue(int mode, const OpIO<T>& io, long long i, bool fx, T kv, T own,
                                              const EpiIn<T>& in, double& part) {
  switch (mode) {
    case kModeApply: op_epilogue<T, kModeApply>(io, i, fx, kv, own, in, part); break;
    case kModeResid: op_epilogue<T, kModeResid>(io, i, fx, kv, own, in, part); break;
    case kModeJacobi: op_epilogue<T, kModeJacobi>(io, i, fx, kv, own, in, part); break;
    case kModeCgQ: op_epilogue<T, kModeCgQ>(io, i, fx, kv, own, in, part); break;
    case kModeChebFirst: op_epilogue<T, kModeChebFirst>(io, i, fx, kv, own, in, part); break;
    case kModeChebStep: op_epilogue<T, kModeChebStep>(io, i, fx, kv, own, in, part); break;
    case kModeChebStepDot: op_epilogue<T, kModeChebStepDot>(io, i, fx, kv, own, in, part); break;
    default: op_epilogue<T, kModeDinvApply>(io, i, fx, kv, own, in, part); break;
  }
}

// Coefficient KE[idx] of the element stiffness: with CLS, the cubic-symmetry
// class value held in a register (sign folded into the FMA operand); otherwise
// the full table in kernel-parameter space.
// (idx is a constant after unrolling, so the table lookup and the register
// selection fold away.)
template <typename T, bool CLS>
__device__ __forceinline__ T ke_coef(const KEP<T>& ke, const T (&kc)[kKEClasses], int idx) {
  if constexpr (CLS) {
    const int t = kKEClass[idx];
    return t > 0 ? kc[t - 1] : (t < 0 ? -kc[-t - 1] : T(0));
  } else {
    return ke.k[idx];
  }
}

template <typename T, class ESrc, int TY, int NZT, bool CLS>
__global__ void __launch_bounds__(256, 2) fine_apply_kernel(const __grid_constant__ FineParams<T, ESrc> p) {
  pdl_entry();
  if (op_skip(p.io)) return;
  using FT = FineTile<TY>;
  constexpr int PY = FT::PY, PP = FT::PP, EY = FT::EY, EP = FT::EP;
  constexpr int NPL = NZT + 2, NSL = NZT + 1;
  T kc[kKEClasses];
#pragma unroll
  for (int k = 0; k < kKEClasses; ++k) kc[k] = CLS ? p.kcls[k] : T(0);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* su = reinterpret_cast<T*>(smem_raw);  // NPL slots x 3 components x PP
  T* se = su + NPL * 3 * PP;               // NSL slots x EP
  __shared__ double red[32];

  const int TX = p.TX;
  const int NX = p.g.nx + 1, NY = p.g.ny + 1, NZ = p.g.nz + 1;
  const int by = blockIdx.x % p.tiles_y, bx = blockIdx.x / p.tiles_y;
  const int x0 = bx * TX, y0 = by * TY;
  const int zb = blockIdx.y * p.ZC, ze = min(zb + p.ZC, NZ);
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int ty = tid % TY, tx = tid / TY;
  const bool active = (tx < TX) && (x0 + tx < NX) && (y0 + ty < NY);
  const int PPA = PY * (TX + 2), EPA = EY * (TX + 1);
  const long long pstride = (long long)NX * NY;
  const long long sstride = (long long)p.g.nx * p.g.ny;
  const T* __restrict__ u = p.io.u;

  // this thread's staging elements (at most two per plane and per slab)
  long long gbase[2], ebase[2];
  bool gval[2], eval[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int i = tid + k * nthr;
    const int ly = i % PY, lx = i / PY;
    const int gx = x0 - 1 + lx, gy = y0 - 1 + ly;
    gval[k] = i < PPA && gx >= 0 && gx < NX && gy >= 0 && gy < NY;
    gbase[k] = gy + (long long)NY * gx;
    const int ey_ = i % EY, ex_ = i / EY;
    const int fx_ = x0 - 1 + ex_, fy_ = y0 - 1 + ey_;
    eval[k] = i < EPA && fx_ >= 0 && fx_ < p.g.nx && fy_ >= 0 && fy_ < p.g.ny;
    ebase[k] = fy_ + (long long)p.g.ny * fx_;
  }
  auto load_plane = [&](int zp, T (&v)[2][3]) {
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      v[k][0] = v[k][1] = v[k][2] = T(0);
      if (gval[k] && zp >= 0 && zp < NZ) {
        const long long n = gbase[k] + zp * pstride;
        const int f = p.fix[n];
        const T* un = u + 3 * n;
        if (!(f & 1)) v[k][0] = un[0];
        if (!(f & 2)) v[k][1] = un[1];
        if (!(f & 4)) v[k][2] = un[2];
      }
    }
  };
  auto store_plane = [&](int zp, const T (&v)[2][3]) {
    T* dst = su + ((zp + NPL) % NPL) * 3 * PP;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int i = tid + k * nthr;
      if (i < PPA) {
        dst[i] = v[k][0];
        dst[PP + i] = v[k][1];
        dst[2 * PP + i] = v[k][2];
      }
    }
  };
  auto load_slab = [&](int zs, T (&v)[2]) {
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      v[k] = T(0);
      if (eval[k] && zs >= 0 && zs < p.g.nz) v[k] = (T)p.esrc(ebase[k] + zs * sstride);
    }
  };
  auto store_slab = [&](int zs, const T (&v)[2]) {
    T* dst = se + ((zs + NSL) % NSL) * EP;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int i = tid + k * nthr;
      if (i < EPA) dst[i] = v[k];
    }
  };

  // prologue: planes zb-1 .. zb+NZT, slabs zb-1 .. zb+NZT-1
  for (int q = zb - 1; q <= zb + NZT; ++q) {
    T v[2][3];
    load_plane(q, v);
    store_plane(q, v);
  }
  for (int q = zb - 1; q <= zb + NZT - 1; ++q) {
    T v[2];
    load_slab(q, v);
    store_slab(q, v);
  }
  __syncthreads();

  const int toff = (tx + 1) * PY + (ty + 1);
  const int eoff = (tx + 1) * EY + (ty + 1);
  double part = 0.0;
  for (int z = zb; z < ze; z += NZT) {
    // next step's planes z+NZT+1 .. z+2NZT and slabs z+NZT .. z+2NZT-1, in flight during the FMAs
    T pv[NZT][2][3];
    T sv[NZT][2];
#pragma unroll
    for (int j = 0; j < NZT; ++j) {
      load_plane(z + NZT + 1 + j, pv[j]);
      load_slab(z + NZT + j, sv[j]);
    }
    if (active) {
#pragma unroll
      for (int j = 0; j < NZT; ++j) {
        const int zn = z + j;
        if (zn < ze) {
          // epilogue inputs first: their loads overlap the FMAs below
          const long long n = p.g.nidx(x0 + tx, y0 + ty, zn);
          const int f = p.fix[n];
          EpiIn<T> in[3];
#pragma unroll
          for (int c = 0; c < 3; ++c) in[c] = fine_epi_load<T>(p.mode, p.io, 3 * n + c);
          T acc[8][3];
#pragma unroll
          for (int e = 0; e < 8; ++e)
#pragma unroll
            for (int c = 0; c < 3; ++c) acc[e][c] = T(0);
#pragma unroll
          for (int dz = -1; dz <= 1; ++dz) {
            const T* pl = su + ((zn + dz + NPL) % NPL) * 3 * PP + toff;
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
#pragma unroll
              for (int dy = -1; dy <= 1; ++dy) {
                const int off = dx * PY + dy;
                const T um0 = pl[off], um1 = pl[PP + off], um2 = pl[2 * PP + off];
#pragma unroll
                for (int ez = -1; ez <= 0; ++ez)
#pragma unroll
                  for (int ex = -1; ex <= 0; ++ex)
#pragma unroll
                    for (int ey = -1; ey <= 0; ++ey) {
                      const int ox = dx - ex, oy = dy - ey, oz = dz - ez;
                      if (ox < 0 || ox > 1 || oy < 0 || oy > 1 || oz < 0 || oz > 1) continue;
                      const int a = corner_index(-ex, -ey, -ez);
                      const int b = corner_index(ox, oy, oz);
                      const int e8 = (ez + 1) * 4 + (ey + 1) * 2 + (ex + 1);
#pragma unroll
                      for (int c = 0; c < 3; ++c) {
                        T t = acc[e8][c];
                        t = fma(ke_coef<T, CLS>(p.ke, kc, (3 * a + c) * 24 + 3 * b + 0), um0, t);
                        t = fma(ke_coef<T, CLS>(p.ke, kc, (3 * a + c) * 24 + 3 * b + 1), um1, t);
                        t = fma(ke_coef<T, CLS>(p.ke, kc, (3 * a + c) * 24 + 3 * b + 2), um2, t);
                        acc[e8][c] = t;
                      }
                    }
              }
            }
          }
          T kv[3] = {T(0), T(0), T(0)};
#pragma unroll
          for (int ez = -1; ez <= 0; ++ez) {
            const T* sl = se + ((zn + ez + NSL) % NSL) * EP + eoff;
#pragma unroll
            for (int ex = -1; ex <= 0; ++ex)
#pragma unroll
              for (int ey = -1; ey <= 0; ++ey) {
                const T E = sl[ex * EY + ey];
                const int e8 = (ez + 1) * 4 + (ey + 1) * 2 + (ex + 1);
#pragma unroll
                for (int c = 0; c < 3; ++c) kv[c] = fma(E, acc[e8][c], kv[c]);
              }
          }
          const T* own = su + ((zn + NPL) % NPL) * 3 * PP + toff;
#pragma unroll
          for (int c = 0; c < 3; ++c)
            fine_epilogue<T>(p.mode, p.io, 3 * n + c, (f >> c) & 1, kv[c], own[c * PP], in[c], part);
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NZT; ++j) {
      store_plane(z + NZT + 1 + j, pv[j]);
      store_slab(z + NZT + j, sv[j]);
    }
    __syncthreads();
  }
  if (p.mode == kModeCgQ || p.mode == kModeChebStepDot) {
    part = block_sum(part, red);
    if (tid == 0) p.io.partials[blockIdx.y * gridDim.x + blockIdx.x] = part;
    if (p.io.fin_count)
      last_block_finalize(p.io.partials, gridDim.x * gridDim.y, p.io.fin_count, p.io.fin, p.io.fin_op, red);
  }
}

// Compile-time tile heights offered to the tile chooser.
#define TP3D_FINE_TY_LIST(X) X(8) X(13) X(16) X(17) X(24) X(32) X(33) X(43) X(64)

}  // namespace tp3d
