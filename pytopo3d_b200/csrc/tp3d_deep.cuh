// The last smoothed level of the V-cycle and the coarsest solve in one thread
// block, with the level's operator in shared memory.
//
// At the bottom of the hierarchy a level holds a few hundred nodes: each of
// its smoothing steps, its residual, the grid transfers and the coarsest
// matrix-vector product, launched separately, cost a kernel's launch, ramp
// and drain for microseconds of work.  Here one block of 1024 threads runs the
// level's whole cycle with block barriers between the phases: it stages the
// level's packed stencil (bf16 or FP32), the coarsest inverse (when it fits),
// diagonal, masks and vectors in shared memory once (asynchronous 16-byte
// copies, all in flight together), smooths, restricts the residual,
// multiplies by the coarsest inverse, prolongs and smooths again, and writes
// the level's iterate back.  Every phase calls the same per-node device
// functions and epilogues as the separate kernels, with plain loads from
// shared memory.  With a bf16 stencil the block reads it node-major: four
// warps share 32 nodes, warp q of the four reads chunks 8q .. 8q+7 of each
// node's 31 16-byte chunks (kDeepRow entries per node) and computes the
// node's three partial rows, and the four partial sums are added in a fixed
// order after a block barrier.  Rows are summed in partial sums (FP32 stencil:
// one per z-plane of neighbours), so they round differently from the separate
// kernels' single sum.
#pragma once

#include "tp3d_hex.cuh"

namespace tp3d {

constexpr int kDeepThreads = 1024;
constexpr int kDeepRow = 248;  // node-major bf16 stencil: 243 entries (k = (jrel * 3 + c) * 3 + d) + 5 zeros

// The node-major bf16 stencil of a level from its FP64 stencil (fixed rows and
// columns and neighbours past the grid zeroed, as in the packed layout).
__global__ void deep_pack_kernel(Grid g, const double* __restrict__ A, const uint8_t* __restrict__ fix,
                                 __nv_bfloat16* SN) {
  const int NX = g.nx + 1, NY = g.ny + 1, NZ = g.nz + 1;
  const long long nn = g.nnode();
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < nn * kDeepRow;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long n = idx / kDeepRow;
    const int k = (int)(idx - n * kDeepRow);
    double v = 0.0;
    if (k < 243) {
      const int jr = k / 9, c = (k / 3) % 3, d = k % 3;
      const int dz = jr / 9 - 1, dx = (jr / 3) % 3 - 1, dy = jr % 3 - 1;
      const int iy = (int)(n % NY);
      const long long r = n / NY;
      const int ix = (int)(r % NX), iz = (int)(r / NX);
      const int x = ix + dx, y = iy + dy, z = iz + dz;
      const bool in = x >= 0 && x < NX && y >= 0 && y < NY && z >= 0 && z < NZ;
      const int fm = in ? fix[g.nidx(x, y, z)] : 7;
      if (!((fix[n] >> c) & 1) && !((fm >> d) & 1)) v = A[(long long)k * nn + n];
    }
    SN[idx] = __double2bfloat16(v);
  }
}

// Part Q of K u at the three DOFs of node n from its row of the node-major
// bf16 stencil in shared memory: the entries of chunks 8Q .. 8Q+7.
constexpr int kDeepPassNodes = 256;  // nodes per pass of the block: 8 groups of 32, four warps per group

template <typename T, int Q>
__device__ __forceinline__ void deep_node_part(const Grid& g, const uint4* row, const T* u, int n, T y[3]) {
  const int NX = g.nx + 1, NY = g.ny + 1, NZ = g.nz + 1;
  const int NXY = NX * NY;
  const int iy = n % NY, r = n / NY;
  const int ix = r % NX, iz = r / NX;
  const int oy0 = iy > 0 ? -1 : 0, oy2 = iy < NY - 1 ? 1 : 0;
  const int ox0 = ix > 0 ? -NY : 0, ox2 = ix < NX - 1 ? NY : 0;
  const int oz0 = iz > 0 ? -NXY : 0, oz2 = iz < NZ - 1 ? NXY : 0;
  T acc[3][2] = {{T(0), T(0)}, {T(0), T(0)}, {T(0), T(0)}};
#pragma unroll
  for (int q = 8 * Q; q < 8 * Q + 8 && q < kDeepRow / 8; ++q) {
    const uint4 w = row[q];
    const unsigned ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int h = 0; h < 8; ++h) {
      const int k = 8 * q + h;
      if (k < 243) {
        const int jr = k / 9, c = (k / 3) % 3, d = k % 3;
        const int a = jr / 9, bb = (jr / 3) % 3, e = jr % 3;
        const int m = n + (a == 0 ? oz0 : (a == 1 ? 0 : oz2)) + (bb == 0 ? ox0 : (bb == 1 ? 0 : ox2)) +
                      (e == 0 ? oy0 : (e == 1 ? 0 : oy2));
        const unsigned bits = (h & 1) ? (ws[h >> 1] & 0xffff0000u) : (ws[h >> 1] << 16);
        acc[c][jr & 1] = fma((T)__uint_as_float(bits), u[3 * m + d], acc[c][jr & 1]);
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) y[c] = acc[c][0] + acc[c][1];
}

template <typename T, typename TS>
struct DeepParams {
  Grid g{}, gc{};               // the level and the coarsest level
  const TS* S = nullptr;        // the level's stencil: bf16 node-major (kDeepRow per node) or FP32 packed
  const uint8_t* fix = nullptr;   // the level's node masks
  const uint8_t* fixc = nullptr;  // the coarsest level's node masks
  const T* dinv = nullptr;
  const double* coef = nullptr;  // Chebyshev coefficients of the level
  const T* inv = nullptr;        // coarsest inverse, cn x cn row-major
  int cn = 0;
  int inv_smem = 0;              // 1: the inverse is staged in shared memory
  const T* b = nullptr;          // the level's right-hand side
  const T* x0 = nullptr;         // its first smoothing step (written by the restriction)
  const T* d0 = nullptr;         // and that step's Chebyshev direction
  T* xout = nullptr;             // the level's iterate after the cycle
  int pre = 1, post = 1;         // smoothing degrees (pre counts the step already taken)
  int cheb = 1;                  // 1 Chebyshev, 0 damped Jacobi
  T omega = T(0);
  const int* done = nullptr;
};

// Bytes of the level's stencil in the block: node-major bf16 (kDeepRow per
// node) or DOF-major packed (81 per DOF).
template <typename TS>
__host__ __device__ constexpr size_t deep_stencil_bytes(long long nn) {
  return sizeof(TS) == 2 ? (size_t)nn * kDeepRow * 2 : (size_t)(81 * 3 * nn) * sizeof(TS);
}

// Shared-memory bytes of the block for a level of `nn` nodes and a coarsest
// level of `nnc` nodes: stencil, six level vectors (x[2], b, d, dinv, r), two
// coarsest vectors, node masks, the four partial rows of a pass (bf16
// stencil), and with inv_smem the coarsest inverse; 16-byte aligned parts.
template <typename T, typename TS>
__host__ __device__ constexpr size_t deep_smem_bytes(long long nn, long long nnc, bool inv_smem) {
  const size_t nd = (size_t)(3 * nn), ndc = (size_t)(3 * nnc);
  auto al = [](size_t x) { return (x + 15) & ~(size_t)15; };
  return al(deep_stencil_bytes<TS>(nn)) + 6 * al(nd * sizeof(T)) + 2 * al(ndc * sizeof(T)) + al((size_t)nn) +
         al((size_t)nnc) + (sizeof(TS) == 2 ? al(4 * 3 * kDeepPassNodes * sizeof(T)) : 0) +
         (inv_smem ? al(ndc * ndc * sizeof(T)) : 0);
}

// 16-byte asynchronous copies global -> shared of the first (bytes / 16) * 16
// bytes (both addresses 16-byte aligned), the tail by plain byte copies; the
// caller waits with deep_copy_wait().
__device__ __forceinline__ void deep_copy_async(void* dst, const void* src, size_t bytes) {
  const size_t n16 = bytes / 16;
  const unsigned char* s8 = reinterpret_cast<const unsigned char*>(src);
  unsigned char* d8 = reinterpret_cast<unsigned char*>(dst);
  for (size_t k = threadIdx.x; k < n16; k += blockDim.x) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(d8 + 16 * k);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(s8 + 16 * k) : "memory");
  }
  for (size_t k = n16 * 16 + threadIdx.x; k < bytes; k += blockDim.x) d8[k] = s8[k];
}
__device__ __forceinline__ void deep_copy_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// K u at DOF i from shared memory, in three partial sums (neighbours in the
// planes z - 1, z, z + 1).
template <typename T, typename TS>
__device__ __forceinline__ T deep_row(const Grid& g, const TS* S, const T* u, int i) {
  const int NX = g.nx + 1, NY = g.ny + 1, NZ = g.nz + 1;
  const int NXY = NX * NY;
  const int ndof = 3 * NXY * NZ;
  const int n = i / 3;
  const int iy = n % NY, r = n / NY;
  const int ix = r % NX, iz = r / NX;
  const int oy0 = iy > 0 ? -1 : 0, oy2 = iy < NY - 1 ? 1 : 0;
  const int ox0 = ix > 0 ? -NY : 0, ox2 = ix < NX - 1 ? NY : 0;
  const int oz0 = iz > 0 ? -NXY : 0, oz2 = iz < NZ - 1 ? NXY : 0;
  T kv[3] = {T(0), T(0), T(0)};
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
        kv[a] = fma(ld_coef<T, LdPlain>(s), u[m3], kv[a]);
        kv[a] = fma(ld_coef<T, LdPlain>(s + ndof), u[m3 + 1], kv[a]);
        kv[a] = fma(ld_coef<T, LdPlain>(s + 2 * (size_t)ndof), u[m3 + 2], kv[a]);
      }
    }
  }
  return (kv[0] + kv[1]) + kv[2];
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
  constexpr bool kNode = sizeof(TS) == 2;  // bf16: node-major
  TS* S = reinterpret_cast<TS*>(q);
  q += al(deep_stencil_bytes<TS>(nn));
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
  q += al((size_t)nnc);
  T* ypart = reinterpret_cast<T*>(q);  // [4 parts][3 components][kDeepPassNodes]
  if (kNode) q += al(4 * 3 * kDeepPassNodes * sizeof(T));
  T* inv = p.inv_smem ? reinterpret_cast<T*>(q) : nullptr;

  const int t = threadIdx.x;
  // stage the operator and the coarsest inverse (asynchronous copies, all in
  // flight while the level's state is loaded), then the level's state
  deep_copy_async(S, p.S, deep_stencil_bytes<TS>(nn));
  if (inv) deep_copy_async(inv, p.inv, (size_t)p.cn * p.cn * sizeof(T));
  for (int i = t; i < nd; i += kDeepThreads) {
    x[0][i] = p.x0[i];
    d[i] = p.d0 ? p.d0[i] : T(0);
    b[i] = p.b[i];
    dinv[i] = p.dinv[i];
  }
  for (int n = t; n < nn; n += kDeepThreads) fix[n] = p.fix[n];
  for (int n = t; n < nnc; n += kDeepThreads) fixc[n] = p.fixc[n];
  deep_copy_wait();
  __syncthreads();

  // K x[cur] of the nodes of pass `base` into ypart (bf16 stencil); the caller
  // waits at a block barrier before reading it
  auto node_pass = [&](int base, const T* xv) {
    const int w = t >> 5, l = t & 31;
    const int nl = (w >> 2) * 32 + l, qp = w & 3;
    const int n = base + nl;
    T y[3] = {T(0), T(0), T(0)};
    if (n < nn) {
      const uint4* row = reinterpret_cast<const uint4*>(reinterpret_cast<const __nv_bfloat16*>(S) + (size_t)n * kDeepRow);
      if (qp == 0) deep_node_part<T, 0>(p.g, row, xv, n, y);
      else if (qp == 1) deep_node_part<T, 1>(p.g, row, xv, n, y);
      else if (qp == 2) deep_node_part<T, 2>(p.g, row, xv, n, y);
      else deep_node_part<T, 3>(p.g, row, xv, n, y);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) ypart[(qp * 3 + c) * kDeepPassNodes + nl] = y[c];
  };
  auto node_sum = [&](int nl, int c) {
    return ((ypart[(0 * 3 + c) * kDeepPassNodes + nl] + ypart[(1 * 3 + c) * kDeepPassNodes + nl]) +
            ypart[(2 * 3 + c) * kDeepPassNodes + nl]) +
           ypart[(3 * 3 + c) * kDeepPassNodes + nl];
  };

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
    auto epi = [&](int i, int n, int c, T kv) {
      const bool fx = (fix[n] >> c) & 1;
      const T own = fx ? T(0) : x[cur][i];
      if (!p.cheb) op_epilogue<T, kModeJacobi>(io, i, fx, kv, own, epi_load<T, kModeJacobi>(io, i), part);
      else if (first) op_epilogue<T, kModeChebFirst>(io, i, fx, kv, own, epi_load<T, kModeChebFirst>(io, i), part);
      else op_epilogue<T, kModeChebStep>(io, i, fx, kv, own, epi_load<T, kModeChebStep>(io, i), part);
    };
    if constexpr (kNode) {
      for (int base = 0; base < nn; base += kDeepPassNodes) {
        node_pass(base, x[cur]);
        __syncthreads();
        const int cnt = 3 * (int)min((long long)kDeepPassNodes, nn - base);
        for (int k = t; k < cnt; k += kDeepThreads) {
          const int nl = k / 3, c = k - 3 * nl;
          epi(3 * (base + nl) + c, base + nl, c, node_sum(nl, c));
        }
        __syncthreads();
      }
    } else {
      for (int i = t; i < nd; i += kDeepThreads) {
        const int n = i / 3, c = i - 3 * n;
        epi(i, n, c, deep_row<T, TS>(p.g, S, x[cur], i));
      }
    }
    __syncthreads();
    cur ^= 1;
  };

  // pre-smoothing (step 0 was taken by the restriction)
  for (int s = 1; s < p.pre; ++s) smooth(s, false);
  // residual
  if constexpr (kNode) {
    for (int base = 0; base < nn; base += kDeepPassNodes) {
      node_pass(base, x[cur]);
      __syncthreads();
      const int cnt = 3 * (int)min((long long)kDeepPassNodes, nn - base);
      for (int k = t; k < cnt; k += kDeepThreads) {
        const int nl = k / 3, c = k - 3 * nl, n = base + nl;
        r[3 * n + c] = ((fix[n] >> c) & 1) ? T(0) : b[3 * n + c] - node_sum(nl, c);
      }
      __syncthreads();
    }
  } else {
    for (int i = t; i < nd; i += kDeepThreads) {
      const int n = i / 3, c = i - 3 * n;
      const bool fx = (fix[n] >> c) & 1;
      r[i] = fx ? T(0) : b[i] - deep_row<T, TS>(p.g, S, x[cur], i);
    }
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
      const T* row = (inv ? inv : p.inv) + (size_t)i * p.cn;
      for (int j = lane; j < p.cn; j += 32) acc += (double)(inv ? row[j] : __ldg(&row[j])) * (double)bc[j];
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
