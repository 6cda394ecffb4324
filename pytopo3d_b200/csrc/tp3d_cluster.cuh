// The last two smoothed levels of the V-cycle and the coarsest solve as one
// thread-block cluster, each level's operator split over the cluster's CTAs
// in shared memory.
//
// Below a few thousand nodes a level's smoothing steps, residual and grid
// transfers each cost a launch's latency for a microsecond of work, and its
// operator (1377 nodes x 496 bytes of bf16 stencil on the 16x8x8 level) is
// too large for one block's shared memory.  Here a cluster of C CTAs (8, or
// 16 where 8 do not fit) runs levels A and B = A + 1 and the coarsest level
// in one launch.  The nodes of every level are split into C contiguous ranges
// (CTA r owns nodes [r * chunk, (r + 1) * chunk)); each CTA stages the
// node-major bf16 stencil rows of its nodes of A and B and its rows of the
// coarsest inverse in its shared memory once, and keeps a full-length copy of
// each level's iterate of which its own range and a halo of one node plane
// (NX*NY + NY + 1 nodes) either side are current.  A smoothing step writes
// each new value of a CTA's own range into its own copy and, by remote stores
// to distributed shared memory (cluster.map_shared_rank), into the copies of
// the CTAs whose halo holds it; one cluster barrier (arrive.release /
// wait.acquire) then publishes the step, so a step costs one pass, one block
// barrier and one cluster barrier.  Buffers alternate between steps, and a
// CTA writes a neighbour's buffer only after every CTA has passed the barrier
// that ended the last step reading it.  The restrictions and the coarsest
// product read the ranges they need from the owners after a barrier.  The arithmetic per node is that of the one-block deep cycle
// (deep_node_part, the same epilogues as op_epilogue, restrict_node,
// prolong_node), so each level's rows round as they do there.
//
// Every CTA takes every cluster barrier (the control flow depends only on the
// level sizes and smoothing degrees), and every access to another CTA's
// shared memory comes before the last barrier, so no CTA exits while another
// still reads or writes it.  The cluster's CTAs are co-scheduled by the hardware, so the
// barriers need no time limit.
#pragma once

#include <cooperative_groups.h>

#include "tp3d_deep.cuh"

namespace tp3d {

constexpr int kClThreads = 1024;
constexpr int kClPassNodes = 256;  // nodes per pass: 8 groups of 32, four warps per group

// Byte offsets of the cluster cycle's shared-memory parts; the same in every
// CTA, so a part of another CTA is reached through the same local address.
struct ClLayout {
  size_t SA, SB, inv, xA0, xA1, rA, bA, dA, dinvA, xB0, xB1, rB, bB, dB, dinvB, bc, xc, fixA, fixB, fixC, ypart;
  size_t total;
  int chA, chB, chC;  // nodes per CTA on A, B and the coarsest level
};

__host__ __device__ inline ClLayout cl_layout(int nA, int nB, int nC, int C) {
  auto al = [](size_t x) { return (x + 15) & ~(size_t)15; };
  ClLayout L{};
  L.chA = (nA + C - 1) / C;
  L.chB = (nB + C - 1) / C;
  L.chC = (nC + C - 1) / C;
  const size_t f = sizeof(float);
  size_t o = 0;
  L.SA = o;    o += al((size_t)L.chA * kDeepRow * 2);
  L.SB = o;    o += al((size_t)L.chB * kDeepRow * 2);
  L.inv = o;   o += al((size_t)3 * L.chC * 3 * nC * f);  // own rows of the coarsest inverse
  L.xA0 = o;   o += al((size_t)3 * nA * f);              // full length
  L.xA1 = o;   o += al((size_t)3 * nA * f);
  L.rA = o;    o += al((size_t)3 * nA * f);
  L.bA = o;    o += al((size_t)3 * L.chA * f);           // own range
  L.dA = o;    o += al((size_t)3 * L.chA * f);
  L.dinvA = o; o += al((size_t)3 * L.chA * f);
  L.xB0 = o;   o += al((size_t)3 * nB * f);              // full length
  L.xB1 = o;   o += al((size_t)3 * nB * f);
  L.rB = o;    o += al((size_t)3 * nB * f);
  L.bB = o;    o += al((size_t)3 * nB * f);
  L.dB = o;    o += al((size_t)3 * L.chB * f);           // own range
  L.dinvB = o; o += al((size_t)3 * L.chB * f);
  L.bc = o;    o += al((size_t)3 * nC * f);              // full length
  L.xc = o;    o += al((size_t)3 * nC * f);
  L.fixA = o;  o += al((size_t)nA);
  L.fixB = o;  o += al((size_t)nB);
  L.fixC = o;  o += al((size_t)nC);
  L.ypart = o; o += al((size_t)4 * 3 * kClPassNodes * f);
  L.total = o;
  return L;
}

struct ClusterParams {
  Grid gA, gB, gC;                   // levels A, B = A + 1 and the coarsest
  const __nv_bfloat16* SA = nullptr;  // node-major bf16 stencils (kDeepRow per node) of A and B
  const __nv_bfloat16* SB = nullptr;
  const uint8_t* fixA = nullptr;
  const uint8_t* fixB = nullptr;
  const uint8_t* fixC = nullptr;
  const float* dinvA = nullptr;
  const float* dinvB = nullptr;
  const double* coefA = nullptr;  // Chebyshev coefficients
  const double* coefB = nullptr;
  const float* inv = nullptr;  // coarsest inverse, cn x cn row-major
  int cn = 0;
  const float* b = nullptr;   // level A's right-hand side
  const float* x0 = nullptr;  // its first smoothing step (written by the restriction)
  const float* d0 = nullptr;  // and that step's Chebyshev direction
  float* xout = nullptr;      // level A's iterate after the cycle
  int preA = 1, postA = 1, preB = 1, postB = 1;  // smoothing degrees (preA counts the step already taken)
  int cheb = 1;                                   // 1 Chebyshev, 0 damped Jacobi
  float omega = 0.f;
  const int* done = nullptr;
};

// One level's view inside a CTA: its own node range, the shared-memory parts
// and the current iterate buffer.
struct ClLevel {
  Grid g;
  int n, chunk, lo, hi, halo;
  const __nv_bfloat16* S;  // own rows
  float* x;                // current iterate, full length
  float* xn;               // the next one
  float* r;                // full length
  float* b;                // indexed by DOF - boff
  int boff;
  float* d;                // own range
  float* dinv;             // own range
  uint8_t* fix;            // full length
  const double* coef;
};

// K x of the own nodes [base, base + kClPassNodes) of a level whose own rows
// start at S (node lo) into ypart: four warps per 32 nodes, warp q of the four
// the chunks 8q .. 8q+7 of each row.  One copy of the unrolled products serves
// every phase of the cycle (kept out of line so that the kernel's code stays
// small).
__device__ __noinline__ void cl_pass(const Grid g, const __nv_bfloat16* S, int lo, int hi, int base, const float* xv,
                                     float* ypart) {
  const int t = threadIdx.x;
  const int w = t >> 5, l = t & 31;
  const int nl = (w >> 2) * 32 + l, qp = w & 3;
  const int n = base + nl;
  float y[3] = {0.f, 0.f, 0.f};
  if (n < hi) {
    const uint4* row = reinterpret_cast<const uint4*>(S + (size_t)(n - lo) * kDeepRow);
    if (qp == 0) deep_node_part<float, 0>(g, row, xv, n, y);
    else if (qp == 1) deep_node_part<float, 1>(g, row, xv, n, y);
    else if (qp == 2) deep_node_part<float, 2>(g, row, xv, n, y);
    else deep_node_part<float, 3>(g, row, xv, n, y);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) ypart[(qp * 3 + c) * kClPassNodes + nl] = y[c];
}

__global__ void __launch_bounds__(kClThreads, 1) cluster_cycle_kernel(const __grid_constant__ ClusterParams p) {
  namespace cg = cooperative_groups;
  pdl_entry();
  if (p.done && *(volatile const int*)p.done) return;  // the same for every CTA of the cluster
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks(), rk = (int)cl.block_rank();
  const int nA = (int)p.gA.nnode(), nB = (int)p.gB.nnode(), nC = (int)p.gC.nnode();
  const ClLayout Ly = cl_layout(nA, nB, nC, C);
  extern __shared__ __align__(16) unsigned char smem[];
  auto fp = [&](size_t off) { return reinterpret_cast<float*>(smem + off); };
  const int t = threadIdx.x;

  auto make = [&](const Grid& g, int n, int chunk, size_t S, size_t x0, size_t x1, size_t r, size_t b, bool b_own,
                  size_t d, size_t dinv, size_t fix, const double* coef) {
    ClLevel V;
    V.g = g;
    V.n = n;
    V.chunk = chunk;
    V.lo = min(n, rk * chunk);
    V.hi = min(n, (rk + 1) * chunk);
    V.halo = (g.nx + 1) * (g.ny + 1) + (g.ny + 1) + 1;
    V.S = reinterpret_cast<const __nv_bfloat16*>(smem + S);
    V.x = fp(x0);
    V.xn = fp(x1);
    V.r = fp(r);
    V.b = fp(b);
    V.boff = b_own ? 3 * V.lo : 0;
    V.d = fp(d);
    V.dinv = fp(dinv);
    V.fix = smem + fix;
    V.coef = coef;
    return V;
  };
  ClLevel A = make(p.gA, nA, Ly.chA, Ly.SA, Ly.xA0, Ly.xA1, Ly.rA, Ly.bA, true, Ly.dA, Ly.dinvA, Ly.fixA, p.coefA);
  ClLevel B = make(p.gB, nB, Ly.chB, Ly.SB, Ly.xB0, Ly.xB1, Ly.rB, Ly.bB, false, Ly.dB, Ly.dinvB, Ly.fixB, p.coefB);
  const int loC = min(nC, rk * Ly.chC), hiC = min(nC, (rk + 1) * Ly.chC);
  float* inv = fp(Ly.inv);
  float* bc = fp(Ly.bc);
  float* xc = fp(Ly.xc);
  uint8_t* fixC = smem + Ly.fixC;
  float* ypart = fp(Ly.ypart);

  // ---- staging: stencil rows (asynchronous copies), then vectors and masks ----
  deep_copy_async(smem + Ly.SA, p.SA + (size_t)A.lo * kDeepRow, (size_t)(A.hi - A.lo) * kDeepRow * 2);
  deep_copy_async(smem + Ly.SB, p.SB + (size_t)B.lo * kDeepRow, (size_t)(B.hi - B.lo) * kDeepRow * 2);
  {
    const int r0 = 3 * loC, nr = 3 * (hiC - loC);
    for (int k = t; k < nr * p.cn; k += kClThreads) inv[k] = p.inv[(size_t)r0 * p.cn + k];
  }
  // full-length arrays start at zero: the transfers read entries with weight 0
  for (size_t k = t; k < (Ly.bA - Ly.xA0) / sizeof(float); k += kClThreads) fp(Ly.xA0)[k] = 0.f;
  for (size_t k = t; k < (Ly.dB - Ly.xB0) / sizeof(float); k += kClThreads) fp(Ly.xB0)[k] = 0.f;
  for (size_t k = t; k < (Ly.fixA - Ly.bc) / sizeof(float); k += kClThreads) fp(Ly.bc)[k] = 0.f;
  __syncthreads();
  for (int i = 3 * A.lo + t; i < 3 * A.hi; i += kClThreads) {
    const int li = i - 3 * A.lo;
    A.b[li] = p.b[i];
    A.d[li] = p.d0 ? p.d0[i] : 0.f;
    A.dinv[li] = p.dinvA[i];
  }
  for (int i = 3 * max(0, A.lo - A.halo) + t; i < 3 * min(nA, A.hi + A.halo); i += kClThreads) A.x[i] = p.x0[i];
  for (int i = 3 * B.lo + t; i < 3 * B.hi; i += kClThreads) B.dinv[i - 3 * B.lo] = p.dinvB[i];
  for (int n = t; n < nA; n += kClThreads) A.fix[n] = p.fixA[n];
  for (int n = t; n < nB; n += kClThreads) B.fix[n] = p.fixB[n];
  for (int n = t; n < nC; n += kClThreads) fixC[n] = p.fixC[n];
  deep_copy_wait();
  __syncthreads();

  // entries [j0, j1) of a full-length array, from the CTAs that own them
  auto pull = [&](float* a, int j0, int j1, int chunk) {
    for (int j = j0 + t; j < j1; j += kClThreads) {
      const int owner = (j / 3) / chunk;
      if (owner != rk) a[j] = *cl.map_shared_rank(a + j, (unsigned)owner);
    }
  };
  // value v of own DOF i (node n) of V into buf[i] of every other CTA whose
  // halo holds node n (remote stores; the next cluster barrier publishes them)
  auto push = [&](const ClLevel& V, float* buf, int n, int i, float v) {
    const int r0 = n - V.halo < 0 ? 0 : (n - V.halo) / V.chunk;
    const int r1 = min(C - 1, (n + V.halo) / V.chunk);
    for (int r = r0; r <= r1; ++r)
      if (r != rk) *cl.map_shared_rank(buf + i, (unsigned)r) = v;
  };
  auto pass = [&](const ClLevel& V, int base, const float* xv) { cl_pass(V.g, V.S, V.lo, V.hi, base, xv, ypart); };
  auto psum = [&](int nl, int c) {
    return ((ypart[(0 * 3 + c) * kClPassNodes + nl] + ypart[(1 * 3 + c) * kClPassNodes + nl]) +
            ypart[(2 * 3 + c) * kClPassNodes + nl]) +
           ypart[(3 * 3 + c) * kClPassNodes + nl];
  };
  // one smoothing step on V's own nodes (first: the Chebyshev first step), each
  // new value also stored into the neighbours' halos; the cluster barrier at
  // the end publishes them
  auto smooth = [&](ClLevel& V, int s, bool first) {
    for (int base = V.lo; base < V.hi; base += kClPassNodes) {
      pass(V, base, V.x);
      __syncthreads();
      const int cnt = 3 * min(kClPassNodes, V.hi - base);
      for (int k = t; k < cnt; k += kClThreads) {
        const int nl = k / 3, c = k - 3 * nl, n = base + nl, i = 3 * n + c, li = i - 3 * V.lo;
        const float kv = psum(nl, c);
        const bool fx = (V.fix[n] >> c) & 1;
        const float own = fx ? 0.f : V.x[i];
        const float bb = V.b[i - V.boff], di = V.dinv[li];
        float out;
        if (!p.cheb) {
          out = fx ? 0.f : own + p.omega * di * (bb - kv);
        } else {
          const float dd = fx ? 0.f
                              : (first ? (float)V.coef[0] * di * (bb - kv)
                                       : (float)V.coef[2 * s] * V.d[li] + (float)V.coef[2 * s + 1] * di * (bb - kv));
          V.d[li] = dd;
          out = own + dd;
        }
        V.xn[i] = out;
        push(V, V.xn, n, i, out);
      }
      if (base + kClPassNodes < V.hi) __syncthreads();
    }
    cl.sync();
    float* tmp = V.x;
    V.x = V.xn;
    V.xn = tmp;
  };
  // residual of V's own DOFs into V.r, then the cluster barrier
  auto residual = [&](ClLevel& V) {
    for (int base = V.lo; base < V.hi; base += kClPassNodes) {
      pass(V, base, V.x);
      __syncthreads();
      const int cnt = 3 * min(kClPassNodes, V.hi - base);
      for (int k = t; k < cnt; k += kClThreads) {
        const int nl = k / 3, c = k - 3 * nl, n = base + nl, i = 3 * n + c;
        V.r[i] = ((V.fix[n] >> c) & 1) ? 0.f : V.b[i - V.boff] - psum(nl, c);
      }
      if (base + kClPassNodes < V.hi) __syncthreads();
    }
    cl.sync();
  };
  // fine node range read by the restriction to coarse nodes [c0, c1)
  auto fine_range = [&](const Grid& gf, const Grid& gc, int c0, int c1, int nf, int* f0, int* f1) {
    const int FX = gf.nx + 1, FY = gf.ny + 1, CX = gc.nx + 1, CY = gc.ny + 1;
    const int H = FX * FY + FY + 1;
    auto f = [&](int c) {
      const int Iy = c % CY, r = c / CY;
      return 2 * Iy + FY * (2 * (r % CX) + FX * 2 * (r / CX));
    };
    *f0 = c1 > c0 ? max(0, f(c0) - H) : 0;
    *f1 = c1 > c0 ? min(nf, f(c1 - 1) + H + 1) : 0;
  };
  // coarse node range read by the prolongation to fine nodes [n0, n1): the
  // coarse z-planes iz / 2 and iz / 2 + 1 of every fine plane iz in the range
  // (the coarse base index of a fine node is not monotone in the node index,
  // so the range is taken by whole planes)
  auto coarse_range = [&](const Grid& gf, const Grid& gc, int n0, int n1, int nc, int* c0, int* c1) {
    const int FXY = (gf.nx + 1) * (gf.ny + 1), CXY = (gc.nx + 1) * (gc.ny + 1);
    *c0 = n1 > n0 ? CXY * ((n0 / FXY) >> 1) : 0;
    *c1 = n1 > n0 ? min(nc, CXY * (((n1 - 1) / FXY >> 1) + 2)) : 0;
  };
  auto node_xyz = [](const Grid& g, int n, int* x, int* y, int* z) {
    const int NY = g.ny + 1, NX = g.nx + 1;
    *y = n % NY;
    const int r = n / NY;
    *x = r % NX;
    *z = r / NX;
  };

  // ---- level A: pre-smoothing (step 0 was taken by the restriction) ----
  for (int s = 1; s < p.preA; ++s) smooth(A, s, false);
  residual(A);
  // ---- restriction A -> B, with B's first smoothing step ----
  {
    int f0, f1;
    fine_range(p.gA, p.gB, B.lo, B.hi, nA, &f0, &f1);
    pull(A.r, 3 * f0, 3 * f1, A.chunk);
    __syncthreads();
    for (int n = B.lo + t; n < B.hi; n += kClThreads) {
      int x, y, z;
      node_xyz(p.gB, n, &x, &y, &z);
      restrict_node<float, LdPlain>(p.gA, p.gB, A.r, B.fix, B.b, x, y, z);
    }
    __syncthreads();
    const float w = p.cheb ? (float)B.coef[0] : p.omega;
    for (int i = 3 * B.lo + t; i < 3 * B.hi; i += kClThreads) {
      const int li = i - 3 * B.lo;
      const float v = w * B.dinv[li] * B.b[i];
      B.x[i] = v;
      push(B, B.x, i / 3, i, v);
      if (p.cheb) B.d[li] = v;
    }
    cl.sync();
  }
  // ---- level B: pre-smoothing, residual ----
  for (int s = 1; s < p.preB; ++s) smooth(B, s, false);
  residual(B);
  // ---- restriction B -> coarsest, coarsest product, prolongation ----
  {
    int f0, f1;
    fine_range(p.gB, p.gC, loC, hiC, nB, &f0, &f1);
    pull(B.r, 3 * f0, 3 * f1, B.chunk);
    __syncthreads();
    for (int n = loC + t; n < hiC; n += kClThreads) {
      int x, y, z;
      node_xyz(p.gC, n, &x, &y, &z);
      restrict_node<float, LdPlain>(p.gB, p.gC, B.r, fixC, bc, x, y, z);
    }
    cl.sync();
    pull(bc, 0, p.cn, Ly.chC);
    __syncthreads();
    // own rows of xc = Inv bc, a warp per row (FP64 accumulation)
    const int warp = t >> 5, lane = t & 31;
    for (int i = 3 * loC + warp; i < 3 * hiC; i += kClThreads / 32) {
      double acc = 0.0;
      const float* row = inv + (size_t)(i - 3 * loC) * p.cn;
      for (int j = lane; j < p.cn; j += 32) acc += (double)row[j] * (double)bc[j];
      acc = warp_sum(acc);
      if (lane == 0) xc[i] = (float)acc;
    }
    cl.sync();
    int c0, c1;
    coarse_range(p.gB, p.gC, B.lo, B.hi, nC, &c0, &c1);
    pull(xc, 3 * c0, 3 * c1, Ly.chC);
    __syncthreads();
    for (int n = B.lo + t; n < B.hi; n += kClThreads) {
      int x, y, z;
      node_xyz(p.gB, n, &x, &y, &z);
      prolong_node<float, LdPlain>(p.gB, p.gC, xc, B.fix, B.x, x, y, z);
#pragma unroll
      for (int c = 0; c < 3; ++c) push(B, B.x, n, 3 * n + c, B.x[3 * n + c]);
    }
    cl.sync();
  }
  // ---- level B: post-smoothing ----
  for (int s = 0; s < p.postB; ++s) smooth(B, s, s == 0);
  // ---- prolongation B -> A ----
  {
    int c0, c1;
    coarse_range(p.gA, p.gB, A.lo, A.hi, nB, &c0, &c1);
    pull(B.x, 3 * c0, 3 * c1, B.chunk);
    __syncthreads();
    for (int n = A.lo + t; n < A.hi; n += kClThreads) {
      int x, y, z;
      node_xyz(p.gA, n, &x, &y, &z);
      prolong_node<float, LdPlain>(p.gA, p.gB, B.x, A.fix, A.x, x, y, z);
#pragma unroll
      for (int c = 0; c < 3; ++c) push(A, A.x, n, 3 * n + c, A.x[3 * n + c]);
    }
    cl.sync();
  }
  // ---- level A: post-smoothing, result ----
  for (int s = 0; s < p.postA; ++s) smooth(A, s, s == 0);
  // every access to another CTA's shared memory came before the last cluster
  // barrier, so the CTAs may leave independently
  for (int i = 3 * A.lo + t; i < 3 * A.hi; i += kClThreads) p.xout[i] = A.x[i];
}

}  // namespace tp3d
