// State of one preconditioned CG run and the scalar steps between its vector
// kernels ("finalize" ops: alpha, beta, stop tests, reliable-update decisions).
// Every scalar lives in device memory so that one iteration can be captured
// into a CUDA graph.  A reduction kernel either writes per-block partials for
// finalize_kernel, or finishes the reduction itself: its last block to arrive
// (last_block_finalize) sums the partials in a fixed order and applies the op,
// which saves a launch per reduction.
#pragma once

#include "tp3d_common.cuh"

namespace tp3d {

struct PcgState {
  double rz, pq, rr, bb, alpha, beta, tol2, rmax2;
  double delta2;   // reliable-update threshold (squared)
  double rr_hi;    // last FP64 residual norm^2
  double rr_best;  // smallest FP64 residual norm^2 so far
  // done: 0 running, 1 converged, 2 iteration cap, 3 breakdown, 4 non-finite,
  //       5 FP64 residual stalled at its attainable floor (accepted),
  //       6 FP64 residual stalled far above the target (mixed: fall back to FP64)
  int done;
  int iters, max_iters;
  int update;   // mixed precision: replace the residual this iteration
  int updates;  // count of reliable updates
  int stall;    // consecutive reliable updates that did not halve the FP64 residual
  int restart;  // mixed precision: FP32 p'Ap <= 0, restart the direction from z
  int nbreak;   // consecutive restarts
};

enum FinalizeOp : int {
  kFinBB = 0,    // bb = ||b||^2, tol2 = rtol^2 bb
  kFinRRInit,    // rr = ||r0||^2 (stop if already converged)
  kFinRZInit,    // rz = r.z
  kFinPQ,        // alpha = rz / p.q
  kFinRR,        // rr = ||r||^2, iteration count, stop test
  kFinRZ,        // beta = rz_new / rz
  kFinRRMixed,   // FP32 recursive residual: decide on a reliable update
  kFinRRHi,      // FP64 true residual after a reliable update: stop test
  kFinValue,     // plain sum into *out (no state change)
  kFinPQMixed,   // as kFinPQ, but a non-positive FP32 p'Ap restarts the direction
  kFinRZMixed,   // as kFinRZ, honouring a pending restart (beta = 0)
};

// True when the op must not run (the solve has stopped, or a reliable-update
// op without a pending update).  The kernels feeding an op skip on the same
// condition, so either every block of a reduction runs or none does.
__device__ __forceinline__ bool finalize_skipped(const PcgState* st, int op) {
  if (((op >= kFinPQ && op <= kFinRRMixed) || op >= kFinPQMixed) && *(volatile const int*)&st->done) return true;
  if (op == kFinRRHi && (*(volatile const int*)&st->done || *(volatile const int*)&st->update == 0)) return true;
  return false;
}

// The op on the reduced value s (one thread).
__device__ inline void finalize_apply(double s, PcgState* st, int op, double rtol2, double* out) {
  switch (op) {
    case kFinBB:
      st->bb = s;
      st->tol2 = rtol2 * s;
      st->iters = 0;
      st->update = 0;
      st->updates = 0;
      st->done = (s == 0.0) ? 1 : 0;
      if (!isfinite(s)) st->done = 4;
      break;
    case kFinRRInit:
      st->rr = s;
      st->rmax2 = s;
      st->rr_hi = s;
      st->rr_best = s;
      st->stall = 0;
      if (!st->done && s <= st->tol2) st->done = 1;
      if (!isfinite(s)) st->done = 4;
      break;
    case kFinRZInit:
      st->rz = s;
      break;
    case kFinPQ:
      st->pq = s;
      if (!(s > 0.0) || !isfinite(s)) st->done = 3;
      else st->alpha = st->rz / s;
      break;
    case kFinRR:
      st->rr = s;
      st->iters += 1;
      if (!isfinite(s)) st->done = 4;
      else if (s <= st->tol2) st->done = 1;
      else if (st->iters >= st->max_iters) st->done = 2;
      break;
    case kFinRZ:
      st->beta = s / st->rz;
      st->rz = s;
      break;
    case kFinRRMixed:
      st->rr = s;
      st->iters += 1;
      if (!isfinite(s)) {
        st->done = 4;
      } else {
        st->update = (st->restart || s <= st->delta2 * st->rmax2 || s <= st->tol2 || st->iters >= st->max_iters)
                         ? 1
                         : 0;
      }
      break;
    case kFinRRHi:
      st->rr_hi = s;
      st->rmax2 = s;
      st->updates += 1;
      if (!isfinite(s)) {
        st->done = 4;
      } else if (s <= st->tol2) {
        st->done = 1;
      } else {
        st->stall = (s > 0.25 * st->rr_best) ? st->stall + 1 : 0;
        st->rr_best = fmin(st->rr_best, s);
        // a stall is an attainable floor only once the residual is small; a stall
        // above 1e-6 relative is a failure (the host then falls back to FP64)
        if (st->stall >= 3) st->done = (s <= 1e-12 * st->bb) ? 5 : 6;
        else if (st->iters >= st->max_iters) st->done = 2;
      }
      break;
    case kFinValue:
      *out = s;
      break;
    case kFinPQMixed:
      // FP32 rounding next to 1e-9 voids can make p'Ap non-positive although K
      // is SPD: skip the step (alpha = 0), force a reliable update and restart
      // the direction from the new preconditioned residual.
      st->pq = s;
      if (!isfinite(s)) {
        st->done = 4;
      } else if (!(s > 0.0)) {
        st->alpha = 0.0;
        st->restart = 1;
        if (++st->nbreak > 5) st->done = 3;
      } else {
        st->alpha = st->rz / s;
      }
      break;
    case kFinRZMixed:
      if (st->restart) {
        st->beta = 0.0;
        st->restart = 0;
      } else {
        st->beta = s / st->rz;
        st->nbreak = 0;
      }
      st->rz = s;
      break;
  }
}

// Called by every thread of every block after the block wrote
// partials[block]; the last block to arrive sums all partials and applies op.
// `count` is zero between reductions (the last block resets it).
__device__ __forceinline__ void last_block_finalize(const double* partials, int nblocks, unsigned int* count,
                                                    PcgState* st, int op, double* red) {
  __shared__ int s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(count, 1u) == (unsigned int)nblocks - 1u;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double v = 0.0;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x) v += __ldcg(&partials[i]);
  const double s = block_sum(v, red);
  if (threadIdx.x == 0) {
    finalize_apply(s, st, op, 0.0, nullptr);
    *count = 0u;
  }
}

}  // namespace tp3d
