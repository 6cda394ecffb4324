// Optimality-criteria update with projected-volume bisection, one cooperative launch.
// Reference: pytopo3d/utils/oc_update.py:25-124 and the change measure of
// pytopo3d/core/optimizer.py:642.
//
// The reference re-filters and re-projects a candidate design for every
// bisection step and syncs the volume to the host.  Here the whole loop runs
// in one persistent kernel: every block owns a set of filter tiles, stages the
// candidate x(lambda) of its tiles (+ halo) in shared memory, filters,
// projects and sums the free volume; per-block partials are combined in a
// fixed order after a (bounded) grid barrier, so every block takes the same
// bisection decision.  Only the best multiplier is kept; the best candidate is
// recomputed from it at the end, so no candidate array is stored.
#include <cfloat>
#include <cmath>

#include "tp3d_filter.cuh"

namespace tp3d {
namespace {

constexpr int kOcMaxBlocks = 4096;

struct OcArgs {
  Grid g;
  FilterCols fc;
  const double* x;
  const double* dc;
  const double* dv;
  const double* Hs;
  const uint8_t* solid;
  const uint8_t* vd;
  double move, target, tol;
  int max_iter;
  Projection pr;
  double* x_new;
  double* rho_new;
  double* stats;
  double* ratio;     // nele
  double* partA;     // kOcMaxBlocks
  double* partB;     // kOcMaxBlocks
  double* partC;     // kOcMaxBlocks
  GridBarrier bar;
};

__device__ __forceinline__ bool is_free(const OcArgs& a, long long e) {
  return !((a.solid && a.solid[e]) || (a.vd && a.vd[e]));
}

// Candidate value (oc_update.py:76-91): free elements move toward
// x sqrt(ratio / lambda) within the move limit; protected ones are clamped.
__device__ __forceinline__ double candidate(const OcArgs& a, long long e, double lam) {
  const bool so = a.solid && a.solid[e], vo = a.vd && a.vd[e];
  const double xe = __ldg(&a.x[e]);
  double v = xe;
  if (!so && !vo) {
    const double r = fmax(__ldg(&a.ratio[e]) / (lam + 1e-30), 1e-30);
    double c = xe * sqrt(r);
    c = fmax(xe - a.move, fmin(xe + a.move, c));
    v = fmin(fmax(c, 0.0), 1.0);
  }
  if (so) v = 1.0;
  if (vo) v = 0.0;
  return v;
}

template <int Z>
__global__ void __launch_bounds__(kFilterThreads) oc_kernel(OcArgs a) {
  extern __shared__ double s[];
  __shared__ double red[32];
  const long long ntiles = filter_ntiles(a.g);
  const long long nele = a.g.nele();
  const int nblk = gridDim.x;

  // ---- ratio normalisation (oc_update.py:54-68) ----
  double m = 0.0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nele; e += (long long)nblk * blockDim.x) {
    if (is_free(a, e)) {
      const double r = fmax(-__ldg(&a.dc[e]) / fmax(__ldg(&a.dv[e]), 1e-20), 0.0);
      a.ratio[e] = r;
      m = fmax(m, r);
    }
  }
  m = block_max(m, red);
  if (threadIdx.x == 0) a.partC[blockIdx.x] = m;
  if (!grid_sync(a.bar)) return;
  double scale = 0.0;
  {
    double t = 0.0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) t = fmax(t, a.partC[i]);
    scale = block_max(t, red);
  }
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nele; e += (long long)nblk * blockDim.x) {
    if (is_free(a, e)) a.ratio[e] = scale > 0.0 ? a.ratio[e] / scale : 1.0;
  }
  if (!grid_sync(a.bar)) return;

  // ---- bisection (oc_update.py:70-122) ----
  double lo = 0.0, hi = 1.0e12;
  double best_err = INFINITY, best_lam = NAN, best_vol = NAN;
  int it = 0;
  for (; it < a.max_iter; ++it) {
    const double lam = 0.5 * (lo + hi);
    double vpart = 0.0;
    for (long long t = blockIdx.x; t < ntiles; t += nblk) {
      const FilterTile tile = filter_tile_at(a.g, t);
      __syncthreads();
      filter_stage<Z>(a.g, tile, s, [&](long long e, int, int, int) { return candidate(a, e, lam); });
      __syncthreads();
      filter_apply<Z>(a.g, a.fc, tile, s, [&](long long e, int, int, int, double v) {
        if (is_free(a, e)) vpart += a.pr.value(v / __ldg(&a.Hs[e]), nullptr);
      });
    }
    vpart = block_sum(vpart, red);
    double* part = (it & 1) ? a.partB : a.partA;
    if (threadIdx.x == 0) part[blockIdx.x] = vpart;
    if (!grid_sync(a.bar)) return;
    const double vol = sum_partials(part, nblk, red);
    const double err = fabs(vol - a.target);
    if (err < best_err) {
      best_err = err;
      best_lam = lam;
      best_vol = vol;
    }
    if (vol > a.target) lo = lam;
    else hi = lam;
    if ((hi - lo) / fmax(hi + lo, DBL_MIN) < a.tol) {
      ++it;
      break;
    }
  }

  // ---- best candidate, its density, and change (optimizer.py:642) ----
  const bool have = !isnan(best_lam);
  double cmax = 0.0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nele; e += (long long)nblk * blockDim.x) {
    const double v = have ? candidate(a, e, best_lam) : __ldg(&a.x[e]);
    a.x_new[e] = v;
    if (is_free(a, e)) cmax = fmax(cmax, fabs(v - __ldg(&a.x[e])));
  }
  cmax = block_max(cmax, red);
  if (threadIdx.x == 0) a.partC[blockIdx.x] = cmax;
  if (!grid_sync(a.bar)) return;
  for (long long t = blockIdx.x; t < ntiles; t += nblk) {
    const FilterTile tile = filter_tile_at(a.g, t);
    __syncthreads();
    filter_stage<Z>(a.g, tile, s, [&](long long e, int, int, int) { return a.x_new[e]; });
    __syncthreads();
    filter_apply<Z>(a.g, a.fc, tile, s, [&](long long e, int, int, int, double v) {
      double r = a.pr.value(v / __ldg(&a.Hs[e]), nullptr);
      if (a.solid && a.solid[e]) r = 1.0;
      if (a.vd && a.vd[e]) r = 0.0;
      a.rho_new[e] = r;
    });
  }
  if (blockIdx.x == 0) {
    double t = 0.0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) t = fmax(t, a.partC[i]);
    t = block_max(t, red);
    if (threadIdx.x == 0) {
      a.stats[0] = best_lam;
      a.stats[1] = best_vol;
      a.stats[2] = (double)it;
      a.stats[3] = t;
      a.stats[4] = scale;
      a.stats[5] = lo;
      a.stats[6] = hi;
      a.stats[7] = have ? best_err : NAN;
    }
  }
}

}  // namespace
}  // namespace tp3d

using namespace tp3d;

extern "C" size_t tp3d_oc_scratch_bytes(int nelx, int nely, int nelz, double rmin) {
  (void)rmin;
  const long long n = (long long)nelx * nely * nelz;
  return (size_t)(n + 3 * kOcMaxBlocks) * sizeof(double) + 256;
}

extern "C" int tp3d_oc_update(int nelx, int nely, int nelz, double rmin, const double* x, const double* dc_dx,
                              const double* dv_dx, const double* Hs, const uint8_t* solid, const uint8_t* void_,
                              double move, double target_free_volume, double beta, double eta,
                              int max_bisection, double bisection_tol, double* x_new, double* rho_new,
                              double* stats, void* scratch, void* stream) {
  if (nelx < 1 || nely < 1 || nelz < 1 || !x || !dc_dx || !dv_dx || !Hs || !x_new || !rho_new || !stats ||
      !scratch)
    return TP3D_ERR_ARG;
  if (!std::isfinite(move) || move <= 0.0) {
    tp3d_set_last_error("move must be positive");
    return TP3D_ERR_ARG;
  }
  if (max_bisection < 1) {
    tp3d_set_last_error("max_bisection_iterations must be at least 1");
    return TP3D_ERR_ARG;
  }
  if (!std::isfinite(beta) || beta <= 0.0 || !(eta > 0.0 && eta < 1.0)) {
    tp3d_set_last_error("invalid projection parameters");
    return TP3D_ERR_ARG;
  }
  FilterCols fc;
  if (int rc = filter_cols_for(rmin, &fc)) return rc;
  const Grid g{nelx, nely, nelz};
  const long long n = g.nele();
  cudaStream_t st = (cudaStream_t)stream;

  OcArgs a{g, fc, x, dc_dx, dv_dx, Hs, solid, void_, move, target_free_volume, bisection_tol,
           max_bisection, Projection(beta, eta), x_new, rho_new, stats};
  double* base = (double*)scratch;
  a.ratio = base;
  a.partA = base + n;
  a.partB = a.partA + kOcMaxBlocks;
  a.partC = a.partB + kOcMaxBlocks;
  unsigned int* bar = (unsigned int*)(a.partC + kOcMaxBlocks);
  a.bar.count = bar;
  a.bar.gen = bar + 1;
  a.bar.err = (int*)(bar + 2);
  TP3D_CHECK(cudaMemsetAsync(bar, 0, 4 * sizeof(unsigned int), st));
  // NaN stats mark a launch that did not finish (e.g. an expired barrier wait)
  TP3D_CHECK(cudaMemsetAsync(stats, 0xff, 8 * sizeof(double), st));

  int dev = 0, nsm = 0;
  TP3D_CHECK(cudaGetDevice(&dev));
  TP3D_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const size_t smem = (size_t)filter_smem_elems(fc.Z) * sizeof(double);
  const long long ntiles = filter_ntiles(g);
  TP3D_DISPATCH_Z(fc.Z, {
    auto kern = oc_kernel<ZC>;
    TP3D_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    TP3D_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kFilterThreads, smem));
    if (per_sm < 1) {
      tp3d_set_last_error("OC kernel does not fit on an SM");
      return TP3D_ERR_CUDA;
    }
    long long grid = std::min<long long>((long long)per_sm * nsm, ntiles);
    grid = std::min<long long>(grid, kOcMaxBlocks);
    void* args[] = {&a};
    TP3D_CHECK(cudaLaunchCooperativeKernel((const void*)kern, dim3((unsigned)grid), dim3(kFilterThreads), args,
                                           smem, st));
  });
  add_launches(1);
  return TP3D_OK;
}
