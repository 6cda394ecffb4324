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
#include <mutex>
#include <vector>

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

// Per-element code written once per call into the ratio scratch: for a free
// element q = sqrt(normalised ratio) >= 0; -1 marks protected solid, -2
// protected void (void wins where both are set, as in the reference).
constexpr double kCodeSolid = -1.0, kCodeVoid = -2.0;

// Candidate value (oc_update.py:76-91): x sqrt(max(r / (lam + 1e-30), 1e-30))
// = x max(q / sqrt(lam + 1e-30), 1e-15), then the move limit and [0, 1].
// `isl` = 1 / sqrt(lam + 1e-30), uniform over the launch.
__device__ __forceinline__ double candidate_q(double xe, double q, double isl, double move) {
  if (q < 0.0) return q == kCodeSolid ? 1.0 : 0.0;
  double c = xe * fmax(q * isl, 1e-15);
  c = fmax(xe - move, fmin(xe + move, c));
  return fmin(fmax(c, 0.0), 1.0);
}

// Projected free volume of the candidate at multiplier lam (oc_update.py:78-111):
// stage candidates of each owned tile (+ halo), filter, project, sum; per-block
// partials go to `part`, and after the grid barrier every block sums them in the
// same order.  Returns false if the barrier wait expired.  (Arrays written
// earlier in this launch are read through L2, __ldcg, never the L1 path.)
template <int Z>
__device__ bool oc_volume(const OcArgs& a, double lam, double* part, double* s, double* red, double* vol) {
  constexpr int SY = kFilterTY + 2 * Z, SX = kFilterTX + 2 * Z, SZ = kFilterKZ + 2 * Z;
  constexpr int NS = SY * SX * SZ;
  const long long ntiles = filter_ntiles(a.g);
  const double isl = 1.0 / sqrt(lam + 1e-30);
  double vpart = 0.0;
  for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const FilterTile tile = filter_tile_at(a.g, t);
    __syncthreads();
#pragma unroll 4
    for (int i = threadIdx.x; i < NS; i += kFilterThreads) {
      const int ly = i % SY, r = i / SY;
      const int lx = r % SX, lz = r / SX;
      const int gx = tile.x0 + lx - Z, gy = tile.y0 + ly - Z, gz = tile.z0 + lz - Z;
      double v = 0.0;
      if (gx >= 0 && gx < a.g.nx && gy >= 0 && gy < a.g.ny && gz >= 0 && gz < a.g.nz) {
        const long long e = a.g.eidx(gx, gy, gz);
        v = candidate_q(__ldg(&a.x[e]), __ldcg(&a.ratio[e]), isl, a.move);
      }
      s[i] = v;
    }
    __syncthreads();
    filter_apply<Z>(a.g, a.fc, tile, s, [&](long long e, int, int, int, double v) {
      if (__ldcg(&a.ratio[e]) >= 0.0) vpart += a.pr.value(v / __ldg(&a.Hs[e]), nullptr);
    });
  }
  vpart = block_sum(vpart, red);
  if (threadIdx.x == 0) part[blockIdx.x] = vpart;
  if (!grid_sync_flip(a.bar.count, a.bar.err)) return false;
  *vol = sum_partials(part, gridDim.x, red);
  return true;
}

template <int Z>
__global__ void __launch_bounds__(kFilterThreads) oc_kernel(OcArgs a) {
  extern __shared__ double s[];
  filter_cols_to_smem<Z>(a.fc, s);  // read back after the first barrier
  __shared__ double red[32];
  const long long ntiles = filter_ntiles(a.g);
  const long long nele = a.g.nele();
  const int nblk = gridDim.x;
  auto solid_at = [&](long long e) { return a.solid && a.solid[e]; };
  auto void_at = [&](long long e) { return a.vd && a.vd[e]; };

  // ---- ratio normalisation (oc_update.py:54-68) ----
  double m = 0.0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nele; e += (long long)nblk * blockDim.x) {
    if (!solid_at(e) && !void_at(e)) {
      const double r = fmax(-__ldg(&a.dc[e]) / fmax(__ldg(&a.dv[e]), 1e-20), 0.0);
      a.ratio[e] = r;
      m = fmax(m, r);
    }
  }
  m = block_max(m, red);
  if (threadIdx.x == 0) a.partC[blockIdx.x] = m;
  if (!grid_sync_flip(a.bar.count, a.bar.err)) return;
  double scale = 0.0;
  {
    double t = 0.0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) t = fmax(t, a.partC[i]);
    scale = block_max(t, red);
  }
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nele; e += (long long)nblk * blockDim.x) {
    double q;
    if (void_at(e)) q = kCodeVoid;
    else if (solid_at(e)) q = kCodeSolid;
    else q = sqrt(scale > 0.0 ? a.ratio[e] / scale : 1.0);
    a.ratio[e] = q;
  }
  if (!grid_sync_flip(a.bar.count, a.bar.err)) return;

  // ---- bisection (oc_update.py:70-122) ----
  // The reference starts from [0, 1e12]; while the projected volume stays at or
  // below the target it only halves the upper bound, so its first midpoints are
  // 1e12 / 2^j, j = 1, 2, ...  The volume does not increase with the
  // multiplier, so the number K of such steps is found by a binary search over
  // j, and steps 1..K need no evaluation of their own: the smallest volume
  // error among them is that of step K (volume closest to the target from
  // below).  Steps K + 1 onwards are the reference's ordinary bisection.  (A
  // tolerance of 1 or more would end the reference's loop after one step; the
  // search is skipped then.)
  double lo = 0.0, hi = 1.0e12;
  double best_err = INFINITY, best_lam = NAN, best_vol = NAN;
  int it = 0, pass = 0;
  bool done = false;
  auto record = [&](double lam, double vol) {
    const double err = fabs(vol - a.target);
    if (err < best_err) {
      best_err = err;
      best_lam = lam;
      best_vol = vol;
    }
    if (vol > a.target) lo = lam;
    else hi = lam;
    ++it;
    if ((hi - lo) / fmax(hi + lo, DBL_MIN) < a.tol) done = true;
  };
  if (a.tol < 1.0) {
    int jlo = 0, jhi = a.max_iter + 1;
    double vlo = NAN, vhi = NAN;
    bool first = true;  // probe j = 1 first: it is the reference's own first step, and K = 0 is common
    while (jhi - jlo > 1) {
      const int jm = first ? 1 : (jlo + jhi) >> 1;
      first = false;
      double v;
      if (!oc_volume<Z>(a, ldexp(1.0e12, -jm), (pass++ & 1) ? a.partB : a.partA, s, red, &v)) return;
      if (v > a.target) {
        jhi = jm;
        vhi = v;
      } else {
        jlo = jm;
        vlo = v;
      }
    }
    if (jlo >= 1) {  // steps 1..jlo: only the best of them (step jlo) is recorded
      it = jlo - 1;
      hi = ldexp(1.0e12, -(jlo - 1));
      record(ldexp(1.0e12, -jlo), vlo);
    }
    if (jhi <= a.max_iter && !done) record(ldexp(1.0e12, -jhi), vhi);  // = 0.5 (lo + hi)
  }
  while (!done && it < a.max_iter) {
    const double lam = 0.5 * (lo + hi);
    double vol;
    if (!oc_volume<Z>(a, lam, (pass++ & 1) ? a.partB : a.partA, s, red, &vol)) return;
    record(lam, vol);
  }

  // ---- best candidate, its density, and change (optimizer.py:642) ----
  const bool have = !isnan(best_lam);
  const double isl = have ? 1.0 / sqrt(best_lam + 1e-30) : 0.0;
  double cmax = 0.0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nele; e += (long long)nblk * blockDim.x) {
    const double xe = __ldg(&a.x[e]), q = a.ratio[e];
    const double v = have ? candidate_q(xe, q, isl, a.move) : xe;
    a.x_new[e] = v;
    if (q >= 0.0) cmax = fmax(cmax, fabs(v - xe));
  }
  cmax = block_max(cmax, red);
  if (threadIdx.x == 0) a.partC[blockIdx.x] = cmax;
  if (!grid_sync_flip(a.bar.count, a.bar.err)) return;
  for (long long t = blockIdx.x; t < ntiles; t += nblk) {
    const FilterTile tile = filter_tile_at(a.g, t);
    __syncthreads();
    filter_stage<Z>(a.g, tile, s, [&](long long e, int, int, int) { return __ldcg(&a.x_new[e]); });
    __syncthreads();
    filter_apply<Z>(a.g, a.fc, tile, s, [&](long long e, int, int, int, double v) {
      double r = a.pr.value(v / __ldg(&a.Hs[e]), nullptr);
      const double q = __ldcg(&a.ratio[e]);
      if (q == kCodeSolid) r = 1.0;
      if (q == kCodeVoid) r = 0.0;
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
  const size_t smem = filter_smem_bytes(fc.Z);
  const long long ntiles = filter_ntiles(g);
  TP3D_DISPATCH_Z(fc.Z, {
    auto kern = oc_kernel<ZC>;
    if (int rc = ensure_dynamic_smem(kern, smem)) return rc;
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

// ---------------------------------------------------------------------------
// OC update without device allocation.
//
// For callers that must not allocate device memory per call: an application
// whose device memory is fully reserved up front by its own allocator, or code
// that cannot accept the implicit device synchronisation that cudaMalloc /
// cudaFree bring.  The scratch of the bisection (normalised ratios, per-block
// partial sums, barrier counters, filter column table) lives in one
// file-scope __device__ array instead.  Every GPU that loads this library
// holds that array (about 2.2 MB) until the process exits.
// ---------------------------------------------------------------------------
namespace {

constexpr long long kNoAllocMaxElements = 1LL << 18;  // e.g. 64x64x64 or 128x64x32
constexpr int kNoAllocMaxCols = (2 * kFilterMaxZ + 1) * (2 * kFilterMaxZ + 1);
constexpr size_t kNoAllocRatioBytes = (size_t)kNoAllocMaxElements * sizeof(double);
constexpr size_t kNoAllocPartBytes = (size_t)3 * kOcMaxBlocks * sizeof(double);
constexpr size_t kNoAllocBarrierBytes = 256;
constexpr size_t kNoAllocDxyBytes = ((kNoAllocMaxCols * sizeof(int2) + 255) / 256) * 256;
constexpr size_t kNoAllocWBytes = (size_t)kNoAllocMaxCols * (2 * kFilterMaxZ + 1) * sizeof(double);
constexpr size_t kNoAllocBytes =
    kNoAllocRatioBytes + kNoAllocPartBytes + kNoAllocBarrierBytes + kNoAllocDxyBytes + kNoAllocWBytes;

static __device__ __align__(256) unsigned char g_oc_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_addr[64] = {};  // per device: device address of g_oc_noalloc_scratch

// Device address of the static scratch on the current device; looked up once per
// device with that device current.
int noalloc_scratch(void** out) {
  int dev = 0;
  TP3D_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    tp3d_set_last_error("device ordinal out of range for the static OC scratch");
    return TP3D_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_oc_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      tp3d_set_last_error(e != cudaSuccess ? cudaGetErrorString(e) : "null symbol address");
      return TP3D_ERR_CUDA;
    }
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return TP3D_OK;
}

// Filter columns for rmin, built on the host in the same order as the
// allocating path's table (rmin - |d| > 1e-9, grouped by (dx, dy)).
int noalloc_columns(double rmin, int* Z, std::vector<int2>* dxy, std::vector<double>* w) {
  if (!(rmin > 0.0) || !std::isfinite(rmin)) return TP3D_ERR_ARG;
  const int R = (int)std::ceil(rmin) + 1;
  int z = 0;
  for (int d = 0; d <= R; ++d)
    if (rmin - std::sqrt((double)(d * d)) > 1e-9) z = d;
  if (z > kFilterMaxZ) {
    tp3d_set_last_error("rmin too large for the stencil filter (max 7)");
    return TP3D_ERR_ARG;
  }
  const int W = 2 * z + 1;
  for (int dx = -z; dx <= z; ++dx)
    for (int dy = -z; dy <= z; ++dy) {
      std::vector<double> col(W, 0.0);
      bool any = false;
      for (int dz = -z; dz <= z; ++dz) {
        const double wt = rmin - std::sqrt((double)(dx * dx + dy * dy + dz * dz));
        if (wt > 1e-9) {
          col[dz + z] = wt;
          any = true;
        }
      }
      if (any) {
        dxy->push_back(make_int2(dx, dy));
        w->insert(w->end(), col.begin(), col.end());
      }
    }
  *Z = z;
  return TP3D_OK;
}

}  // namespace

extern "C" long long tp3d_oc_noalloc_max_elements(void) { return kNoAllocMaxElements; }

extern "C" int tp3d_oc_update_noalloc(int nelx, int nely, int nelz, double rmin, const double* x,
                                      const double* dc_dx, const double* dv_dx, const double* Hs,
                                      const uint8_t* solid, const uint8_t* void_, double move,
                                      double target_free_volume, double beta, double eta, int max_bisection,
                                      double bisection_tol, double* x_new, double* rho_new, double* stats,
                                      void* stream) {
  if (nelx < 1 || nely < 1 || nelz < 1 || !x || !dc_dx || !dv_dx || !Hs || !x_new || !rho_new || !stats)
    return TP3D_ERR_ARG;
  const long long n = (long long)nelx * nely * nelz;
  if (n > kNoAllocMaxElements) {
    tp3d_set_last_error(
        "tp3d_oc_update_noalloc: the grid has more elements than the static scratch holds (max 262144); "
        "use tp3d_oc_update with caller-provided scratch");
    return TP3D_ERR_ARG;
  }
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
  int Z = 0;
  std::vector<int2> dxy;
  std::vector<double> w;
  if (int rc = noalloc_columns(rmin, &Z, &dxy, &w)) return rc;
  void* base_v = nullptr;
  if (int rc = noalloc_scratch(&base_v)) return rc;
  unsigned char* base = (unsigned char*)base_v;
  cudaStream_t st = (cudaStream_t)stream;

  const Grid g{nelx, nely, nelz};
  OcArgs a{g, FilterCols{}, x, dc_dx, dv_dx, Hs, solid, void_, move, target_free_volume, bisection_tol,
           max_bisection, Projection(beta, eta), x_new, rho_new, stats};
  a.ratio = (double*)base;
  a.partA = (double*)(base + kNoAllocRatioBytes);
  a.partB = a.partA + kOcMaxBlocks;
  a.partC = a.partB + kOcMaxBlocks;
  unsigned int* bar = (unsigned int*)(base + kNoAllocRatioBytes + kNoAllocPartBytes);
  a.bar.count = bar;
  a.bar.gen = bar + 1;
  a.bar.err = (int*)(bar + 2);
  int2* d_dxy = (int2*)(base + kNoAllocRatioBytes + kNoAllocPartBytes + kNoAllocBarrierBytes);
  double* d_w = (double*)((unsigned char*)d_dxy + kNoAllocDxyBytes);
  a.fc.dxy = d_dxy;
  a.fc.w = d_w;
  a.fc.ncols = (int)dxy.size();
  a.fc.Z = Z;
  // The array keeps the previous call's contents: the column table is
  // rewritten and the barrier counters cleared on every call.
  TP3D_CHECK(cudaMemcpyAsync(d_dxy, dxy.data(), dxy.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
  TP3D_CHECK(cudaMemcpyAsync(d_w, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  TP3D_CHECK(cudaMemsetAsync(bar, 0, kNoAllocBarrierBytes, st));
  TP3D_CHECK(cudaMemsetAsync(stats, 0xff, 8 * sizeof(double), st));

  int dev = 0, nsm = 0;
  TP3D_CHECK(cudaGetDevice(&dev));
  TP3D_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const size_t smem = filter_smem_bytes(Z);
  const long long ntiles = filter_ntiles(g);
  TP3D_DISPATCH_Z(Z, {
    auto kern = oc_kernel<ZC>;
    if (int rc = ensure_dynamic_smem(kern, smem)) return rc;
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
