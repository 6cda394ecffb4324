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
#include <atomic>
#include <cfloat>
#include <cmath>
#include <mutex>

#include "tp3d_filter.cuh"

namespace tp3d {
namespace {

constexpr int kOcMaxBlocks = 4096;
constexpr int kOcBatch = 8;  // staged candidates per thread whose loads are in flight together

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
  long long spin_limit;   // polls before a grid-barrier wait gives up
  unsigned int phantom;   // blocks the barrier waits for that never arrive (wait-expiry test only)
};

// Wait-expiry test hook (tp3d_debug_expire_oc_waits): 0 = normal waits.
std::atomic<long long> g_test_spin_limit{0};
std::atomic<int> g_test_phantom{0};

void set_wait_policy(OcArgs& a) {
  const long long lim = g_test_spin_limit.load();
  a.spin_limit = lim > 0 ? lim : kSpinLimit;
  a.phantom = (unsigned int)g_test_phantom.load();
}

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
    // kOcBatch elements per thread at a time: all their loads are issued
    // before the first candidate is formed, so they are in flight together
    for (int i0 = threadIdx.x; i0 < NS; i0 += kOcBatch * kFilterThreads) {
      double xv[kOcBatch], qv[kOcBatch];
      unsigned in = 0;
#pragma unroll
      for (int b = 0; b < kOcBatch; ++b) {
        const int i = i0 + b * kFilterThreads;
        xv[b] = 0.0;
        qv[b] = 0.0;
        if (i < NS) {
          const int ly = i % SY, r = i / SY;
          const int lx = r % SX, lz = r / SX;
          const int gx = tile.x0 + lx - Z, gy = tile.y0 + ly - Z, gz = tile.z0 + lz - Z;
          if (gx >= 0 && gx < a.g.nx && gy >= 0 && gy < a.g.ny && gz >= 0 && gz < a.g.nz) {
            const long long e = a.g.eidx(gx, gy, gz);
            xv[b] = __ldg(&a.x[e]);
            qv[b] = __ldcg(&a.ratio[e]);
            in |= 1u << b;
          }
        }
      }
#pragma unroll
      for (int b = 0; b < kOcBatch; ++b) {
        const int i = i0 + b * kFilterThreads;
        if (i < NS) s[i] = ((in >> b) & 1u) ? candidate_q(xv[b], qv[b], isl, a.move) : 0.0;
      }
    }
    __syncthreads();
    filter_apply<Z>(a.g, a.fc, tile, s, [&](long long e, int, int, int, double v) {
      if (__ldcg(&a.ratio[e]) >= 0.0) vpart += a.pr.value(v / __ldg(&a.Hs[e]), nullptr);
    });
  }
  vpart = block_sum(vpart, red);
  if (threadIdx.x == 0) part[blockIdx.x] = vpart;
  if (!grid_sync_flip(a.bar.count, a.bar.err, a.spin_limit, a.phantom)) return false;
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
  if (!grid_sync_flip(a.bar.count, a.bar.err, a.spin_limit, a.phantom)) return;
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
  if (!grid_sync_flip(a.bar.count, a.bar.err, a.spin_limit, a.phantom)) return;

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
    constexpr int kProbes = 16;  // the search over j <= 81 makes at most 8 probes
    int pj[kProbes];
    double pv[kProbes];
    int np = 0;
    bool first = true;  // probe j = 1 first: it is the reference's own first step, and K = 0 is common
    auto eval_j = [&](int j, double* v) {
      return oc_volume<Z>(a, ldexp(1.0e12, -j), (pass++ & 1) ? a.partB : a.partA, s, red, v);
    };
    while (jhi - jlo > 1) {
      const int jm = first ? 1 : (jlo + jhi) >> 1;
      first = false;
      double v;
      if (!eval_j(jm, &v)) return;
      if (v > a.target) {
        jhi = jm;
        vhi = v;
      } else {
        jlo = jm;
        vlo = v;
        if (np < kProbes) {
          pj[np] = jm;
          pv[np] = v;
          ++np;
        }
      }
    }
    if (jlo >= 1) {
      // Steps 1..K (K = jlo) only halve the upper bound, and their volumes do
      // not decrease with j, so the smallest error among them is step K's.
      // The reference keeps the FIRST step with the smallest error (strict <,
      // oc_update.py:106): if steps before K have exactly step K's volume (a
      // plateau, e.g. every candidate held at its move limit), it reports the
      // first of them.  Those steps form a range j0..K; j0 is found from the
      // probes (jb: largest probe below K with a smaller volume, jeq: smallest
      // probe with step K's volume), evaluating step K - 1 when no probe
      // decides it and bisecting (jb, jeq] only when a tie is seen.
      int jb = 0, jeq = jlo;
      for (int i = 0; i < np; ++i) {
        if (pv[i] < vlo) jb = max(jb, pj[i]);
        else if (pv[i] == vlo) jeq = min(jeq, pj[i]);
      }
      if (jeq == jlo && jb < jlo - 1) {
        double v;
        if (!eval_j(jlo - 1, &v)) return;
        if (v == vlo) jeq = jlo - 1;
        else jb = jlo - 1;
      }
      while (jeq - jb > 1) {
        const int jm = (jb + jeq) >> 1;
        double v;
        if (!eval_j(jm, &v)) return;
        if (v == vlo) jeq = jm;
        else jb = jm;
      }
      best_err = fabs(vlo - a.target);
      best_lam = ldexp(1.0e12, -jeq);
      best_vol = vlo;
      hi = ldexp(1.0e12, -jlo);
      it = jlo;
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
  if (!grid_sync_flip(a.bar.count, a.bar.err, a.spin_limit, a.phantom)) return;
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
  set_wait_policy(a);
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
namespace tp3d_oc_noalloc {

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

// The filter column table of a radius, built in place in the static scratch:
// thread i evaluates candidate column i (filter_column, the same function and
// order as the host-built tables of the allocating path) and writes it at its
// rank among the columns that have a tap.  No host buffer is involved.
__global__ void __launch_bounds__(256) noalloc_columns_kernel(double rmin, int Z, int2* dxy, double* w) {
  __shared__ int has_tap[256];
  const int W = 2 * Z + 1, i = threadIdx.x;
  double col[2 * kFilterMaxZ + 1];
  const bool any = i < W * W && filter_column(rmin, Z, i, col);
  has_tap[i] = any ? 1 : 0;
  __syncthreads();
  if (any) {
    int pos = 0;
    for (int k = 0; k < i; ++k) pos += has_tap[k];
    dxy[pos] = make_int2(i / W - Z, i % W - Z);
    for (int j = 0; j < W; ++j) w[(size_t)pos * W + j] = col[j];
  }
}
static_assert((2 * kFilterMaxZ + 1) * (2 * kFilterMaxZ + 1) <= 256, "one thread per candidate column");

}  // namespace tp3d_oc_noalloc
using namespace tp3d_oc_noalloc;

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
  const int Z = filter_radius_z(rmin);
  if (Z < 0 || !std::isfinite(rmin)) return TP3D_ERR_ARG;
  if (Z > kFilterMaxZ) {
    tp3d_set_last_error("rmin too large for the stencil filter (max 7)");
    return TP3D_ERR_ARG;
  }
  void* base_v = nullptr;
  if (int rc = noalloc_scratch(&base_v)) return rc;
  unsigned char* base = (unsigned char*)base_v;
  cudaStream_t st = (cudaStream_t)stream;

  const Grid g{nelx, nely, nelz};
  OcArgs a{g, FilterCols{}, x, dc_dx, dv_dx, Hs, solid, void_, move, target_free_volume, bisection_tol,
           max_bisection, Projection(beta, eta), x_new, rho_new, stats};
  set_wait_policy(a);
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
  a.fc.ncols = filter_columns_build(rmin, Z, nullptr, nullptr);  // count only
  a.fc.Z = Z;
  // The array keeps the previous call's contents: the column table is
  // rebuilt on the device and the barrier counters cleared on every call.
  noalloc_columns_kernel<<<1, 256, 0, st>>>(rmin, Z, d_dxy, d_w);
  TP3D_CHECK_LAUNCH();
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
  add_launches(2);
  return TP3D_OK;
}

extern "C" int tp3d_debug_expire_oc_waits(long long spin_limit, int phantom_blocks) {
  if (spin_limit < 0 || phantom_blocks < 0 || phantom_blocks > 1024) return TP3D_ERR_ARG;
  g_test_spin_limit.store(spin_limit);
  g_test_phantom.store(phantom_blocks);
  return TP3D_OK;
}
