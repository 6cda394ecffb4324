// Density filter, Heaviside projection and the filter transpose (chain rule).
// Reference: pytopo3d/utils/filter.py:26-228.
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "tp3d_filter.cuh"

namespace tp3d {

namespace {

struct ColsEntry {
  int2* dxy = nullptr;
  double* w = nullptr;
  int ncols = 0;
  int Z = 0;
};

std::mutex g_cols_mu;
std::map<std::pair<int, unsigned long long>, ColsEntry> g_cols;

}  // namespace

// Taps: integer offsets d with rmin - |d| > 1e-9 and weight rmin - sqrt(|d|^2)
// (pytopo3d/utils/filter.py:193-206), grouped by (dx, dy) column.
int filter_cols_for(double rmin, FilterCols* out) {
  if (!(rmin > 0.0) || !std::isfinite(rmin)) return TP3D_ERR_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return TP3D_ERR_CUDA;
  unsigned long long bits;
  static_assert(sizeof(bits) == sizeof(rmin), "");
  memcpy(&bits, &rmin, sizeof(bits));
  std::lock_guard<std::mutex> lk(g_cols_mu);
  auto key = std::make_pair(dev, bits);
  auto it = g_cols.find(key);
  if (it == g_cols.end()) {
    const int Z = filter_radius_z(rmin);
    if (Z < 0) return TP3D_ERR_ARG;
    if (Z > kFilterMaxZ) {
      tp3d_set_last_error("rmin too large for the stencil filter (max 7)");
      return TP3D_ERR_ARG;
    }
    const int ncols = filter_columns_build(rmin, Z, nullptr, nullptr);
    std::vector<int2> dxy(ncols);
    std::vector<double> w((size_t)ncols * (2 * Z + 1));
    filter_columns_build(rmin, Z, dxy.data(), w.data());
    ColsEntry e;
    e.ncols = (int)dxy.size();
    e.Z = Z;
    if (cudaMalloc(&e.dxy, dxy.size() * sizeof(int2)) != cudaSuccess) return TP3D_ERR_CUDA;
    if (cudaMalloc(&e.w, w.size() * sizeof(double)) != cudaSuccess) return TP3D_ERR_CUDA;
    if (cudaMemcpy(e.dxy, dxy.data(), dxy.size() * sizeof(int2), cudaMemcpyHostToDevice) != cudaSuccess)
      return TP3D_ERR_CUDA;
    if (cudaMemcpy(e.w, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
      return TP3D_ERR_CUDA;
    it = g_cols.emplace(key, e).first;
  }
  out->dxy = it->second.dxy;
  out->w = it->second.w;
  out->ncols = it->second.ncols;
  out->Z = it->second.Z;
  return TP3D_OK;
}

namespace {

// Hs = H 1 (row sums), 0 -> 1 (filter.py:224-226).
template <int Z>
__global__ void __launch_bounds__(kFilterThreads) rowsum_kernel(Grid g, FilterCols fc, double* Hs) {
  extern __shared__ double s[];
  const FilterTile t = filter_tile_at(g, blockIdx.x);
  filter_cols_to_smem<Z>(fc, s);
  filter_stage<Z>(g, t, s, [](long long, int, int, int) { return 1.0; });
  __syncthreads();
  filter_apply<Z>(g, fc, t, s, [&](long long e, int, int, int, double v) { Hs[e] = (v == 0.0) ? 1.0 : v; });
}

// build_physical_density (filter.py:63-100).
template <int Z>
__global__ void __launch_bounds__(kFilterThreads)
    project_kernel(Grid g, FilterCols fc, const double* __restrict__ x, const double* __restrict__ Hs,
                   Projection pr, const uint8_t* __restrict__ solid, const uint8_t* __restrict__ vd,
                   double* rf, double* rp, double* dp) {
  extern __shared__ double s[];
  const FilterTile t = filter_tile_at(g, blockIdx.x);
  filter_cols_to_smem<Z>(fc, s);
  filter_stage<Z>(g, t, s, [&](long long e, int, int, int) { return __ldg(&x[e]); });
  __syncthreads();
  filter_apply<Z>(g, fc, t, s, [&](long long e, int, int, int, double v) {
    const double f = v / __ldg(&Hs[e]);
    double d;
    double r = pr.value(f, &d);
    const bool so = solid && solid[e], vo = vd && vd[e];
    if (so) r = 1.0;
    if (vo) r = 0.0;
    if (so || vo) d = 0.0;
    if (rf) rf[e] = f;
    rp[e] = r;
    if (dp) dp[e] = d;
  });
}

// apply_density_filter_chain_rule (filter.py:103-119): H^T (g dproj / Hs).
template <int Z>
__global__ void __launch_bounds__(kFilterThreads)
    transpose_kernel(Grid g, FilterCols fc, const double* __restrict__ gin, const double* __restrict__ dp,
                     const double* __restrict__ Hs, double* out) {
  extern __shared__ double s[];
  const FilterTile t = filter_tile_at(g, blockIdx.x);
  filter_cols_to_smem<Z>(fc, s);
  filter_stage<Z>(g, t, s, [&](long long e, int, int, int) {
    const double gd = dp ? __ldg(&gin[e]) * __ldg(&dp[e]) : __ldg(&gin[e]);
    return gd / __ldg(&Hs[e]);
  });
  __syncthreads();
  filter_apply<Z>(g, fc, t, s, [&](long long e, int, int, int, double v) { out[e] = v; });
}

__global__ void heaviside_kernel(const double* __restrict__ rf, long long n, Projection pr, double* out,
                                 double* der) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double d;
    const double r = pr.value(rf[i], &d);
    if (out) out[i] = r;
    if (der) der[i] = d;
  }
}

int check_grid(int nx, int ny, int nz) {
  if (nx < 1 || ny < 1 || nz < 1) {
    tp3d_set_last_error("nelx, nely, and nelz must all be positive");
    return TP3D_ERR_ARG;
  }
  return TP3D_OK;
}

template <class K>
int launch_filter(K kernel, const Grid& g, int Z, cudaStream_t st) {
  const size_t smem = filter_smem_bytes(Z);
  if (int rc = ensure_dynamic_smem(kernel, smem)) return rc;
  (void)st;
  return TP3D_OK;
}

}  // namespace
}  // namespace tp3d

using namespace tp3d;

extern "C" int tp3d_filter_rowsum(int nelx, int nely, int nelz, double rmin, double* Hs, void* stream) {
  if (int rc = check_grid(nelx, nely, nelz)) return rc;
  if (!Hs) return TP3D_ERR_ARG;
  FilterCols fc;
  if (int rc = filter_cols_for(rmin, &fc)) return rc;
  const Grid g{nelx, nely, nelz};
  cudaStream_t st = (cudaStream_t)stream;
  const size_t smem = filter_smem_bytes(fc.Z);
  TP3D_DISPATCH_Z(fc.Z, {
    if (int rc = launch_filter(rowsum_kernel<ZC>, g, ZC, st)) return rc;
    rowsum_kernel<ZC><<<(unsigned)filter_ntiles(g), kFilterThreads, smem, st>>>(g, fc, Hs);
  });
  add_launches(1);
  TP3D_CHECK_LAUNCH();
  return TP3D_OK;
}

extern "C" int tp3d_filter_project(int nelx, int nely, int nelz, double rmin, const double* x,
                                   const double* Hs, double beta, double eta, const uint8_t* solid,
                                   const uint8_t* void_, double* rho_filtered, double* rho_physical,
                                   double* dproj, void* stream) {
  if (int rc = check_grid(nelx, nely, nelz)) return rc;
  if (!x || !Hs || !rho_physical) return TP3D_ERR_ARG;
  if (!std::isfinite(beta) || beta <= 0.0) {
    tp3d_set_last_error("beta must be positive");
    return TP3D_ERR_ARG;
  }
  if (!(eta > 0.0 && eta < 1.0)) {
    tp3d_set_last_error("eta must be between 0 and 1");
    return TP3D_ERR_ARG;
  }
  FilterCols fc;
  if (int rc = filter_cols_for(rmin, &fc)) return rc;
  const Grid g{nelx, nely, nelz};
  cudaStream_t st = (cudaStream_t)stream;
  const size_t smem = filter_smem_bytes(fc.Z);
  const Projection pr(beta, eta);
  TP3D_DISPATCH_Z(fc.Z, {
    if (int rc = launch_filter(project_kernel<ZC>, g, ZC, st)) return rc;
    project_kernel<ZC><<<(unsigned)filter_ntiles(g), kFilterThreads, smem, st>>>(
        g, fc, x, Hs, pr, solid, void_, rho_filtered, rho_physical, dproj);
  });
  add_launches(1);
  TP3D_CHECK_LAUNCH();
  return TP3D_OK;
}

extern "C" int tp3d_filter_transpose(int nelx, int nely, int nelz, double rmin, const double* gin,
                                     const double* dproj, const double* Hs, double* out, void* stream) {
  if (int rc = check_grid(nelx, nely, nelz)) return rc;
  if (!gin || !Hs || !out) return TP3D_ERR_ARG;
  FilterCols fc;
  if (int rc = filter_cols_for(rmin, &fc)) return rc;
  const Grid g{nelx, nely, nelz};
  cudaStream_t st = (cudaStream_t)stream;
  const size_t smem = filter_smem_bytes(fc.Z);
  TP3D_DISPATCH_Z(fc.Z, {
    if (int rc = launch_filter(transpose_kernel<ZC>, g, ZC, st)) return rc;
    transpose_kernel<ZC><<<(unsigned)filter_ntiles(g), kFilterThreads, smem, st>>>(g, fc, gin, dproj, Hs, out);
  });
  add_launches(1);
  TP3D_CHECK_LAUNCH();
  return TP3D_OK;
}

extern "C" int tp3d_heaviside(const double* rho_filtered, long long n, double beta, double eta, double* out,
                              double* derivative, void* stream) {
  if (n < 0 || (n > 0 && !rho_filtered)) return TP3D_ERR_ARG;
  if (!std::isfinite(beta) || beta <= 0.0) {
    tp3d_set_last_error("beta must be positive");
    return TP3D_ERR_ARG;
  }
  if (!(eta > 0.0 && eta < 1.0)) {
    tp3d_set_last_error("eta must be between 0 and 1");
    return TP3D_ERR_ARG;
  }
  if (n == 0) return TP3D_OK;
  const Projection pr(beta, eta);
  const int blocks = (int)std::min<long long>((n + 255) / 256, 148 * 16);
  heaviside_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(rho_filtered, n, pr, out, derivative);
  add_launches(1);
  TP3D_CHECK_LAUNCH();
  return TP3D_OK;
}
