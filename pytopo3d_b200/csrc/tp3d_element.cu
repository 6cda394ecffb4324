// Element strain energy, SIMP sensitivities and compliance.
// Reference: pytopo3d/core/compliance.py:18-75, pytopo3d/core/optimizer.py:596-625.
#include <cmath>
#include <cstring>

#include "tp3d_filter.cuh"

namespace tp3d {

struct KEd {
  double k[576];  // row-major 24x24 element stiffness
};

// u_e^T KE u_e using the symmetry of KE (24 diagonal + 276 off-diagonal terms).
__device__ __forceinline__ double element_energy(const Grid& g, const double* __restrict__ U, int x, int y,
                                                 int z, const KEd& ke) {
  double u[24];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const long long n = g.nidx(x + corner_ox(a), y + corner_oy(a), z + corner_oz(a));
#pragma unroll
    for (int c = 0; c < 3; ++c) u[3 * a + c] = __ldg(&U[3 * n + c]);
  }
  double diag = 0.0, off = 0.0;
#pragma unroll
  for (int i = 0; i < 24; ++i) {
    diag = fma(ke.k[i * 24 + i] * u[i], u[i], diag);
    double t = 0.0;
#pragma unroll
    for (int j = i + 1; j < 24; ++j) t = fma(ke.k[i * 24 + j], u[j], t);
    off = fma(u[i], t, off);
  }
  return diag + 2.0 * off;
}

__device__ __forceinline__ double simp_pow(double r, double p) {
  if (p == 3.0) return r * r * r;
  if (p == 2.0) return r * r;
  if (p == 1.0) return r;
  return pow(r, p);
}
// numpy's scalar power takes exact fast paths for exponents 2, 1 and 0.5 and
// calls C pow otherwise; mirror that so rho^(p-1) rounds the same way.
__device__ __forceinline__ double np_pow(double r, double p) {
  if (p == 2.0) return r * r;
  if (p == 1.0) return r;
  if (p == 0.5) return sqrt(r);
  if (p == 0.0) return 1.0;
  return pow(r, p);
}

namespace {

__global__ void ce_kernel(Grid g, const double* __restrict__ U, const __grid_constant__ KEd ke, double* ce) {
  const long long n = g.nele();
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(e % g.ny);
    const long long r = e / g.ny;
    const int x = (int)(r % g.nx), z = (int)(r / g.nx);
    ce[e] = element_energy(g, U, x, y, z, ke);
  }
}

// ce, dc = -p (1-Emin) rho^(p-1) ce, dv = free, and per-block partial sums of
// (Emin + (1-Emin) rho^p) ce.
__global__ void __launch_bounds__(256) sens_kernel(Grid g, const double* __restrict__ U,
                                                   const __grid_constant__ KEd ke,
                                                   const double* __restrict__ rho, const uint8_t* __restrict__ fr,
                                                   double penal, double* ce_out, double* dc, double* dv,
                                                   double* partials) {
  __shared__ double red[32];
  const long long n = g.nele();
  const double c0 = -penal * (kE0 - kEmin);
  double part = 0.0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(e % g.ny);
    const long long r = e / g.ny;
    const int x = (int)(r % g.nx), z = (int)(r / g.nx);
    const double ce = element_energy(g, U, x, y, z, ke);
    const double rh = __ldg(&rho[e]);
    if (ce_out) ce_out[e] = ce;
    const double E = kEmin + (kE0 - kEmin) * np_pow(rh, penal);
    part += E * ce;
    dc[e] = c0 * np_pow(rh, penal - 1.0) * ce;
    dv[e] = fr[e] ? 1.0 : 0.0;
  }
  part = block_sum(part, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = part;
}

__global__ void finish_sum_kernel(const double* partials, int n, double* out) {
  __shared__ double red[32];
  const double s = sum_partials(partials, n, red);
  if (threadIdx.x == 0) *out = s;
}

constexpr int kSensBlocks = 148 * 8;

bool load_ke(const double* KE_host, KEd* ke) {
  if (!KE_host) return false;
  std::memcpy(ke->k, KE_host, sizeof(ke->k));
  return true;
}

}  // namespace
}  // namespace tp3d

using namespace tp3d;

extern "C" int tp3d_element_compliance(int nelx, int nely, int nelz, const double* U, const double* KE_host,
                                       double* ce, void* stream) {
  if (nelx < 1 || nely < 1 || nelz < 1 || !U || !ce) return TP3D_ERR_ARG;
  KEd ke;
  if (!load_ke(KE_host, &ke)) return TP3D_ERR_ARG;
  const Grid g{nelx, nely, nelz};
  const int blocks = (int)std::min<long long>((g.nele() + 255) / 256, kSensBlocks);
  ce_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(g, U, ke, ce);
  add_launches(1);
  TP3D_CHECK_LAUNCH();
  return TP3D_OK;
}

extern "C" size_t tp3d_sensitivity_scratch_bytes(int nelx, int nely, int nelz) {
  const long long n = (long long)nelx * nely * nelz;
  return (size_t)(2 * n + kSensBlocks + 32) * sizeof(double);
}

extern "C" int tp3d_sensitivity(int nelx, int nely, int nelz, double rmin, const double* U,
                                const double* KE_host, const double* rho_physical, const double* dproj,
                                const double* Hs, const uint8_t* free_mask, double penal, double* ce,
                                double* dc_dx, double* dv_dx, double* compliance, void* scratch,
                                void* stream) {
  if (nelx < 1 || nely < 1 || nelz < 1 || !U || !rho_physical || !dproj || !Hs || !free_mask || !dc_dx ||
      !dv_dx || !compliance || !scratch)
    return TP3D_ERR_ARG;
  KEd ke;
  if (!load_ke(KE_host, &ke)) return TP3D_ERR_ARG;
  const Grid g{nelx, nely, nelz};
  const long long n = g.nele();
  double* dc = (double*)scratch;
  double* dv = dc + n;
  double* partials = dv + n;
  cudaStream_t st = (cudaStream_t)stream;
  const int blocks = (int)std::min<long long>((n + 255) / 256, kSensBlocks);
  sens_kernel<<<blocks, 256, 0, st>>>(g, U, ke, rho_physical, free_mask, penal, ce, dc, dv, partials);
  TP3D_CHECK_LAUNCH();
  finish_sum_kernel<<<1, 256, 0, st>>>(partials, blocks, compliance);
  add_launches(2);
  TP3D_CHECK_LAUNCH();
  if (int rc = tp3d_filter_transpose(nelx, nely, nelz, rmin, dc, dproj, Hs, dc_dx, stream)) return rc;
  return tp3d_filter_transpose(nelx, nely, nelz, rmin, dv, dproj, Hs, dv_dx, stream);
}
