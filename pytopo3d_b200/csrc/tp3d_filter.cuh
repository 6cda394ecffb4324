// Cone density filter as a shared-memory stencil.
//
// The reference builds an explicit sparse H with weights rmin - |d| for
// integer offsets d with rmin - |d| > 1e-9, truncated at the domain boundary
// (pytopo3d/utils/filter.py:122-228).  H is symmetric, so H x and H^T g are the
// same stencil.  Here H is never formed: a block stages a (32 + 2Z) x (TX + 2Z)
// x (KZ + 2Z) tile of the input (zero outside the domain, which reproduces the
// boundary truncation) in shared memory, and each thread produces KZ outputs
// along z.  Taps are grouped in (dx, dy) columns so each staged value is loaded
// once per column and reused for all KZ outputs.
#pragma once

#include "tp3d_common.cuh"

namespace tp3d {

constexpr int kFilterTY = 32;   // outputs along y per block (one warp)
constexpr int kFilterTX = 8;    // outputs along x per block (warps per block)
constexpr int kFilterKZ = 8;    // outputs along z per thread
constexpr int kFilterThreads = kFilterTY * kFilterTX;
constexpr int kFilterMaxZ = 6;  // supports rmin <= 7 (the staged tile of Z = 7 exceeds shared memory)

struct FilterCols {
  const int2* dxy;    // (dx, dy) per column
  const double* w;    // ncols x (2Z+1) weights, 0 where the tap is absent
  int ncols;
  int Z;              // max |offset| along any axis
};

// Host: columns for a radius, cached per (device, rmin).  Returns nonzero on error.
int filter_cols_for(double rmin, FilterCols* out);

// Largest offset along one axis with a positive cone weight: the largest d with
// rmin - d > 1e-9 (pytopo3d/utils/filter.py:193-206).  -1 for an invalid rmin.
__host__ __device__ inline int filter_radius_z(double rmin) {
  if (!(rmin > 0.0) || !(rmin < 1.0e6)) return -1;
  int Z = 0;
  for (int d = 1; d <= (int)rmin + 1; ++d)
    if (rmin - sqrt((double)(d * d)) > 1e-9) Z = d;
  return Z;
}

// Column i of the (2Z+1)^2 candidate columns of a radius with max offset Z,
// in row-major order over (dx, dy) in [-Z, Z]^2: writes its 2Z+1 weights along
// dz (rmin - sqrt(dx^2 + dy^2 + dz^2) where that exceeds 1e-9, else 0) and
// returns whether it has any tap (pytopo3d/utils/filter.py:193-206).
__host__ __device__ inline bool filter_column(double rmin, int Z, int i, double* wcol) {
  const int W = 2 * Z + 1;
  const int dx = i / W - Z, dy = i % W - Z;
  bool any = false;
  for (int dz = -Z; dz <= Z; ++dz) {
    const double wt = rmin - sqrt((double)(dx * dx + dy * dy + dz * dz));
    const bool tap = wt > 1e-9;
    any = any || tap;
    wcol[dz + Z] = tap ? wt : 0.0;
  }
  return any;
}

// The column table of a radius with max offset Z <= kFilterMaxZ: the columns
// of filter_column that have a tap, in that order, with their (dx, dy)
// offsets.  Returns the number of columns; dxy / w may be null (count only).
// The host builds the cached tables with it, and the allocation-free OC path
// builds its table on the device from filter_column in the same order, so
// both give the same columns and bit-identical weights (IEEE sqrt and
// subtraction on both sides).
__host__ __device__ inline int filter_columns_build(double rmin, int Z, int2* dxy, double* w) {
  const int W = 2 * Z + 1;
  int n = 0;
  for (int i = 0; i < W * W; ++i) {
    double col[2 * kFilterMaxZ + 1];
    if (filter_column(rmin, Z, i, col)) {
      if (dxy) dxy[n] = make_int2(i / W - Z, i % W - Z);
      if (w)
        for (int j = 0; j < W; ++j) w[(size_t)n * W + j] = col[j];
      ++n;
    }
  }
  return n;
}

__host__ __device__ inline int filter_smem_elems(int Z) {
  return (kFilterTY + 2 * Z) * (kFilterTX + 2 * Z) * (kFilterKZ + 2 * Z);
}

// Columns of a radius with max offset Z: at most (2Z+1)^2.  Kernels copy the
// column table (weights, then offsets) into shared memory after the staged
// tile, so the stencil loop reads it with broadcast shared loads.
__host__ __device__ inline int filter_max_cols(int Z) { return (2 * Z + 1) * (2 * Z + 1); }
__host__ __device__ inline size_t filter_smem_bytes(int Z) {
  return (size_t)filter_smem_elems(Z) * sizeof(double) +
         (size_t)filter_max_cols(Z) * ((2 * Z + 1) * sizeof(double) + sizeof(int2));
}

// Copy fc's table into the shared table area of `s` (call before a barrier
// that precedes the first filter_apply).
template <int Z>
__device__ __forceinline__ void filter_cols_to_smem(const FilterCols& fc, double* s) {
  constexpr int W = 2 * Z + 1;
  double* sw = s + filter_smem_elems(Z);
  int2* sd = reinterpret_cast<int2*>(sw + filter_max_cols(Z) * W);
  for (int i = threadIdx.x; i < fc.ncols * W; i += blockDim.x) sw[i] = __ldg(&fc.w[i]);
  for (int i = threadIdx.x; i < fc.ncols; i += blockDim.x) sd[i] = fc.dxy[i];
}

struct FilterTile {
  int x0, y0, z0;
};

__host__ __device__ inline int filter_tiles_x(const Grid& g) { return (g.nx + kFilterTX - 1) / kFilterTX; }
__host__ __device__ inline int filter_tiles_y(const Grid& g) { return (g.ny + kFilterTY - 1) / kFilterTY; }
__host__ __device__ inline int filter_tiles_z(const Grid& g) { return (g.nz + kFilterKZ - 1) / kFilterKZ; }
__host__ __device__ inline long long filter_ntiles(const Grid& g) {
  return (long long)filter_tiles_x(g) * filter_tiles_y(g) * filter_tiles_z(g);
}
__device__ inline FilterTile filter_tile_at(const Grid& g, long long t) {
  const int ty = filter_tiles_y(g), tx = filter_tiles_x(g);
  FilterTile r;
  r.y0 = (int)(t % ty) * kFilterTY;
  t /= ty;
  r.x0 = (int)(t % tx) * kFilterTX;
  r.z0 = (int)(t / tx) * kFilterKZ;
  return r;
}

// Stage `load(e, x, y, z)` (called only for in-domain elements) into `s`.
template <int Z, class Load>
__device__ __forceinline__ void filter_stage(const Grid& g, const FilterTile& t, double* s, Load load) {
  constexpr int SY = kFilterTY + 2 * Z, SX = kFilterTX + 2 * Z, SZ = kFilterKZ + 2 * Z;
  for (int i = threadIdx.x; i < SY * SX * SZ; i += blockDim.x) {
    const int ly = i % SY;
    const int r = i / SY;
    const int lx = r % SX, lz = r / SX;
    const int gx = t.x0 + lx - Z, gy = t.y0 + ly - Z, gz = t.z0 + lz - Z;
    double v = 0.0;
    if (gx >= 0 && gx < g.nx && gy >= 0 && gy < g.ny && gz >= 0 && gz < g.nz)
      v = load(g.eidx(gx, gy, gz), gx, gy, gz);
    s[i] = v;
  }
}

// Apply the staged stencil; calls `store(e, x, y, z, value)` for in-domain outputs.
template <int Z, class Store>
__device__ __forceinline__ void filter_apply(const Grid& g, const FilterCols& fc, const FilterTile& t,
                                             const double* s, Store store) {
  constexpr int SY = kFilterTY + 2 * Z, SX = kFilterTX + 2 * Z;
  constexpr int W = 2 * Z + 1;
  const int ly = threadIdx.x % kFilterTY, lx = threadIdx.x / kFilterTY;
  const double* sw = s + filter_smem_elems(Z);  // table copied by filter_cols_to_smem
  const int2* sd = reinterpret_cast<const int2*>(sw + filter_max_cols(Z) * W);
  double acc[kFilterKZ];
#pragma unroll
  for (int k = 0; k < kFilterKZ; ++k) acc[k] = 0.0;
  for (int c = 0; c < fc.ncols; ++c) {
    const int2 d = sd[c];
    const double* wc = sw + c * W;
    double wv[W];
#pragma unroll
    for (int j = 0; j < W; ++j) wv[j] = wc[j];
    const double* col = s + (size_t)(lx + Z + d.x) * SY + (ly + Z + d.y);
    double v[kFilterKZ + 2 * Z];
#pragma unroll
    for (int j = 0; j < kFilterKZ + 2 * Z; ++j) v[j] = col[(size_t)j * SX * SY];
#pragma unroll
    for (int k = 0; k < kFilterKZ; ++k) {
#pragma unroll
      for (int j = 0; j < W; ++j) acc[k] = fma(wv[j], v[k + j], acc[k]);
    }
  }
  const int gx = t.x0 + lx, gy = t.y0 + ly;
  if (gx < g.nx && gy < g.ny) {
#pragma unroll
    for (int k = 0; k < kFilterKZ; ++k) {
      const int gz = t.z0 + k;
      if (gz < g.nz) store(g.eidx(gx, gy, gz), gx, gy, gz, acc[k]);
    }
  }
}

// Heaviside projection (pytopo3d/utils/filter.py:26-60).
struct Projection {
  double beta, eta, tbe, den;
  __host__ Projection(double b, double e) : beta(b), eta(e) {
    tbe = tanh(b * e);
    den = tanh(b * e) + tanh(b * (1.0 - e));
  }
  // Same operation order as the reference: divide by the denominator.
  __device__ __forceinline__ double value(double rf, double* deriv) const {
    const double t = tanh(beta * (rf - eta));
    if (deriv) *deriv = beta * (1.0 - t * t) / den;
    const double r = (tbe + t) / den;
    return fmin(fmax(r, 0.0), 1.0);
  }
};

// Dispatch a templated launcher on Z at runtime.
#define TP3D_DISPATCH_Z(Zval, ...)                      \
  switch (Zval) {                                       \
    case 0: { constexpr int ZC = 0; __VA_ARGS__; } break; \
    case 1: { constexpr int ZC = 1; __VA_ARGS__; } break; \
    case 2: { constexpr int ZC = 2; __VA_ARGS__; } break; \
    case 3: { constexpr int ZC = 3; __VA_ARGS__; } break; \
    case 4: { constexpr int ZC = 4; __VA_ARGS__; } break; \
    case 5: { constexpr int ZC = 5; __VA_ARGS__; } break; \
    case 6: { constexpr int ZC = 6; __VA_ARGS__; } break; \
    default: return TP3D_ERR_ARG;                       \
  }

}  // namespace tp3d
