// Obstacle masks on the device: cube, sphere and cylinder primitives OR-ed
// into a flat uint8 element mask.
// Reference: pytopo3d/utils/obstacles.py:12-193 (create_cube_obstacle,
// create_sphere_obstacle, create_cylinder_obstacle) and the OR of several
// obstacles in parse_obstacle_config_file (obstacles.py:237-269).
//
// The reference turns each obstacle's fractional centre, size and radius into
// integer element indices on the host (int() truncation) and then tests every
// element with integer arithmetic.  The caller passes those integers
// (tp3d_obstacle); each thread here tests 16 consecutive elements of the
// Fortran-ordered mask against every primitive and writes them with one
// 16-byte store (the mask write, 1 byte per element, is the only HBM traffic).
#include <algorithm>

#include "tp3d_common.cuh"

namespace tp3d {
namespace {

constexpr int kMaskShapes = 32;  // primitives per launch (the host splits longer lists)
constexpr int kMaskPerThread = 16;

struct MaskArgs {
  Grid g;
  int nshapes;
  int accumulate;  // 1: OR into the existing mask (later chunks of a long list)
  tp3d_obstacle s[kMaskShapes];
};

__device__ __forceinline__ bool inside(const tp3d_obstacle& o, int x, int y, int z) {
  const int c[3] = {x, y, z};
  if (o.kind == TP3D_OBSTACLE_CUBE) {
    return x >= o.lo[0] && x < o.hi[0] && y >= o.lo[1] && y < o.hi[1] && z >= o.lo[2] && z < o.hi[2];
  }
  if (o.kind == TP3D_OBSTACLE_SPHERE) {
    const long long dx = x - o.center[0], dy = y - o.center[1], dz = z - o.center[2];
    return dx * dx + dy * dy + dz * dz <= o.r2;
  }
  // cylinder: distance in the plane perpendicular to the axis, bounded along it
  long long d2 = 0;
#pragma unroll
  for (int k = 0; k < 3; ++k)
    if (k != o.axis) {
      const long long d = c[k] - o.center[k];
      d2 += d * d;
    }
  const int a = c[o.axis];
  return d2 <= o.r2 && a >= o.lo[o.axis] && a < o.hi[o.axis];
}

__global__ void __launch_bounds__(256) obstacle_mask_kernel(const __grid_constant__ MaskArgs p, uint8_t* mask) {
  const long long n = p.g.nele();
  const long long e0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * kMaskPerThread;
  if (e0 >= n) return;
  int y = (int)(e0 % p.g.ny);
  long long r = e0 / p.g.ny;
  int x = (int)(r % p.g.nx), z = (int)(r / p.g.nx);
  uint8_t v[kMaskPerThread];
#pragma unroll
  for (int k = 0; k < kMaskPerThread; ++k) {
    bool in = false;
    if (e0 + k < n) {
      for (int i = 0; i < p.nshapes && !in; ++i) in = inside(p.s[i], x, y, z);
    }
    v[k] = in ? 1 : 0;
    if (++y == p.g.ny) {  // next element in Fortran order
      y = 0;
      if (++x == p.g.nx) {
        x = 0;
        ++z;
      }
    }
  }
  uint8_t* out = mask + e0;
  const bool full = e0 + kMaskPerThread <= n && ((uintptr_t)out & 15) == 0;
  if (full) {
    uint4 w;
    if (p.accumulate) w = *reinterpret_cast<const uint4*>(out);
    else w = make_uint4(0, 0, 0, 0);
    unsigned int* wp = &w.x;
#pragma unroll
    for (int k = 0; k < kMaskPerThread; ++k) wp[k >> 2] |= (unsigned int)v[k] << (8 * (k & 3));
    *reinterpret_cast<uint4*>(out) = w;
  } else {
    for (int k = 0; k < kMaskPerThread && e0 + k < n; ++k) out[k] = p.accumulate ? (uint8_t)(out[k] | v[k]) : v[k];
  }
}

}  // namespace
}  // namespace tp3d

using namespace tp3d;

extern "C" int tp3d_obstacle_mask(int nelx, int nely, int nelz, const tp3d_obstacle* shapes, int nshapes,
                                  uint8_t* mask, void* stream) {
  if (nelx < 1 || nely < 1 || nelz < 1 || nshapes < 0 || !mask || (nshapes > 0 && !shapes)) {
    tp3d_set_last_error("tp3d_obstacle_mask: invalid grid, shape list or mask pointer");
    return TP3D_ERR_ARG;
  }
  for (int i = 0; i < nshapes; ++i) {
    const tp3d_obstacle& o = shapes[i];
    if (o.kind < TP3D_OBSTACLE_CUBE || o.kind > TP3D_OBSTACLE_CYLINDER ||
        (o.kind == TP3D_OBSTACLE_CYLINDER && (o.axis < 0 || o.axis > 2))) {
      tp3d_set_last_error("tp3d_obstacle_mask: unknown obstacle kind or cylinder axis");
      return TP3D_ERR_ARG;
    }
  }
  const Grid g{nelx, nely, nelz};
  cudaStream_t st = (cudaStream_t)stream;
  const long long threads = (g.nele() + kMaskPerThread - 1) / kMaskPerThread;
  const unsigned int blocks = (unsigned int)((threads + 255) / 256);
  int done = 0, launches = 0;
  do {  // one launch per chunk of up to kMaskShapes primitives (at least one launch: clears the mask)
    MaskArgs a{};
    a.g = g;
    a.nshapes = std::min(kMaskShapes, nshapes - done);
    a.accumulate = done > 0 ? 1 : 0;
    for (int i = 0; i < a.nshapes; ++i) a.s[i] = shapes[done + i];
    obstacle_mask_kernel<<<blocks, 256, 0, st>>>(a, mask);
    TP3D_CHECK_LAUNCH();
    done += a.nshapes;
    ++launches;
  } while (done < nshapes);
  add_launches(launches);
  return TP3D_OK;
}
