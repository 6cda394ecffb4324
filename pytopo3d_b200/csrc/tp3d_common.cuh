// Shared definitions for the topo3d_b200 CUDA library (sm_100a).
//
// Index conventions are those of PyTopo3D:
//   element e = y + nely * (x + nelx * z)               (pytopo3d/utils/filter.py:85-87)
//   node    n = iy + (nely+1) * (ix + (nelx+1) * iz)    (pytopo3d/utils/assembly.py:121-129)
//   DOF       = 3 * n + c, c in {x, y, z}
//   local corner order = H8_NODE_OFFSETS                (pytopo3d/utils/assembly.py:17-26)
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/topo3d_b200.h"

namespace tp3d {

struct Grid {
  int nx, ny, nz;  // element counts (nelx, nely, nelz)
  __host__ __device__ long long nele() const { return (long long)nx * ny * nz; }
  __host__ __device__ long long nnode() const { return (long long)(nx + 1) * (ny + 1) * (nz + 1); }
  __host__ __device__ long long eidx(int x, int y, int z) const {
    return y + (long long)ny * (x + (long long)nx * z);
  }
  __host__ __device__ long long nidx(int x, int y, int z) const {
    return y + (long long)(ny + 1) * (x + (long long)(nx + 1) * z);
  }
};

// Local corner index of the corner at offset (ox, oy, oz) in {0,1}^3.
// Order: (0,0,0) (0,1,0) (1,1,0) (1,0,0) (0,0,1) (0,1,1) (1,1,1) (1,0,1).
__host__ __device__ constexpr int corner_index(int ox, int oy, int oz) {
  return oz * 4 + (ox ? (oy ? 2 : 3) : (oy ? 1 : 0));
}
__host__ __device__ constexpr int corner_ox(int a) { return ((a & 3) == 2 || (a & 3) == 3) ? 1 : 0; }
__host__ __device__ constexpr int corner_oy(int a) { return ((a & 3) == 1 || (a & 3) == 2) ? 1 : 0; }
__host__ __device__ constexpr int corner_oz(int a) { return a >> 2; }

constexpr double kEmin = 1.0e-9;
constexpr double kE0 = 1.0;

// ---------------------------------------------------------------------------
// reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide sum; every thread gets the result.  `scratch` holds >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  double t = (threadIdx.x < nw) ? scratch[threadIdx.x] : 0.0;
  if (wid == 0) t = warp_sum(t);
  if (threadIdx.x == 0) scratch[0] = t;
  __syncthreads();
  t = scratch[0];
  __syncthreads();
  return t;
}
__device__ __forceinline__ double block_max(double v, double* scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  double t = (threadIdx.x < nw) ? scratch[threadIdx.x] : -INFINITY;
  if (wid == 0) t = warp_max(t);
  if (threadIdx.x == 0) scratch[0] = t;
  __syncthreads();
  t = scratch[0];
  __syncthreads();
  return t;
}

// Deterministic sum of `n` partials, computed identically by every block.
__device__ __forceinline__ double sum_partials(const double* p, int n, double* scratch) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += p[i];
  return block_sum(v, scratch);
}

// ---------------------------------------------------------------------------
// Grid-wide barrier for cooperative (co-resident) launches.  The spin is
// bounded: after `kSpinLimit` polls (with the back-off of the waits below,
// about a second) the barrier gives up, raises `*err` and returns false so
// that every block can leave its loop and the host reads a status instead of
// the GPU hanging.
// ---------------------------------------------------------------------------
constexpr long long kSpinLimit = 1ll << 23;

struct GridBarrier {
  unsigned int* count;       // arrivals in the current generation
  volatile unsigned int* gen;  // generation counter
  int* err;
};

__device__ __forceinline__ bool grid_sync(GridBarrier b) {
  __syncthreads();
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    const unsigned int nblk = gridDim.x * gridDim.y * gridDim.z;
    const unsigned int g0 = *b.gen;
    __threadfence();
    const unsigned int arrived = atomicAdd(b.count, 1u) + 1u;
    int ok = 1;
    if (arrived == nblk) {
      *b.count = 0;
      __threadfence();
      atomicAdd((unsigned int*)b.gen, 1u);
    } else {
      long long spins = 0;
      while (*b.gen == g0) {
        if (++spins > kSpinLimit || *(volatile int*)b.err != 0) {
          atomicExch(b.err, TP3D_ERR_TIMEOUT);
          ok = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Grid-wide barrier with one atomic per block: block 0 adds 2^31 - (nblocks - 1),
// every other block adds 1, so the top bit of the word flips exactly when the
// last block arrives, and each block waits for the flip of the value it saw.
// The word returns to its low bits after every barrier, so it needs no reset
// between barriers or launches (only a zero before the first launch, and
// after an expired wait).  Bounded: the wait polls without sleeping for its
// first 64 polls (the common case, a few microseconds), then backs off with
// __nanosleep; after `limit` polls (kSpinLimit: about a second) it raises *err
// and returns false, and every other block leaves at its next poll.
// `phantom` counts blocks that never arrive: with phantom > 0 the word can
// never flip, so every wait runs out.  Only the wait-expiry test sets it (with
// a short limit), to check that an expired wait reaches the host as an error.
__device__ __forceinline__ bool grid_sync_flip(unsigned int* word, int* err, long long limit = kSpinLimit,
                                               unsigned int phantom = 0) {
  __syncthreads();
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    const unsigned int nblk = gridDim.x * gridDim.y * gridDim.z + phantom;
    const unsigned int inc = (blockIdx.x | blockIdx.y | blockIdx.z) == 0 ? 0x80000000u - (nblk - 1) : 1u;
    __threadfence();
    const unsigned int seen = atomicAdd(word, inc);
    int ok = 1;
    long long spins = 0;
    while (((seen ^ *(volatile unsigned int*)word) & 0x80000000u) == 0) {
      if (++spins > limit || *(volatile int*)err != 0) {
        atomicExch(err, TP3D_ERR_TIMEOUT);
        ok = 0;
        break;
      }
      if (spins > 64) __nanosleep(64);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

inline int cuda_status(cudaError_t e) { return e == cudaSuccess ? TP3D_OK : TP3D_ERR_CUDA; }

// Programmatic dependent launch.  The solver loop's kernels begin with
// pdl_entry(): wait until the kernel before this one in the stream has
// completed and its writes are visible (every global access of the kernel
// comes after this), then let the next kernel's blocks be scheduled as this
// grid's last blocks run, so that its launch latency overlaps this kernel's
// tail.  A kernel launched without the programmatic-serialization attribute
// passes the wait at once.  Kernels with a grid barrier never use it.
__device__ __forceinline__ void pdl_entry() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Kernel launch, with the programmatic-serialization attribute when pdl is
// set (the kernel must begin with pdl_entry()).
template <typename... P, typename... A>
inline cudaError_t launch_kernel(bool pdl, void (*kern)(P...), dim3 grid, dim3 block, size_t smem,
                                 cudaStream_t st, A&&... args) {
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, static_cast<A&&>(args)...);
}

// The same for a kernel given as a function pointer and an argument array.
inline cudaError_t launch_kernel_c(bool pdl, const void* kern, dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                                   void** args) {
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelExC(&cfg, kern, args);
}

// Process-wide count of kernel launches issued by this library (graph
// replays add the graph's kernel-node count).
void add_launches(long long n);

// Raises a kernel's dynamic shared-memory limit to the most the device allows
// it (the opt-in maximum less its static shared memory), once per process and
// kernel, under a lock: later calls change nothing, so no thread alters a
// kernel's attribute while another launches it (solvers are created and driven
// from several host threads).  TP3D_ERR_ARG if `bytes` exceeds that limit.
int ensure_dynamic_smem(const void* func, int bytes);
template <typename... P>
inline int ensure_dynamic_smem(void (*func)(P...), size_t bytes) {
  return ensure_dynamic_smem(reinterpret_cast<const void*>(func), (int)bytes);
}

}  // namespace tp3d

#define TP3D_CHECK(expr)                            \
  do {                                              \
    cudaError_t _e = (expr);                        \
    if (_e != cudaSuccess) {                        \
      tp3d_set_last_error(cudaGetErrorString(_e));  \
      return TP3D_ERR_CUDA;                         \
    }                                               \
  } while (0)

#define TP3D_CHECK_LAUNCH() TP3D_CHECK(cudaGetLastError())

extern "C" void tp3d_set_last_error(const char* msg);
