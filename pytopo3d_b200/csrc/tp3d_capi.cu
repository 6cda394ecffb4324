// Library-wide C ABI helpers: error reporting and version.
#include <atomic>
#include <mutex>
#include <string>
#include <unordered_map>

#include "tp3d_common.cuh"

namespace {
thread_local std::string g_last_error;
}

extern "C" void tp3d_set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }

extern "C" const char* tp3d_last_error(void) { return g_last_error.c_str(); }

extern "C" int tp3d_abi_version(void) { return 1; }

namespace {
std::atomic<long long> g_launches{0};
}
namespace tp3d {
void add_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int ensure_dynamic_smem(const void* func, int bytes) {
  static std::mutex m;
  static std::unordered_map<const void*, int> limit;
  std::lock_guard<std::mutex> g(m);
  auto it = limit.find(func);
  if (it != limit.end() && it->second >= bytes) return TP3D_OK;
  int dev = 0, optin = 0;
  cudaFuncAttributes fa{};
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
      cudaFuncGetAttributes(&fa, func) != cudaSuccess)
    return TP3D_ERR_CUDA;
  const int most = optin - (int)fa.sharedSizeBytes;  // the kernel's static shared memory counts too
  const cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
  if (e != cudaSuccess) {
    tp3d_set_last_error(cudaGetErrorString(e));
    return TP3D_ERR_CUDA;
  }
  limit[func] = most;
  return bytes <= most ? TP3D_OK : TP3D_ERR_ARG;
}
}  // namespace tp3d

extern "C" long long tp3d_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }
