// Library-wide C ABI helpers: error reporting and version.
#include <atomic>
#include <string>

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
}  // namespace tp3d

extern "C" long long tp3d_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }
