// File-scope device storage of igpu_jk_device_static, the J/K entry point
// that allocates no device memory.  On the host, the array names below are
// host-side stand-ins, not device addresses: host code only ever passes
// the addresses that cudaGetSymbolAddress returns.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "noalloc.hpp"

namespace igpu {

constexpr size_t SCRATCH_DOUBLES = STATIC_SCRATCH_DOUBLES;
constexpr size_t BOUNDS_DOUBLES = STATIC_BOUNDS_DOUBLES;
constexpr int MAX_LAUNCHES = STATIC_MAX_LAUNCHES;

static __device__ __align__(256) double g_scratch[SCRATCH_DOUBLES];
static __device__ __align__(256) double g_bounds[BOUNDS_DOUBLES];
static __device__ __align__(256) unsigned long long g_work[MAX_LAUNCHES];

namespace {
std::mutex g_mutex;
std::vector<StaticBufs> g_bufs;  // per device; scratch == nullptr until resolved
}  // namespace

cudaError_t static_buffers(StaticBufs* out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_mutex);
  if ((int)g_bufs.size() <= dev) g_bufs.resize(dev + 1, StaticBufs{});
  StaticBufs& b = g_bufs[dev];
  if (!b.scratch) {
    // set-up, once per device, with that device current: the device
    // addresses of the three arrays (recorded only if all three resolve)
    void *ps = nullptr, *pb = nullptr, *pw = nullptr;
    if ((e = cudaGetSymbolAddress(&ps, g_scratch)) != cudaSuccess) return e;
    if ((e = cudaGetSymbolAddress(&pb, g_bounds)) != cudaSuccess) return e;
    if ((e = cudaGetSymbolAddress(&pw, g_work)) != cudaSuccess) return e;
    b.scratch = static_cast<double*>(ps);
    b.bounds = static_cast<double*>(pb);
    b.work = static_cast<unsigned long long*>(pw);
    b.scratch_doubles = SCRATCH_DOUBLES;
    b.bounds_doubles = BOUNDS_DOUBLES;
    b.max_launches = MAX_LAUNCHES;
  }
  *out = b;
  return cudaSuccess;
}

}  // namespace igpu
