// File-scope device storage of the allocation-free J/K entry point
// (igpu_jk_device_static).  Kept in its own module so that, with lazy module
// loading, the storage is reserved only in processes that use that entry.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "noalloc.hpp"

namespace igpu {

namespace {
constexpr size_t SCRATCH_DOUBLES = STATIC_SCRATCH_DOUBLES;
constexpr size_t BOUNDS_DOUBLES = STATIC_BOUNDS_DOUBLES;
constexpr int MAX_LAUNCHES = STATIC_MAX_LAUNCHES;

__device__ __align__(256) double g_scratch[SCRATCH_DOUBLES];
__device__ __align__(256) double g_bounds[BOUNDS_DOUBLES];
__device__ __align__(256) unsigned long long g_work[MAX_LAUNCHES];

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
    // addresses resolved once per device
    void* p = nullptr;
    if ((e = cudaGetSymbolAddress(&p, g_scratch)) != cudaSuccess) return e;
    b.scratch = static_cast<double*>(p);
    if ((e = cudaGetSymbolAddress(&p, g_bounds)) != cudaSuccess) return e;
    b.bounds = static_cast<double*>(p);
    if ((e = cudaGetSymbolAddress(&p, g_work)) != cudaSuccess) return e;
    b.work = static_cast<unsigned long long*>(p);
    b.scratch_doubles = SCRATCH_DOUBLES;
    b.bounds_doubles = BOUNDS_DOUBLES;
    b.max_launches = MAX_LAUNCHES;
  }
  *out = b;
  return cudaSuccess;
}

}  // namespace igpu
