// File-scope device storage behind the allocation-free J/K entry point
// igpu_jk_device_static (noalloc.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

namespace igpu {

// Capacities: team scratch 64 MiB, density shell-block bounds 16 MiB
// (ndens * nsh^2 doubles), one work counter per class launch.
constexpr size_t STATIC_SCRATCH_DOUBLES = size_t(8) << 20;
constexpr size_t STATIC_BOUNDS_DOUBLES = size_t(2) << 20;
constexpr int STATIC_MAX_LAUNCHES = 1024;

struct StaticBufs {
  double* scratch = nullptr;
  size_t scratch_doubles = 0;
  double* bounds = nullptr;
  size_t bounds_doubles = 0;
  unsigned long long* work = nullptr;
  int max_launches = 0;
};

// Addresses of that storage on the current device, resolved once per device
// with cudaGetSymbolAddress (nothing is allocated).
cudaError_t static_buffers(StaticBufs* out);

}  // namespace igpu
