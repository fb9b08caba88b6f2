// Density-direct ERI gradient (DirectGradContractor) on the device.
#pragma once
#include <vector>

#include "../../include/integral_gpu.h"

namespace igpu {

// Host-side data the gradient driver keeps on the plan.
struct GradState {
  std::vector<double> expv;  // primitive exponents, shell order
  std::vector<double> eff;   // effective coefficients, shell order
};

}  // namespace igpu

int grad_host(igpu_plan* P, const igpu_term* coulomb, int ncoul, const igpu_term* exchange, int nexch,
              const uint32_t* bra_subset, size_t nsub, double threshold, int precision, double* out);
int grad_device(igpu_plan* P, const igpu_term* d_coulomb, int ncoul, const igpu_term* d_exchange, int nexch,
                const uint32_t* bra_subset, size_t nsub, double threshold, int precision, double* d_out,
                void* stream);
