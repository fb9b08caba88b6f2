#include <string>

#include "grad.hpp"

int grad_host(igpu_plan*, const igpu_term*, int, const igpu_term*, int, const uint32_t*, size_t, double, int,
              double*) {
  return IGPU_ERR_UNSUPPORTED;
}
int grad_device(igpu_plan*, const igpu_term*, int, const igpu_term*, int, const uint32_t*, size_t, double, int,
                double*, void*) {
  return IGPU_ERR_UNSUPPORTED;
}
