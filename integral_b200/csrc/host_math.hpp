#pragma once
#include <array>
#include <vector>

#include "igpu_internal.hpp"

namespace igpu {

double ipow(double a, int b);
double shell_norm(double alpha, int l);
double effective_coeff(double alpha, double coef, int l);
double monomial_to_raw(int l);
std::vector<std::array<int, 3>> cart_comps(int l);
std::vector<double> c2s_effective(int l);

struct RysTables {
  std::vector<RysMeta> meta;     // index n = 1..MAX_ROOTS
  std::vector<double> coef;      // per n at meta[n].off: [(sub*n + i)*2 + {0,1}][17]
  double lag_x[MAX_ROOTS * MAX_ROOTS] = {0};
  double lag_w[MAX_ROOTS * MAX_ROOTS] = {0};
};
const RysTables& rys_tables();

}  // namespace igpu
