// ORACLE — test infrastructure only (see oracle.hpp).
#pragma once
#include <array>
#include <cstdint>
#include <vector>

#include "oracle.hpp"

namespace oracle {

uint64_t splitmix64(uint64_t x);
// Order-independent identity of one screened canonical quartet (i >= j,
// k >= l, (kl) <= (ij)) with its density mask; summed (mod 2^64) over the
// screened list it fingerprints the list.
uint64_t quartet_key(int i, int j, int k, int l, uint64_t mask);

struct QuartetSink {
  uint64_t count = 0;
  uint64_t hash = 0;
  std::vector<std::array<int, 4>>* list = nullptr;
  std::vector<uint64_t>* masks = nullptr;
  void add(int i, int j, int k, int l, uint64_t mask) {
    count += 1;
    hash += quartet_key(i, j, k, l, mask);
    if (list) list->push_back({i, j, k, l});
    if (masks) masks->push_back(mask);
  }
};

struct JKArgs {
  int ndens = 0;
  const double* D[64];
  const double* bounds[64];
  double* J[64];
  double* K[64];
  double threshold = 0.0;
  bool want_k = true;
  bool count_only = false;
};

struct DirectPlan {
  const Basis& basis;
  Engine engine;
  std::vector<double> schwarz;
  std::vector<std::array<int, 2>> pairs;
  DirectPlan(const Basis& b, Engine e);
  std::vector<double> density_bounds(const double* d) const;
  void accumulate_bra_pair(int i, int j, const JKArgs& a, QuartetSink* sink) const;
  void scatter_block(const int idx[4], const double* block, uint64_t mask, const JKArgs& a) const;
};

struct GradTerm {
  double factor;
  const double* left;
  const double* right;
};
struct BoundedTerm {
  GradTerm term;
  std::vector<double> left_max, right_max;
};
struct GradDensity {
  std::vector<BoundedTerm> coulomb, exchange;
  double block_bound(int nsh, int i, int j, int k, int l) const;
};

struct GradPlan {
  const Basis& basis;
  Engine engine;
  std::vector<std::vector<double>> eff_2a;
  std::vector<std::vector<double>> s2c;
  std::vector<std::vector<PrimPair>> pair_first_2a, pair_second_2a;
  std::vector<double> schwarz;
  GradPlan(const Basis& b, Engine e);
  std::vector<double> shell_block_max(const double* m) const;
  GradDensity density(const std::vector<GradTerm>& coul, const std::vector<GradTerm>& exch) const;
  std::vector<double> weight_block(const int idx[4], double degeneracy, const GradDensity& d) const;
  void shifted_block(const int idx[4], int pos, int lp, bool weighted, bool use_rys,
                     double* out) const;
  void quartet(const int idx[4], double degeneracy, const GradDensity& d, double* out) const;
  void contract_weights(const int idx[4], const std::vector<double>& w, double* out) const;
  void dense_contract(const double* gamma, double* out) const;
  void accumulate_bra_pair(int i, int j, const GradDensity& d, double threshold, double* out,
                           QuartetSink* sink, bool count_only) const;
};

void run_jk(const DirectPlan& plan, const JKArgs& a, const std::vector<int>& bras, int nthreads,
            QuartetSink* sink);
void run_grad(const GradPlan& plan, const GradDensity& dens, double threshold,
              const std::vector<int>& bras, int nthreads, double* out, QuartetSink* sink,
              bool count_only);

}  // namespace oracle
