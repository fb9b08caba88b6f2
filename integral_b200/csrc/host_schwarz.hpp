// Exact Schwarz bounds (host_schwarz.cpp on the host, schwarz_dev.cu on the
// device, both running schwarz_core.cuh): the diagonal quartets (ij|ij)
// evaluated with the reference's arithmetic, bit for bit, wherever its Auto
// engine policy picks Obara-Saika / Head-Gordon-Pople.
#pragma once
#include <utility>
#include <vector>

#include "schwarz_core.cuh"

namespace igpu {

// One shell as the reference engine sees it: raw exponents, effective
// coefficients (src/shell.rs:182-187) and, for a spherical shell, its
// (2l+1) x n_cart transform with the normalisation ratio folded in
// (src/spherical.rs:37-48); c2s == nullptr for a Cartesian shell.
struct SchwarzShell {
  int l = 0;
  double center[3] = {0.0, 0.0, 0.0};
  std::vector<double> exps, coefs;
  const double* c2s = nullptr;
};

// src/integrals.rs:374-388: does Auto pick OS/HGP for bra degree ne, ket
// degree nf and contraction degree `degree` (the product of the four raw
// primitive counts)?
bool auto_picks_os(int ne, int nf, long long degree);

// Q = sqrt(max |(mu nu|mu nu)|) of shells (si, sj) in that order
// (src/integrals.rs:850-860).  Returns false, leaving q untouched, when
// Auto picks the Rys engine for the quartet.
bool schwarz_exact(const SchwarzShell& si, const SchwarzShell& sj, double& q);

// schwarz_exact over a list of ordered shell pairs on `nthreads` host
// threads (<= 0: all hardware threads); done[x] = 1 where q[x] was set.
void schwarz_exact_many(const std::vector<SchwarzShell>& shells, const std::vector<std::pair<int, int>>& pairs,
                        std::vector<double>& q, std::vector<unsigned char>& done, int nthreads);

// Inputs of the shared evaluation (schwarz_core.cuh): the Boys table and its
// constants (host pointers), the work-array layout of the class (li, lj) for
// at most maxpp primitive pairs (eoff receives the e-offset table the
// layout's eoff must point to), and the kappa of every primitive
// combination of (si, sj), si outer.
sc::BoysDev schwarz_boys_view();
const std::vector<double>& schwarz_boys_table();
sc::SClass schwarz_class_layout(int li, int lj, int maxpp, std::vector<int>& eoff);
void schwarz_kappa(const SchwarzShell& si, const SchwarzShell& sj, double* out);

}  // namespace igpu
