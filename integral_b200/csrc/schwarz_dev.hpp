// Exact Schwarz bounds on the device (schwarz_dev.cu), host interface.
#pragma once
#include <cuda_runtime.h>

#include "schwarz_core.cuh"

namespace igpu {

// Exact Schwarz bounds on the device (schwarz_dev.cu): the listed shell
// pairs (i, j) of one class (l_i, l_j), reference orientation, with the
// shells' centres, primitive counts and offsets into the raw exponents and
// effective coefficients, their c2s offsets (-1: Cartesian), and the host's
// kappa of every primitive combination of each pair (i outer).
struct SchwarzPairsDev {
  int npairs;
  const int* pi;
  const int* pj;
  const double* centers;
  const int* nprim;
  const int* prim_off;
  const double* exps;
  const double* coefs;
  const int* c2s_off;
  const double* c2s;
  const long long* kappa_off;
  const double* kappa;
};
// q_out[x] = Q of listed pair x, evaluated by teams of `team` lanes (1 or
// 32); the scratch holds grid * (128 / team) * C.total doubles.
cudaError_t launch_schwarz_exact(const sc::BoysDev& B, const sc::SClass& C, const SchwarzPairsDev& in,
                                 double* scratch, int grid, int team, double* q_out, cudaStream_t s);

}  // namespace igpu
