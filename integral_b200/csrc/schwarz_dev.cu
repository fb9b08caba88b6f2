// Exact Schwarz bounds on the device: one thread, or one warp for the
// larger classes, per shell pair runs the shared evaluation of the
// reference's OS/HGP diagonal quartet (schwarz_core.cuh).  Compiled with -fmad=false, so that no product and sum
// fuse and every value rounds as on the host and in the reference.
#include "schwarz_dev.hpp"

namespace igpu {

__global__ void __launch_bounds__(128) schwarz_exact_kernel(sc::BoysDev B, sc::SClass C, SchwarzPairsDev in,
                                                            double* scratch, double* q_out, int team) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nthreads = gridDim.x * blockDim.x;
  const int lane = tid % team, t = tid / team, nteams = nthreads / team;
  // one thread per pair: interleaved slices; one warp per pair: contiguous
  const sc::Slice W = team == 1 ? sc::Slice{scratch + tid, (size_t)nthreads} : sc::Slice{scratch + (size_t)t * C.total, 1};
  const sc::Team T{lane, team};
  for (int x = t; x < in.npairs; x += nteams) {
    const int i = in.pi[x], j = in.pj[x];
    const int ci = in.c2s_off[i], cj = in.c2s_off[j];
    const double q = sc::sc_schwarz(B, C, W, T, in.centers + 3 * i, in.centers + 3 * j, in.nprim[i], in.nprim[j],
                                    in.exps + in.prim_off[i], in.coefs + in.prim_off[i], in.exps + in.prim_off[j],
                                    in.coefs + in.prim_off[j], in.kappa + in.kappa_off[x],
                                    ci >= 0 ? in.c2s + ci : nullptr, cj >= 0 ? in.c2s + cj : nullptr);
    if (lane == 0) q_out[x] = q;
  }
}

cudaError_t launch_schwarz_exact(const sc::BoysDev& B, const sc::SClass& C, const SchwarzPairsDev& in,
                                 double* scratch, int grid, int team, double* q_out, cudaStream_t s) {
  if (in.npairs == 0) return cudaSuccess;
  if (team != 1 && team != 32) return cudaErrorInvalidValue;
  schwarz_exact_kernel<<<grid, 128, 0, s>>>(B, C, in, scratch, q_out, team);
  return cudaGetLastError();
}

}  // namespace igpu
