// Exact Schwarz bounds on the device: one thread per shell pair runs the
// shared evaluation of the reference's OS/HGP diagonal quartet
// (schwarz_core.cuh).  Compiled with -fmad=false, so that no product and sum
// fuse and every value rounds as on the host and in the reference.
#include "schwarz_dev.hpp"

namespace igpu {

__global__ void __launch_bounds__(128) schwarz_exact_kernel(sc::BoysDev B, sc::SClass C, SchwarzPairsDev in,
                                                            double* scratch, double* q_out) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nthreads = gridDim.x * blockDim.x;
  const sc::Slice W{scratch + tid, (size_t)nthreads};
  for (int x = tid; x < in.npairs; x += nthreads) {
    const int i = in.pi[x], j = in.pj[x];
    const int ci = in.c2s_off[i], cj = in.c2s_off[j];
    q_out[x] = sc::sc_schwarz(B, C, W, in.centers + 3 * i, in.centers + 3 * j, in.nprim[i], in.nprim[j],
                              in.exps + in.prim_off[i], in.coefs + in.prim_off[i], in.exps + in.prim_off[j],
                              in.coefs + in.prim_off[j], in.kappa + in.kappa_off[x],
                              ci >= 0 ? in.c2s + ci : nullptr, cj >= 0 ? in.c2s + cj : nullptr);
  }
}

cudaError_t launch_schwarz_exact(const sc::BoysDev& B, const sc::SClass& C, const SchwarzPairsDev& in,
                                 double* scratch, int grid, double* q_out, cudaStream_t s) {
  if (in.npairs == 0) return cudaSuccess;
  schwarz_exact_kernel<<<grid, 128, 0, s>>>(B, C, in, scratch, q_out);
  return cudaGetLastError();
}

}  // namespace igpu
