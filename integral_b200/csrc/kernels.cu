// Registry of the per-class quartet kernels (compiled in class_tu.cu, one
// module per bra pair class) and the small utility kernels (density
// shell-block bounds, symmetry check).  The host plan (plan*.cpp) calls only
// the functions declared in launch.hpp.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "launch.hpp"

namespace igpu {

constexpr int NPC = (KERNEL_MAX_L + 1) * (KERNEL_MAX_L + 2) / 2;
constexpr int GNPC = (GRAD_KERNEL_MAX_L + 1) * (GRAD_KERNEL_MAX_L + 2) / 2;

namespace {
struct ClassUnit {
  bool grad;
  ClassRegFn reg;
  ConstUpFn up;
};
std::vector<ClassUnit>& class_units() {
  static std::vector<ClassUnit> v;
  return v;
}
}  // namespace

int add_class_unit(bool grad, ClassRegFn reg, ConstUpFn up) {
  class_units().push_back({grad, reg, up});
  return (int)class_units().size();
}

static KernelEntry g_table[NPC * NPC];
static KernelEntry g_grad_table[GNPC * GNPC];
static std::once_flag g_once, g_grad_once;

int kernel_npc() { return NPC; }

static void set_smem_limits(KernelEntry* tab, int n) {
  for (int q = 0; q < n; ++q) {
    KernelEntry& e = tab[q];
    if (!e.valid) continue;
    cudaFuncSetAttribute(reinterpret_cast<const void*>(e.k64), cudaFuncAttributeMaxDynamicSharedMemorySize, e.smem64);
    cudaFuncSetAttribute(reinterpret_cast<const void*>(e.k32), cudaFuncAttributeMaxDynamicSharedMemorySize, e.smem32);
  }
}

const KernelEntry* grad_entry(int pcb, int pck) {
  std::call_once(g_grad_once, [] {
    for (const ClassUnit& u : class_units())
      if (u.grad) u.reg(g_grad_table, GNPC);
    set_smem_limits(g_grad_table, GNPC * GNPC);
  });
  if (pcb < 0 || pck < 0 || pcb >= GNPC || pck >= GNPC || pcb < pck) return nullptr;
  const KernelEntry* e = &g_grad_table[pcb * GNPC + pck];
  return e->valid ? e : nullptr;
}

const KernelEntry* kernel_entry(int pcb, int pck) {
  std::call_once(g_once, [] {
    for (const ClassUnit& u : class_units())
      if (!u.grad) u.reg(g_table, NPC);
    set_smem_limits(g_table, NPC * NPC);
  });
  if (pcb < 0 || pck < 0 || pcb >= NPC || pck >= NPC || pcb < pck) return nullptr;
  const KernelEntry* e = &g_table[pcb * NPC + pck];
  return e->valid ? e : nullptr;
}

cudaError_t upload_all_constants(const ConstData& c) {
  for (const ClassUnit& u : class_units()) {
    cudaError_t e = u.up(c);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

int blocks_per_sm(const KernelEntry* e, bool fp32) {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, reinterpret_cast<const void*>(fp32 ? e->k32 : e->k64), 128,
                                                fp32 ? e->smem32 : e->smem64);
  return n < 1 ? 1 : n;
}

cudaError_t launch_quartets(const KernelEntry* e, bool fp32, int grid, const KernelArgs& args,
                            cudaStream_t stream) {
  auto k = fp32 ? e->k32 : e->k64;
  int smem = fp32 ? e->smem32 : e->smem64;
  k<<<grid, 128, smem, stream>>>(args);
  return cudaGetLastError();
}

// ------------------------------------------------------------ utilities

// max |M| over every ordered shell block (src/direct.rs:103-125); one thread
// per (matrix, i, j).  With `symmetrise`, block (i,j) takes the max of (i,j)
// and (j,i) (src/direct_grad.rs:292-312).
__global__ void shell_block_max_kernel(const double* __restrict__ D, int nmat, const DevShell* __restrict__ sh,
                                       int nsh, int nao, int symmetrise, double* __restrict__ out) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t per = (size_t)nsh * nsh;
  if (t >= per * nmat) return;
  const int d = (int)(t / per);
  const int r = (int)(t % per);
  const int i = r / nsh, j = r % nsh;
  const double* M = D + (size_t)d * nao * nao;
  const DevShell si = sh[i], sj = sh[j];
  double mx = 0.0;
  for (int a = 0; a < si.nfunc; ++a)
    for (int b = 0; b < sj.nfunc; ++b) mx = fmax(mx, fabs(M[(size_t)(si.off + a) * nao + sj.off + b]));
  if (symmetrise)
    for (int a = 0; a < sj.nfunc; ++a)
      for (int b = 0; b < si.nfunc; ++b) mx = fmax(mx, fabs(M[(size_t)(sj.off + a) * nao + si.off + b]));
  out[t] = mx;
}

cudaError_t launch_shell_block_max(const double* D, int nmat, const DevShell* sh, int nsh, int nao,
                                   int symmetrise, double* out, cudaStream_t s) {
  const size_t n = (size_t)nsh * nsh * nmat;
  if (n == 0) return cudaSuccess;
  shell_block_max_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(D, nmat, sh, nsh, nao, symmetrise, out);
  return cudaGetLastError();
}

// out[d] += (H[d] + H[d]^T) / 2: the symmetric J/K from one-orientation
// accumulators.
__global__ void symmetrize_add_kernel(const double* __restrict__ H, double* __restrict__ out, int nmat, int nao) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t n2 = (size_t)nao * nao;
  if (t >= n2 * nmat) return;
  const size_t d = t / n2, r = (t % n2) / nao, c = t % nao;
  const double* M = H + d * n2;
  out[t] += 0.5 * (M[r * nao + c] + M[c * nao + r]);
}

cudaError_t launch_symmetrize_add(const double* H, double* out, int nmat, int nao, cudaStream_t s) {
  const size_t n = (size_t)nao * nao * nmat;
  if (n == 0) return cudaSuccess;
  symmetrize_add_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(H, out, nmat, nao);
  return cudaGetLastError();
}

// out[i] = (float)in[i]: the FP32 copy of the densities read by the FP32
// launches of the mixed J/K path.
__global__ void to_float_kernel(const double* __restrict__ in, float* __restrict__ out, size_t n) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = (float)in[t];
}

cudaError_t launch_to_float(const double* in, float* out, size_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  to_float_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(in, out, n);
  return cudaGetLastError();
}

// flag[0] += 1 for every element with M[r][c] != M[c][r] (bitwise compare).
__global__ void asym_count_kernel(const double* __restrict__ D, int nmat, int nao, unsigned long long* flag) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t n2 = (size_t)nao * nao;
  if (t >= n2 * nmat) return;
  const size_t d = t / n2, r = (t % n2) / nao, c = t % nao;
  if (c <= r) return;
  const double* M = D + d * n2;
  if (__double_as_longlong(M[r * nao + c]) != __double_as_longlong(M[c * nao + r])) atomicAdd(flag, 1ull);
}

cudaError_t launch_asym_count(const double* D, int nmat, int nao, unsigned long long* flag, cudaStream_t s) {
  const size_t n = (size_t)nao * nao * nmat;
  if (n == 0) return cudaSuccess;
  asym_count_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(D, nmat, nao, flag);
  return cudaGetLastError();
}

// ------------------------------------------------------ molecule batches
//
// A batch stores molecule m's nao x nao matrices with row stride P (the
// largest molecule's AO count) at m*P*(P+1), and its nsh x nsh shell-block
// bounds with row stride S (the largest shell count) at m*S*(S+1): the
// addresses that global indices m*P + local (AOs) and m*S + local (shells)
// give in a row-major P- or S-stride matrix.

// Shell-block maxima of every molecule's density (src/direct.rs:103-125;
// with `symmetrise` the max over (i,j) and (j,i), src/direct_grad.rs:292-312).
__global__ void batch_block_max_kernel(const double* __restrict__ D, const DevShell* __restrict__ sh, int nmol,
                                       int S, int P, int symmetrise, double* __restrict__ out) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t per = (size_t)S * S;
  if (t >= per * nmol) return;
  const int m = (int)(t / per);
  const int r = (int)(t % per);
  const int i = m * S + r / S, j = m * S + r % S;
  const DevShell si = sh[i], sj = sh[j];
  double mx = 0.0;
  for (int a = 0; a < si.nfunc; ++a)
    for (int b = 0; b < sj.nfunc; ++b) mx = fmax(mx, fabs(D[(size_t)(si.off + a) * P + sj.off + b]));
  if (symmetrise)
    for (int a = 0; a < sj.nfunc; ++a)
      for (int b = 0; b < si.nfunc; ++b) mx = fmax(mx, fabs(D[(size_t)(sj.off + a) * P + si.off + b]));
  out[(size_t)i * S + j] = mx;  // = m*S*(S+1) + i_local*S + j_local
}

cudaError_t launch_batch_block_max(const double* D, const DevShell* sh, int nmol, int S, int P, int symmetrise,
                                   double* out, cudaStream_t s) {
  const size_t n = (size_t)S * S * nmol;
  if (n == 0) return cudaSuccess;
  batch_block_max_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(D, sh, nmol, S, P, symmetrise, out);
  return cudaGetLastError();
}

// out_m += (H_m + H_m^T) / 2 for every molecule block.
__global__ void batch_symmetrize_add_kernel(const double* __restrict__ H, double* __restrict__ out, int nmol, int P) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t per = (size_t)P * P;
  if (t >= per * nmol) return;
  const size_t m = t / per, r = (t % per) / P, c = t % P;
  const size_t base = m * (size_t)P * (P + 1);
  out[base + r * P + c] += 0.5 * (H[base + r * P + c] + H[base + c * P + r]);
}

cudaError_t launch_batch_symmetrize_add(const double* H, double* out, int nmol, int P, cudaStream_t s) {
  const size_t n = (size_t)P * P * nmol;
  if (n == 0) return cudaSuccess;
  batch_symmetrize_add_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(H, out, nmol, P);
  return cudaGetLastError();
}

}  // namespace igpu
