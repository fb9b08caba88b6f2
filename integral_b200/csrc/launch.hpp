// Host-callable launchers of the device code (kernels.cu, class_tu.cu).
#pragma once
#include <cuda_runtime.h>

#include "igpu_internal.hpp"

namespace igpu {

// Highest shell l of the compiled quartet-kernel classes.
#ifndef KERNEL_MAX_L
#define KERNEL_MAX_L 2
#endif

struct KernelEntry {
  void (*k64)(KernelArgs) = nullptr;
  void (*k32)(KernelArgs) = nullptr;
  int team = 1;          // lanes per quartet
  int smem64 = 0;        // dynamic shared memory per 128-thread block
  int smem32 = 0;
  size_t slot = 0;       // scratch doubles per team
  bool valid = false;
};

// Highest shell l of the compiled gradient classes.
#ifndef GRAD_KERNEL_MAX_L
#define GRAD_KERNEL_MAX_L 3
#endif

// Every class translation unit (class_tu.cu, grad_tu.cu: one per bra pair
// class, or one per (bra, ket) class for the largest bras) adds itself at
// load time: `reg` fills its entries of the value or gradient table, `up`
// uploads the constant tables of its device module.
using ClassRegFn = void (*)(KernelEntry* tab, int npc);
using ConstUpFn = cudaError_t (*)(const ConstData&);
int add_class_unit(bool grad, ClassRegFn reg, ConstUpFn up);

int kernel_npc();
// Gradient kernel of the class (pcb | pck), same conventions; the entry's
// slot is the gradient scratch per team.
const KernelEntry* grad_entry(int pcb, int pck);
// Entry of the class (pcb | pck), pair classes pc = l_a(l_a+1)/2 + l_b with
// l_a >= l_b and pcb >= pck; nullptr when the class is not compiled.
const KernelEntry* kernel_entry(int pcb, int pck);
cudaError_t upload_all_constants(const ConstData& c);
int blocks_per_sm(const KernelEntry* e, bool fp32);
cudaError_t launch_quartets(const KernelEntry* e, bool fp32, int grid, const KernelArgs& args,
                            cudaStream_t stream);
cudaError_t launch_shell_block_max(const double* D, int nmat, const DevShell* sh, int nsh, int nao,
                                   int symmetrise, double* out, cudaStream_t s);
cudaError_t launch_symmetrize_add(const double* H, double* out, int nmat, int nao, cudaStream_t s);
cudaError_t launch_to_float(const double* in, float* out, size_t n, cudaStream_t s);
cudaError_t launch_asym_count(const double* D, int nmat, int nao, unsigned long long* flag, cudaStream_t s);
// Molecule batches (plan_batch.cpp): matrices of molecule m at m*P*(P+1),
// row stride P; shell blocks at m*S*(S+1), row stride S.
cudaError_t launch_batch_block_max(const double* D, const DevShell* sh, int nmol, int S, int P, int symmetrise,
                                   double* out, cudaStream_t s);
cudaError_t launch_batch_symmetrize_add(const double* H, double* out, int nmol, int P, cudaStream_t s);

}  // namespace igpu
