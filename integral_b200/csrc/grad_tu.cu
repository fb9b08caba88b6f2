// Gradient kernels of one bra pair class: compiled once per PCB (with
// -DPCB=<n>, pair class pc = l_a(l_a+1)/2 + l_b of the evaluation bra), it
// instantiates the FP64 and FP32 gradient kernels of every ket class
// pck <= PCB and exports their registration and its module constants.
#include <utility>

#include "grad_kernel.cuh"
#include "launch.hpp"

#ifndef PCB
#error "compile with -DPCB=<bra pair class>"
#endif

#define IGPU_CAT2(a, b) a##b
#define IGPU_CAT(a, b) IGPU_CAT2(a, b)

namespace igpu {
namespace {

template <int PCK>
void register_one(KernelEntry* tab, int npc) {
  constexpr int LA = pc_la(PCB), LB = pc_lb(PCB), LC = pc_la(PCK), LD = pc_lb(PCK);
  using G64 = GradShape<LA, LB, LC, LD, double>;
  using G32 = GradShape<LA, LB, LC, LD, float>;
  KernelEntry e;
  e.k64 = grad_kernel<LA, LB, LC, LD, double>;
  e.k32 = grad_kernel<LA, LB, LC, LD, float>;
  e.team = G64::T;
  e.smem64 = (128 / G64::T) * G64::SMEM_PER_TEAM * (int)sizeof(double);
  e.smem32 = (128 / G32::T) * G32::SMEM_PER_TEAM * (int)sizeof(float);
  e.slot = grad_slot_layout(LA, LB, LC, LD).total;
  e.valid = true;
  tab[PCB * npc + PCK] = e;
}

template <int... I>
void register_all(KernelEntry* tab, int npc, std::integer_sequence<int, I...>) {
  (register_one<I>(tab, npc), ...);
}

}  // namespace

void IGPU_CAT(register_grad_classes_, PCB)(KernelEntry* tab, int npc) {
  register_all(tab, npc, std::make_integer_sequence<int, PCB + 1>{});
}

cudaError_t IGPU_CAT(upload_grad_constants_, PCB)(const ConstData& c) { return upload_module_constants(c); }

}  // namespace igpu
