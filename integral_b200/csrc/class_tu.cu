// One translation unit per bra pair class: compiled once per PCB (the pair
// class pc = l_a(l_a+1)/2 + l_b of the evaluation bra) with -DPCB=<n>, it
// instantiates the FP64 and FP32 quartet kernels of every ket class
// pck <= PCB and exports their registration and its module constants.
#include <utility>

#include "launch.hpp"
#include "quartet.cuh"

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
  KernelEntry e;
  e.k64 = quartet_kernel<LA, LB, LC, LD, double>;
  e.k32 = quartet_kernel<LA, LB, LC, LD, float>;
  e.team = TeamShape<LA, LB, LC, LD, double>::T;
  e.smem64 = (128 / e.team) * TeamShape<LA, LB, LC, LD, double>::TEAM_BYTES;
  e.smem32 = (128 / e.team) * TeamShape<LA, LB, LC, LD, float>::TEAM_BYTES;
  e.slot = slot_layout(LA, LB, LC, LD).total;
  e.valid = true;
  tab[PCB * npc + PCK] = e;
}

template <int... I>
void register_all(KernelEntry* tab, int npc, std::integer_sequence<int, I...>) {
  (register_one<I>(tab, npc), ...);
}

}  // namespace

void IGPU_CAT(register_classes_, PCB)(KernelEntry* tab, int npc) {
  register_all(tab, npc, std::make_integer_sequence<int, PCB + 1>{});
}

cudaError_t IGPU_CAT(upload_constants_, PCB)(const ConstData& c) { return upload_module_constants(c); }

}  // namespace igpu
