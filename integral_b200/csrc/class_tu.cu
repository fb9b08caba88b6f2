// One translation unit per bra pair class: compiled with -DPCB=<n> (the pair
// class pc = l_a(l_a+1)/2 + l_b of the evaluation bra), it instantiates the
// FP64 and FP32 quartet kernels of every ket class pck <= PCB, or, with
// -DPCK=<k> as well, of ket class k alone (the build splits the largest bra
// classes that way so that their kernels compile in parallel), and adds
// their registration and its module constants to the registry at load time.
#include <utility>

#include "launch.hpp"
#include "quartet.cuh"

#ifndef PCB
#error "compile with -DPCB=<bra pair class>"
#endif
#ifdef PCK
#define PCK_LO PCK
#define PCK_HI PCK
#else
#define PCK_LO 0
#define PCK_HI PCB
#endif

namespace igpu {
namespace {

template <int K>
void register_one(KernelEntry* tab, int npc) {
  constexpr int LA = pc_la(PCB), LB = pc_lb(PCB), LC = pc_la(K), LD = pc_lb(K);
  KernelEntry e;
  e.k64 = quartet_kernel<LA, LB, LC, LD, double>;
  e.k32 = quartet_kernel<LA, LB, LC, LD, float>;
  e.team = TeamShape<LA, LB, LC, LD, double>::T;
  e.smem64 = (128 / e.team) * TeamShape<LA, LB, LC, LD, double>::TEAM_BYTES;
  e.smem32 = (128 / e.team) * TeamShape<LA, LB, LC, LD, float>::TEAM_BYTES;
  e.slot = slot_layout(LA, LB, LC, LD).total;
  e.valid = true;
  tab[PCB * npc + K] = e;
}

template <int... I>
void register_all(KernelEntry* tab, int npc, std::integer_sequence<int, I...>) {
  (register_one<PCK_LO + I>(tab, npc), ...);
}

void register_unit(KernelEntry* tab, int npc) {
  register_all(tab, npc, std::make_integer_sequence<int, PCK_HI - PCK_LO + 1>{});
}

cudaError_t upload_unit(const ConstData& c) { return upload_module_constants(c); }

const int g_added = add_class_unit(false, register_unit, upload_unit);

}  // namespace
}  // namespace igpu
