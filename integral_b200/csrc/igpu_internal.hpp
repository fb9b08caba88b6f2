// Internal data layout shared by the host plan (plan*.cpp) and the device
// kernels (kernels.cu).  Everything here is plain data in device memory.
#pragma once
#include <cstddef>
#include <cstdint>

namespace igpu {

constexpr int MAX_L = 6;             // reference engine cap (src/engine/os.rs:34)
constexpr int MAX_GRAD_L = MAX_L - 1;
constexpr int GPU_MAX_L = 4;         // highest shell l with compiled quartet kernels
constexpr int MAX_ROOTS = 13;
constexpr int RYS_NC = 17;           // degree-16 Chebyshev series per root/weight
constexpr int MAX_DENS = 64;
constexpr int ADDR_TAB_DEG_HOST = 20;  // degrees of the device triple table

// One shell on the device.
struct DevShell {
  double cx, cy, cz;
  int l;
  int nprim;
  int off;       // first function (AO) index
  int nfunc;     // n_cart or 2l+1
  int atom;      // index into Basis::atoms()
  int spherical;
  int prim_off;  // first primitive in the exponent/coefficient arrays
  int pad;
};

// One primitive pair of a shell pair in evaluation orientation (first shell
// A, second shell B, l_A >= l_B), surviving the 1e-32 pair screen of the
// reference (src/engine/os_eri.rs:211-244).
struct PrimPairD {
  double zeta;       // alpha + beta
  double alpha;      // exponent on A (gradient raise on A)
  double beta;       // exponent on B
  double px, py, pz; // Gaussian product centre
  double pax, pay, paz;  // P - A
  double e;          // kappa * c_A * c_B (effective coefficients)
};

// FP32 copy of one primitive pair for the FP32 launches, rounded once at
// plan creation: the FP32 header then needs no double loads or conversions.
// P - Q of a quartet is formed as (A - C) + (PA - QC), with A - C (the
// evaluation shells' centres) rounded once per quartet, so no absolute
// coordinate enters an FP32 difference.
struct PrimPairF {
  float zeta, e;
  float pax, pay, paz;
  float alpha, beta;
  float pad;
};

// One canonical shell pair (i >= j in the reference's sense) with its
// evaluation orientation.  An auxiliary pair of density fitting (an aux shell
// with the unit s dummy, src/df.rs:1-37) has i = the aux shell's position in
// the aux basis, j = -1 and tri = -1.
struct PairD {
  int a, b;       // evaluation orientation shells (l_a >= l_b)
  int i, j;       // canonical shells (i >= j)
  int prim_off;   // into PrimPairD array
  int nprim;      // surviving primitive pairs
  int tri;        // i*(i+1)/2 + j
  int cls;        // pair class index (l_a*(l_a+1)/2 + l_b)
  double abx, aby, abz;  // A - B
  double q;       // Schwarz bound Q[i][j]
};

// Rys table metadata for n roots: finite branch T < t_hi uses n_sub equal
// subintervals of width `width`; coefficients at `off` laid out as
// [(sub*n + i)*2 + {0 root, 1 weight}][RYS_NC].
struct RysMeta {
  int n_sub;
  int off;
  double width;
  double t_hi;
};

// Task list of one class-pair launch: for each listed bra (position in the
// bra class' Q-sorted pair list) kets 0..nket-1 of the ket class' sorted
// list.  prefix[b] = sum of nket over earlier bras (64-bit).
struct TaskList {
  const int* bra_pair;          // pair index per task bra
  const int* ket_pairs;         // Q-sorted pair indices of the ket class
  const unsigned long long* prefix;  // nbra + 1 entries
  const int* ket_start;         // first ket position per bra (NULL = 0)
  int nbra;
  unsigned long long total;
};

// Constant tables every device module needs (uploaded per module).
struct ConstData {
  const int* addr_lxyz;
  int n_addr;
  const RysMeta* meta;   // MAX_ROOTS + 1 entries
  const double* lag_x;   // MAX_ROOTS x MAX_ROOTS
  const double* lag_w;
  const float* lag_xf;
  const float* lag_wf;
  const double* tab;     // device Chebyshev tables
  const float* tab_f;
};

// Output modes of the quartet kernels.
enum Mode : int {
  MODE_JK = 0,
  MODE_DENSE = 1,
  MODE_SCHWARZ = 2,
  MODE_BUILDER = 3,
  MODE_GRAD = 4,
  MODE_PACKED = 5,
  MODE_DF3 = 6,  // density fitting (mu nu|P): main pair x (aux shell, unit s)
  MODE_DF2 = 7,  // density fitting (P|Q): (aux shell, unit s) x (aux shell, unit s)
  MODE_BLOCK = 8,  // one shell-quartet block in a requested shell order
};

struct JKDev {
  const double* D;       // ndens x nao x nao
  const float* Df;       // its FP32 copy, read by the FP32 launches
  const double* bounds;  // ndens x nsh x nsh  (density_shell_bounds)
  double* J;             // symmetric: one-orientation accumulators J', K'
  double* K;             //   (J = (J' + J'^T)/2 added by the finalize pass)
  int ndens;
  int want_k;
  int symmetric;         // every density symmetric (bitwise)
  double threshold;
};

// Two-particle density of the gradient as product terms factor * L (x) R
// (GradDensityTerm, src/direct_grad.rs:21-25).  Per term: device pointers to
// the nao x nao matrices and to their symmetrised shell-block maxima
// (nsh x nsh, src/direct_grad.rs:292-312).  c* = Coulomb-type terms, x* =
// exchange-type terms.
struct GradDev {
  const double* const* cl;
  const double* const* cr;
  const double* const* cl_max;
  const double* const* cr_max;
  const double* cf;      // factors
  const double* const* xl;
  const double* const* xr;
  const double* const* xl_max;
  const double* const* xr_max;
  const double* xf;
  int ncoul, nexch;
  double threshold;
  double* out;           // natom x 3, dE/dR accumulated
};

struct Counters {
  unsigned long long quartets;
  unsigned long long hash;
  unsigned long long fp32_quartets;
  unsigned long long prim_quartets;
  unsigned long long skipped;
  unsigned long long pad[3];
};

// Everything a quartet kernel needs.
struct KernelArgs {
  const DevShell* shells;
  const PairD* pairs;
  const PrimPairD* prims;
  const PrimPairF* primsf;  // FP32 copy of prims (same order)
  const double* c2s;     // c2s matrices (ratio folded), c2s_off[l] into it
  int c2s_off[GPU_MAX_L + 3];
  int nsh;
  int nao;
  TaskList task;
  int mode;
  int fp32;              // this launch evaluates in FP32
  double* scratch;       // per-team slots for the post phase
  size_t slot_doubles;
  JKDev jk;
  GradDev grad;
  double* dense;         // nao^4 (MODE_DENSE / MODE_BUILDER); packed triangle (MODE_PACKED)
  const long long* packed_start;  // MODE_PACKED: first AO-pair index of every canonical shell pair
  double* schwarz_out;   // per pair Q (MODE_SCHWARZ)
  Counters* counters;
  int builder_swap;      // builder mode: requested bra is the evaluation ket
  const unsigned* bra_bitmap;  // optional: reference bra pairs to keep (bit per pair)
  unsigned long long* work_counter;  // next unclaimed task (dynamic chunks)
  unsigned long long chunk;          // tasks claimed per grab (per warp)
  size_t acc_offset;     // slot offset of the running bra-block J accumulators
  int kinds;             // 0 all shells Cartesian, 1 all spherical, 2 mixed
  double omega;          // 0: Coulomb 1/r; > 0: long-range erf(omega r)/r
  int naux;              // MODE_DF3 / MODE_DF2: auxiliary functions
  size_t dense_len;      // MODE_DF3 / MODE_DF2 / MODE_BLOCK: doubles in `dense`
  unsigned* store_fault; // MODE_DF3 / MODE_DF2 / MODE_BLOCK: set when an index falls outside `dense`
  int blk_shells[4];     // MODE_BLOCK: requested shells (i, j, k, l)
  int blk_dims[4];       // MODE_BLOCK: their function counts
  // FP32 launches of the mixed J/K path: a primitive quartet whose magnitude
  // bound |E_ab E_cd| 2 pi^{5/2} / (p q sqrt(p + q)) is below prim_cut is
  // skipped (0: every primitive quartet is evaluated)
  double prim_cut;
};

}  // namespace igpu
