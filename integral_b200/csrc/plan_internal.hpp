// Internal header of the host plan: the plan object, its device buffers and
// task lists, and the helpers that the C-ABI entry points share.  The entry
// points are split by subsystem: plan.cpp (plan, Schwarz, launches,
// profiles), plan_jk.cpp (direct J/K), plan_dense.cpp (dense tensor,
// EriBuilder, screened tensor, blocks, packed tensor), plan_df.cpp (density
// fitting) and plan_grad.cpp (the gradient).  Included by those files only.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/integral_gpu.h"
#include "host_math.hpp"
#include "host_schwarz.hpp"
#include "launch.hpp"
#include "noalloc.hpp"
#include "schwarz_dev.hpp"

namespace igpu {
namespace host {
extern thread_local std::string g_err;

inline int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
inline int cuda_fail(cudaError_t e, const char* where) {
  g_err = std::string(where) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? IGPU_ERR_OUT_OF_MEMORY : IGPU_ERR_CUDA;
}
#define CK(expr)                                             \
  do {                                                       \
    cudaError_t _e = (expr);                                 \
    if (_e != cudaSuccess) return cuda_fail(_e, #expr);      \
  } while (0)

inline int pair_class(int la, int lb) { return la * (la + 1) / 2 + lb; }
inline int pc_la_host(int pc) {
  int la = 0;
  while ((la + 1) * (la + 2) / 2 <= pc) ++la;
  return la;
}

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t ensure(size_t count) {
    if (count <= n && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
    if (e == cudaSuccess) n = std::max<size_t>(count, 1);
    return e;
  }
  cudaError_t upload(const std::vector<T>& v, cudaStream_t s) {
    cudaError_t e = ensure(v.size());
    if (e != cudaSuccess || v.empty()) return e;
    return cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
  }
};

// One class-pair launch of the quartet kernels.
struct Launch {
  int pcb = 0, pck = 0;
  bool fp32 = false;
  int builder_swap = 0;
  int nbra = 0;
  unsigned long long total = 0;
  DevBuf<int> bra_pair, ket_start, own_kets;
  DevBuf<unsigned long long> prefix;
  const int* ket_list = nullptr;  // device Q-sorted pair list of the ket class
};

struct TaskSet {
  std::vector<std::unique_ptr<Launch>> launches;
};

// Per-launch counters, work counters, events and records of one run of a
// task set (run_tasks / collect_profile).
struct LaunchLog {
  DevBuf<Counters> counters;
  DevBuf<unsigned long long> work;
  std::vector<cudaEvent_t> events;
  std::vector<igpu_launch_record> profile;
  std::vector<size_t> profile_launch;
  ~LaunchLog() {
    for (cudaEvent_t ev : events) cudaEventDestroy(ev);
  }
};

// Mixed-precision J/K task lists kept per plan (see igpu_plan::mixed_keys).
constexpr size_t kMixedTaskSets = 4;

}  // namespace host
}  // namespace igpu


// the plan's members name these types unqualified
using namespace igpu;
using namespace igpu::host;

struct igpu_plan {
  int device = 0;
  int engine = 0;
  int nsh = 0, nao = 0, natom = 0, npairs = 0;
  // molecule batch (igpu_batch_*): shells of molecule m at global indices
  // m*nsh + local and AOs at m*nao + local, with nsh and nao the per-molecule
  // maxima, so that every row-major index the kernels form from them lands
  // in molecule m's own block at m*nao*(nao+1) (m*nsh*(nsh+1) for shell
  // blocks); pairs and quartets never cross molecules
  bool batch = false;
  // per class, per molecule: its run [first, end) of class_groups[class]
  std::vector<std::vector<std::pair<int, int>>> class_mol_groups;

  bool spherical_any = false;
  std::vector<DevShell> shells;
  std::vector<std::array<double, 3>> atoms;
  std::vector<PairD> pairs;            // canonical order p = tri(i, j)
  std::vector<PrimPairD> prims;
  std::vector<double> c2s;
  int c2s_off[GPU_MAX_L + 3] = {0};
  std::vector<std::vector<int>> class_pairs;  // per pair class: nprim desc, then Q desc
  std::vector<std::vector<std::pair<size_t, size_t>>> class_groups;  // equal-nprim runs
  std::vector<double> schwarz;               // nsh x nsh
  // the shells as the host Schwarz evaluation sees them; the upper triangle
  // Q[j][i] (j < i) is evaluated on the first igpu_schwarz call
  std::vector<SchwarzShell> sshells;
  size_t schwarz_exact_pairs = 0;  // canonical pairs whose Q is the host's exact value
  bool schwarz_upper_done = false;
  // device
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  DevBuf<DevShell> d_shells;
  DevBuf<PairD> d_pairs;
  DevBuf<PrimPairD> d_prims;
  DevBuf<PrimPairF> d_primsf;  // FP32 copy for the FP32 launches
  DevBuf<double> d_c2s;
  DevBuf<int> d_class_lists;
  std::vector<int> class_list_off;
  DevBuf<double> d_scratch;
  DevBuf<Counters> d_counters;
  DevBuf<double> d_schwarz_pair;
  // per-call device buffers
  DevBuf<double> d_D, d_J, d_K, d_bounds, d_dense, d_Jh, d_Kh;
  DevBuf<float> d_Df;  // FP32 copy of the densities (mixed J/K)
  DevBuf<unsigned long long> d_flag;
  DevBuf<unsigned> d_bitmap;
  std::map<std::pair<double, double>, std::unique_ptr<TaskSet>> jk_tasks;  // (threshold, fp64 cutoff)
  // mixed-precision keys in insertion order: their cutoff follows max|D|,
  // so every new density would add one; at most kMixedTaskSets are kept
  std::vector<std::pair<double, double>> mixed_keys;
  // chunk multiplier per J/K or gradient launch class (igpu_autotune_jk,
  // igpu_autotune_grad); tune_mult != 0
  // overrides every launch while the tuner measures
  std::map<int, int> tuned_mult;
  int tune_mult = 0;
  // blocks-per-SM cap of the grid per launch class (0: the occupancy limit);
  // tune_bps != 0 overrides every launch while the tuner measures (-1: the
  // occupancy limit)
  std::map<int, int> tuned_bps;
  int tune_bps = 0;
  std::unique_ptr<TaskSet> dense_tasks;
  double mixed_cutoff = 1e-3;
  // primitive screen of the FP32 launches of the mixed path: bound * max|D|
  // below this skips a primitive quartet (0: none)
  double mixed_prim_cut = 1e-15;
  double erf_omega = 0.0;  // 0: Coulomb; > 0: erf(omega r)/r for every later call
  bool all_spherical = false;
  igpu_stats last{};
  // the launch log of the last J/K or gradient call; a molecule batch logs
  // its gradient phase in log2 (cur_log selects the one run_tasks fills)
  LaunchLog log, log2;
  LaunchLog* cur_log = &log;
  // gradient: term matrices, their block maxima and the device term tables
  DevBuf<double> d_gmat, d_gmax, d_gfac, d_gout;
  DevBuf<const double*> d_gptr;
  // packed tensor: first AO-pair index of every canonical shell pair
  DevBuf<long long> d_packed_start;
  // density fitting: the auxiliary basis, attached after the main shells,
  // pairs and primitive pairs (their counts stay nsh, npairs, nprims_main)
  int nprims_main = 0;
  bool has_aux = false;
  int naux_sh = 0, naux = 0;
  std::vector<std::vector<int>> aux_class_pairs;  // per aux pair class: nprim desc, then Q desc
  std::vector<double> aux_q;                      // Schwarz factor per aux shell
  DevBuf<int> d_aux_lists;
  DevBuf<unsigned> d_fault;
};

namespace igpu {
namespace host {

// plan.cpp: the core every entry point shares
int ensure_constants(int dev);
size_t grid_for(const KernelEntry* e, bool fp32, unsigned long long total, int bps_cap = 0);
KernelArgs base_args(igpu_plan* P);
double model_flops_prim(int la, int lb, int lc, int ld);
double model_flops_quartet(int la, int lb, int lc, int ld, bool sph, int ndens, bool jk);
double model_flops_grad_prim(int la, int lb, int lc, int ld);
double model_flops_grad_quartet(int la, int lb, int lc, int ld, bool sph, int nterm_c, int nterm_x);
double mixed_split(double cutoff, double dmax);
double fp32_class_scale(int lmax);
int class_lmax(int pca, int pcb);
int tune_key(int pcb, int pck, bool fp32, bool grad);
void tune_record(igpu_plan* P, int m, bool grad, std::map<int, std::map<int, float>>& best);
void tune_keep(igpu_plan* P, const std::map<int, std::map<int, float>>& best, bool bps);
int tune_two_stage(igpu_plan* P, bool grad, const std::function<int()>& run);
size_t slot_with_acc(const KernelEntry* e, int pcb, const KernelArgs& A);
int run_tasks(igpu_plan* P, TaskSet& ts, KernelArgs A, cudaStream_t s, uint32_t& launches);
int collect_profile(igpu_plan* P, int ndens, bool jk, int grad_terms_c = -1, int grad_terms_x = 0);
std::unique_ptr<Launch> make_launch(igpu_plan* P, int pcb, int pck, bool fp32, const std::vector<int>& bras,
                                    const std::vector<int>& nket, const std::vector<int>& kstart,
                                    const int* ket_list_dev, int swap, cudaStream_t s, int& rc);
std::unique_ptr<Launch> owned_launch(igpu_plan* P, int pcb, int pck, const std::vector<int>& bras,
                                     const std::vector<int>& nket, const std::vector<int>& kets, int& rc);
int build_jk_tasks(igpu_plan* P, double tau, double fp64_cut, TaskSet& ts);
TaskSet* cached_tasks(igpu_plan* P, double threshold, double fp64_cut, int& rc);
int check_bra_subset(igpu_plan* P, const uint32_t* sub, size_t nsub, std::vector<unsigned>& bitmap,
                     bool accumulate);
int run_schwarz(igpu_plan* P);
cudaError_t upload_prims(igpu_plan* P);
int exact_schwarz(igpu_plan* P);
int exact_schwarz_pairs(igpu_plan* P, const std::vector<std::pair<int, int>>& pairs, std::vector<double>& q,
                        std::vector<unsigned char>& done);

}  // namespace host
}  // namespace igpu
