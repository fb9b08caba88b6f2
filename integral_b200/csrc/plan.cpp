// Host plan and C ABI (include/integral_gpu.h).
//
// The plan mirrors the precompute of the reference's DirectContractor /
// DirectGradContractor / EriBuilder constructors (src/direct.rs:59-87,
// src/direct_grad.rs:180-247, src/eri_builder.rs:238-270): shell metadata,
// AO offsets, atoms, effective coefficients, c2s matrices, canonical shell
// pairs with their screened primitive-pair data, and the Schwarz bounds —
// the latter evaluated on the device at creation.  Canonical pairs are
// bucketed by angular class and sorted by Q so that, for a threshold tau,
// the kets accepted by Q_bra*Q_ket >= tau form a prefix of every bra's ket
// list; the per-class task lists are cached per threshold.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/integral_gpu.h"
#include "host_math.hpp"
#include "launch.hpp"
#include "noalloc.hpp"

using namespace igpu;

namespace {
thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* where) {
  g_err = std::string(where) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? IGPU_ERR_OUT_OF_MEMORY : IGPU_ERR_CUDA;
}
#define CK(expr)                                             \
  do {                                                       \
    cudaError_t _e = (expr);                                 \
    if (_e != cudaSuccess) return cuda_fail(_e, #expr);      \
  } while (0)

int pair_class(int la, int lb) { return la * (la + 1) / 2 + lb; }
int pc_la_host(int pc) {
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

std::mutex g_const_mutex;
std::vector<int> g_const_ready;  // per device
}  // namespace

struct igpu_plan {
  int device = 0;
  int engine = 0;
  int nsh = 0, nao = 0, natom = 0, npairs = 0;
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
  // device
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  DevBuf<DevShell> d_shells;
  DevBuf<PairD> d_pairs;
  DevBuf<PrimPairD> d_prims;
  DevBuf<double> d_c2s;
  DevBuf<int> d_class_lists;
  std::vector<int> class_list_off;
  DevBuf<double> d_scratch;
  DevBuf<Counters> d_counters;
  DevBuf<double> d_schwarz_pair;
  // per-call device buffers
  DevBuf<double> d_D, d_J, d_K, d_bounds, d_dense, d_Jh, d_Kh;
  DevBuf<unsigned long long> d_work;
  DevBuf<unsigned long long> d_flag;
  DevBuf<unsigned> d_bitmap;
  std::map<std::pair<double, double>, std::unique_ptr<TaskSet>> jk_tasks;  // (threshold, fp64 cutoff)
  // mixed-precision keys in insertion order: their cutoff follows max|D|,
  // so every new density would add one; at most kMixedTaskSets are kept
  std::vector<std::pair<double, double>> mixed_keys;
  // chunk multiplier per J/K launch class (igpu_autotune_jk); tune_mult != 0
  // overrides every launch while the tuner measures
  std::map<int, int> tuned_mult;
  int tune_mult = 0;
  std::unique_ptr<TaskSet> dense_tasks;
  double mixed_cutoff = 1e-4;
  double erf_omega = 0.0;  // 0: Coulomb; > 0: erf(omega r)/r for every later call
  bool all_spherical = false;
  igpu_stats last{};
  DevBuf<Counters> d_launch_counters;
  std::vector<cudaEvent_t> events;
  std::vector<igpu_launch_record> profile;
  std::vector<size_t> profile_launch;
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

namespace {

// Mixed-precision J/K task lists kept per plan (see igpu_plan::mixed_keys).
constexpr size_t kMixedTaskSets = 4;

// Upload the angular tables and the Rys tables to this device once.
int ensure_constants(int dev) {
  std::lock_guard<std::mutex> lk(g_const_mutex);
  if ((int)g_const_ready.size() <= dev) g_const_ready.resize(dev + 1, 0);
  if (g_const_ready[dev]) return IGPU_OK;
  const RysTables& T = rys_tables();
  std::vector<int> lxyz;
  for (int d = 0; d <= ADDR_TAB_DEG_HOST; ++d)
    for (auto& c : cart_comps(d)) lxyz.push_back(c[0] | (c[1] << 8) | (c[2] << 16));
  double* d_tab = nullptr;
  float* d_tab_f = nullptr;
  CK(cudaMalloc(&d_tab, T.coef.size() * sizeof(double)));
  CK(cudaMalloc(&d_tab_f, T.coef.size() * sizeof(float)));
  std::vector<float> tf(T.coef.begin(), T.coef.end());
  CK(cudaMemcpy(d_tab, T.coef.data(), T.coef.size() * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_tab_f, tf.data(), tf.size() * sizeof(float), cudaMemcpyHostToDevice));
  float lxf[MAX_ROOTS * MAX_ROOTS], lwf[MAX_ROOTS * MAX_ROOTS];
  for (int i = 0; i < MAX_ROOTS * MAX_ROOTS; ++i) {
    lxf[i] = (float)T.lag_x[i];
    lwf[i] = (float)T.lag_w[i];
  }
  ConstData c;
  c.addr_lxyz = lxyz.data();
  c.n_addr = (int)lxyz.size();
  c.meta = T.meta.data();
  c.lag_x = T.lag_x;
  c.lag_w = T.lag_w;
  c.lag_xf = lxf;
  c.lag_wf = lwf;
  c.tab = d_tab;
  c.tab_f = d_tab_f;
  CK(upload_all_constants(c));
  g_const_ready[dev] = 1;
  return IGPU_OK;
}

size_t grid_for(const KernelEntry* e, bool fp32, unsigned long long total) {
  static int nsm = 0;
  if (!nsm) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (nsm <= 0) nsm = 1;
  }
  const int teams_per_block = 128 / e->team;
  const unsigned long long need = (total + teams_per_block - 1) / teams_per_block;
  const unsigned long long cap = (unsigned long long)blocks_per_sm(e, fp32) * nsm;
  return (size_t)std::max<unsigned long long>(1, std::min(need, cap));
}

KernelArgs base_args(igpu_plan* P) {
  KernelArgs A;
  std::memset(&A, 0, sizeof(A));
  A.shells = P->d_shells.p;
  A.pairs = P->d_pairs.p;
  A.prims = P->d_prims.p;
  A.c2s = P->d_c2s.p;
  for (int l = 0; l < GPU_MAX_L + 3; ++l) A.c2s_off[l] = P->c2s_off[l];
  A.nsh = P->nsh;
  A.nao = P->nao;
  A.counters = P->d_counters.p;
  A.kinds = P->all_spherical ? 1 : (P->spherical_any ? 2 : 0);
  A.omega = P->erf_omega;
  return A;
}

// Fixed flop model of the reference's Rys formulation (src/engine/rys.rs:
// 137-309) per surviving primitive quartet: header, roots/weights by
// Clenshaw, per root the recurrence coefficients, per axis VRR + bra HRR +
// ket HRR, and the 4-flop assembly of every Cartesian element.
double model_flops_prim(int la, int lb, int lc, int ld) {
  auto nc = [](int l) { return (double)((l + 1) * (l + 2) / 2); };
  const int n = (la + lb + lc + ld) / 2 + 1, nb = la + lb, nk = lc + ld;
  const double N4 = nc(la) * nc(lb) * nc(lc) * nc(ld);
  const double per_root = 12.0 + 3.0 * (3.0 * (nb + 1) * (nk + 1) + 2.0 * lb * (nb + 1) * (nk + 1) +
                                        2.0 * ld * (la + 1) * (lb + 1) * (nk + 1)) +
                          4.0 * N4;
  return 40.0 + 2.0 * n * 34.0 + n * per_root;
}
// Per shell quartet: c2s of spherical shells (2 flops per multiply-add of
// each axis contraction) and the J/K contraction, 4 flops per element and
// density for each of the 8 permutation images.
double model_flops_quartet(int la, int lb, int lc, int ld, bool sph, int ndens, bool jk) {
  auto nc = [](int l) { return (double)((l + 1) * (l + 2) / 2); };
  double dims[4] = {nc(la), nc(lb), nc(lc), nc(ld)};
  const int ls[4] = {la, lb, lc, ld};
  double f = 0.0;
  if (sph)
    for (int a = 0; a < 4; ++a) {
      double rest = 1.0;
      for (int q = 0; q < 4; ++q)
        if (q != a) rest *= dims[q];
      const double out = 2.0 * ls[a] + 1.0;
      f += 2.0 * out * dims[a] * rest;
      dims[a] = out;
    }
  if (jk) f += 4.0 * 8.0 * dims[0] * dims[1] * dims[2] * dims[3] * ndens;
  return f;
}
// Gradient per primitive quartet: the reference's three raised and up to
// three lowered shifted classes (src/direct_grad.rs:431-470), each at the
// value model above.
double model_flops_grad_prim(int la, int lb, int lc, int ld) {
  double f = model_flops_prim(la + 1, lb, lc, ld) + model_flops_prim(la, lb + 1, lc, ld) +
             model_flops_prim(la, lb, lc + 1, ld);
  if (la > 0) f += model_flops_prim(la - 1, lb, lc, ld);
  if (lb > 0) f += model_flops_prim(la, lb - 1, lc, ld);
  if (lc > 0) f += model_flops_prim(la, lb, lc - 1, ld);
  return f;
}
// Gradient per shell quartet: the weight block (4 flops per Coulomb term and
// 10 per exchange term and element), its pull-back to Cartesian, and the
// dots of W with the six shifted blocks on three axes.
double model_flops_grad_quartet(int la, int lb, int lc, int ld, bool sph, int nterm_c, int nterm_x) {
  auto nc = [](int l) { return (double)((l + 1) * (l + 2) / 2); };
  const double W = nc(la) * nc(lb) * nc(lc) * nc(ld);
  double f = W * (4.0 * nterm_c + 10.0 * nterm_x) + 6.0 * 3.0 * 2.0 * W;
  if (sph) f += model_flops_quartet(la, lb, lc, ld, true, 0, false);
  return f;
}

// Key of a J/K launch class in the tuned-chunk table.
int tune_key(int pcb, int pck, bool fp32) { return (pcb * 64 + pck) * 2 + (fp32 ? 1 : 0); }

// Scratch doubles per team: the class slot plus, for symmetric J/K, the
// running bra-block accumulators (bra index + ndens blocks of the bra pair).
size_t slot_with_acc(const KernelEntry* e, int pcb, const KernelArgs& A) {
  if (A.mode != MODE_JK || !A.jk.symmetric) return e->slot;
  const int la = pc_la_host(pcb), lb = pcb - la * (la + 1) / 2;
  const size_t nab = (size_t)((la + 1) * (la + 2) / 2) * ((lb + 1) * (lb + 2) / 2);
  return e->slot + 1 + (size_t)A.jk.ndens * nab;
}

// Run every launch of a task set; quartet kernels only.  Per-launch device
// time and counters are kept for igpu_last_profile.
int run_tasks(igpu_plan* P, TaskSet& ts, KernelArgs A, cudaStream_t s, uint32_t& launches) {
  const bool grad = A.mode == MODE_GRAD;
  auto entry = [grad](int pcb, int pck) { return grad ? grad_entry(pcb, pck) : kernel_entry(pcb, pck); };
  size_t need = 0;
  for (auto& L : ts.launches) {
    if (L->total == 0) continue;
    const KernelEntry* e = entry(L->pcb, L->pck);
    if (!e) return fail(IGPU_ERR_UNSUPPORTED, "angular class not compiled for the GPU");
    need = std::max(need, grid_for(e, L->fp32, L->total) * (128 / e->team) * slot_with_acc(e, L->pcb, A));
  }
  CK(P->d_scratch.ensure(need));
  const size_t nl = ts.launches.size();
  CK(P->d_launch_counters.ensure(nl));
  CK(cudaMemsetAsync(P->d_launch_counters.p, 0, nl * sizeof(Counters), s));
  CK(P->d_work.ensure(nl));
  CK(cudaMemsetAsync(P->d_work.p, 0, nl * sizeof(unsigned long long), s));
  while (P->events.size() < 2 * nl) {
    cudaEvent_t ev;
    CK(cudaEventCreate(&ev));
    P->events.push_back(ev);
  }
  P->profile.clear();
  P->profile_launch.clear();
  for (size_t li = 0; li < nl; ++li) {
    Launch* L = ts.launches[li].get();
    if (L->total == 0) continue;
    const KernelEntry* e = entry(L->pcb, L->pck);
    const size_t grid = grid_for(e, L->fp32, L->total);
    A.scratch = P->d_scratch.p;
    A.slot_doubles = slot_with_acc(e, L->pcb, A);
    A.acc_offset = e->slot;
    A.work_counter = P->d_work.p + li;
    int mult = 16;
    if (P->tune_mult) {
      mult = P->tune_mult;
    } else if (A.mode == MODE_JK) {
      auto t = P->tuned_mult.find(tune_key(L->pcb, L->pck, L->fp32));
      if (t != P->tuned_mult.end()) mult = t->second;
    }
    A.chunk = (unsigned long long)(32 / e->team) * mult;
    if (A.counters) A.counters = P->d_launch_counters.p + li;
    A.task.bra_pair = L->bra_pair.p;
    A.task.ket_pairs = L->ket_list;
    A.task.prefix = L->prefix.p;
    A.task.ket_start = L->ket_start.n ? L->ket_start.p : nullptr;
    A.task.nbra = L->nbra;
    A.task.total = L->total;
    A.fp32 = L->fp32 ? 1 : 0;
    A.builder_swap = L->builder_swap;
    CK(cudaEventRecord(P->events[2 * li], s));
    CK(launch_quartets(e, L->fp32, (int)grid, A, s));
    CK(cudaEventRecord(P->events[2 * li + 1], s));
    ++launches;
    igpu_launch_record r{};
    r.la = pc_la_host(L->pcb);
    r.lb = L->pcb - r.la * (r.la + 1) / 2;
    r.lc = pc_la_host(L->pck);
    r.ld = L->pck - r.lc * (r.lc + 1) / 2;
    r.fp32 = L->fp32 ? 1 : 0;
    r.team = e->team;
    r.grid = (uint32_t)grid;
    r.tasks = L->total;
    r.chunk = (uint32_t)A.chunk;
    P->profile.push_back(r);
    P->profile_launch.push_back(li);
  }
  return IGPU_OK;
}

// After the stream is synchronised: per-launch times, counters, model flops.
int collect_profile(igpu_plan* P, int ndens, bool jk, int grad_terms_c = -1, int grad_terms_x = 0) {
  const size_t nl = P->profile.empty() ? 0 : P->profile_launch.back() + 1;
  std::vector<Counters> c(nl);
  if (nl) CK(cudaMemcpy(c.data(), P->d_launch_counters.p, nl * sizeof(Counters), cudaMemcpyDeviceToHost));
  P->last = igpu_stats{};
  for (size_t k = 0; k < P->profile.size(); ++k) {
    igpu_launch_record& r = P->profile[k];
    const size_t li = P->profile_launch[k];
    float ms = 0.f;
    cudaEventElapsedTime(&ms, P->events[2 * li], P->events[2 * li + 1]);
    r.ms = ms;
    r.quartets = c[li].quartets;
    r.prim_quartets = c[li].prim_quartets;
    if (grad_terms_c >= 0)
      r.model_flops = (double)r.prim_quartets * model_flops_grad_prim(r.la, r.lb, r.lc, r.ld) +
                      (double)r.quartets * model_flops_grad_quartet(r.la, r.lb, r.lc, r.ld, P->all_spherical,
                                                                    grad_terms_c, grad_terms_x);
    else
      r.model_flops = (double)r.prim_quartets * model_flops_prim(r.la, r.lb, r.lc, r.ld) +
                      (double)r.quartets * model_flops_quartet(r.la, r.lb, r.lc, r.ld, P->all_spherical, ndens, jk);
    P->last.quartets += c[li].quartets;
    P->last.quartet_hash += c[li].hash;
    P->last.quartets_fp32 += c[li].fp32_quartets;
    P->last.prim_quartets += c[li].prim_quartets;
    P->last.model_flops += r.model_flops;
    P->last.kernel_ms += ms;
  }
  P->last.launches = (uint32_t)P->profile.size();
  return IGPU_OK;
}

// Build one Launch from host vectors.
std::unique_ptr<Launch> make_launch(igpu_plan* P, int pcb, int pck, bool fp32, const std::vector<int>& bras,
                                    const std::vector<int>& nket, const std::vector<int>& kstart,
                                    const int* ket_list_dev, int swap, cudaStream_t s, int& rc) {
  auto L = std::make_unique<Launch>();
  L->pcb = pcb;
  L->pck = pck;
  L->fp32 = fp32;
  L->builder_swap = swap;
  std::vector<int> b;
  std::vector<int> ks;
  std::vector<unsigned long long> pre(1, 0);
  for (size_t x = 0; x < bras.size(); ++x) {
    if (nket[x] <= 0) continue;
    b.push_back(bras[x]);
    ks.push_back(kstart.empty() ? 0 : kstart[x]);
    pre.push_back(pre.back() + (unsigned long long)nket[x]);
  }
  L->nbra = (int)b.size();
  L->total = pre.back();
  L->ket_list = ket_list_dev;
  rc = IGPU_OK;
  cudaError_t e;
  if ((e = L->bra_pair.upload(b, s)) || (e = L->prefix.upload(pre, s))) {
    rc = cuda_fail(e, "task upload");
    return nullptr;
  }
  bool any_start = std::any_of(ks.begin(), ks.end(), [](int v) { return v != 0; });
  if (any_start && (e = L->ket_start.upload(ks, s))) {
    rc = cuda_fail(e, "task upload");
    return nullptr;
  }
  return L;
}

// Screened J/K task lists for threshold tau: for every class pair (CA >= CB)
// and bra of CA, the kets of CB with Q_bra*Q_ket >= tau (a prefix of the
// Q-sorted list; the upper triangle when CA == CB).  With fp64_cut > 0 the
// prefix is split: kets with Q_bra*Q_ket >= fp64_cut run in FP64, the rest in
// FP32.
int build_jk_tasks(igpu_plan* P, double tau, double fp64_cut, TaskSet& ts) {
  const int npc = (int)P->class_pairs.size();
  for (int ca = 0; ca < npc; ++ca)
    for (int cb = 0; cb <= ca; ++cb) {
      const auto& B = P->class_pairs[ca];
      const auto& K = P->class_pairs[cb];
      if (B.empty() || K.empty()) continue;
      std::vector<double> qk(K.size());
      for (size_t x = 0; x < K.size(); ++x) qk[x] = P->pairs[K[x]].q;
      // One segment per (bra, ket group of equal primitive-pair count): the
      // lanes of a warp then run equal primitive loops.  Within a group the
      // kets are Q-descending, so the accepted kets are a prefix.
      const auto& groups = P->class_groups[cb];
      std::vector<int> bras, n64, n32, st64, st32;
      for (size_t bp = 0; bp < B.size(); ++bp) {
        const double qb = P->pairs[B[bp]].q;
        for (const auto& grp : groups) {
          const size_t gs = grp.first, ge = grp.second;
          if (ca == cb && gs > bp) break;  // kets at class positions <= bp only
          size_t lo = gs, hi = ge;  // first ket with qb*qk < tau
          while (lo < hi) {
            size_t mid = (lo + hi) / 2;
            if (qb * qk[mid] >= tau)
              lo = mid + 1;
            else
              hi = mid;
          }
          size_t end = lo;
          if (ca == cb) end = std::min(end, bp + 1);
          if (end <= gs) continue;
          size_t split = end;
          if (fp64_cut > 0.0) {
            size_t l2 = gs, h2 = end;
            while (l2 < h2) {
              size_t mid = (l2 + h2) / 2;
              if (qb * qk[mid] >= fp64_cut)
                l2 = mid + 1;
              else
                h2 = mid;
            }
            split = l2;
          }
          bras.push_back(B[bp]);
          st64.push_back((int)gs);
          n64.push_back((int)(split - gs));
          st32.push_back((int)split);
          n32.push_back((int)(end - split));
        }
      }
      const int* klist = P->d_class_lists.p + P->class_list_off[cb];
      int rc;
      auto L64 = make_launch(P, ca, cb, false, bras, n64, st64, klist, 0, P->stream, rc);
      if (!L64) return rc;
      ts.launches.push_back(std::move(L64));
      if (fp64_cut > 0.0) {
        auto L32 = make_launch(P, ca, cb, true, bras, n32, st32, klist, 0, P->stream, rc);
        if (!L32) return rc;
        ts.launches.push_back(std::move(L32));
      }
    }
  return IGPU_OK;
}

// The task list of (threshold, fp64 cutoff), built on first use and cached.
// A mixed list's cutoff follows the maximum of the density (or term
// matrices), so only the kMixedTaskSets most recent mixed lists are kept;
// FP64 lists (cutoff 0, one per threshold) stay.  Every entry point
// synchronises before it returns, so an evicted list has no launch in
// flight.
TaskSet* cached_tasks(igpu_plan* P, double threshold, double fp64_cut, int& rc) {
  rc = IGPU_OK;
  const auto key = std::make_pair(threshold, fp64_cut);
  auto it = P->jk_tasks.find(key);
  if (it != P->jk_tasks.end()) return it->second.get();
  if (fp64_cut > 0.0 && P->mixed_keys.size() >= kMixedTaskSets) {
    P->jk_tasks.erase(P->mixed_keys.front());
    P->mixed_keys.erase(P->mixed_keys.begin());
  }
  auto ts = std::make_unique<TaskSet>();
  rc = build_jk_tasks(P, threshold, fp64_cut, *ts);
  if (rc) return nullptr;
  cudaError_t e = cudaStreamSynchronize(P->stream);
  if (e != cudaSuccess) {
    rc = cuda_fail(e, "task list upload");
    return nullptr;
  }
  TaskSet* out = ts.get();
  P->jk_tasks.emplace(key, std::move(ts));
  if (fp64_cut > 0.0) P->mixed_keys.push_back(key);
  return out;
}

int check_bra_subset(igpu_plan* P, const uint32_t* sub, size_t nsub, std::vector<unsigned>& bitmap) {
  bitmap.assign(((size_t)P->npairs + 31) / 32, 0u);
  for (size_t x = 0; x < nsub; ++x) {
    if (sub[x] >= (uint32_t)P->npairs) return fail(IGPU_ERR_NONCANONICAL_BRA, "bra pair index out of range");
    bitmap[sub[x] / 32] |= 1u << (sub[x] % 32);
  }
  return IGPU_OK;
}

int run_schwarz(igpu_plan* P) {
  // one (P|P) quartet per canonical pair, no screening
  TaskSet ts;
  const int npc = (int)P->class_pairs.size();
  for (int c = 0; c < npc; ++c) {
    const auto& B = P->class_pairs[c];
    if (B.empty()) continue;
    std::vector<int> nk(B.size(), 1), ks(B.size());
    std::iota(ks.begin(), ks.end(), 0);
    int rc;
    auto L = make_launch(P, c, c, false, B, nk, ks, P->d_class_lists.p + P->class_list_off[c], 0, P->stream, rc);
    if (!L) return rc;
    ts.launches.push_back(std::move(L));
  }
  CK(P->d_schwarz_pair.ensure(P->npairs));
  KernelArgs A = base_args(P);
  A.mode = MODE_SCHWARZ;
  A.omega = 0.0;  // Coulomb bounds (they bound the attenuated integrals too)
  A.schwarz_out = P->d_schwarz_pair.p;
  A.counters = nullptr;
  uint32_t launches = 0;
  int rc = run_tasks(P, ts, A, P->stream, launches);
  if (rc) return rc;
  std::vector<double> q(P->npairs);
  CK(cudaMemcpyAsync(q.data(), P->d_schwarz_pair.p, q.size() * sizeof(double), cudaMemcpyDeviceToHost, P->stream));
  CK(cudaStreamSynchronize(P->stream));
  P->schwarz.assign((size_t)P->nsh * P->nsh, 0.0);
  for (int p = 0; p < P->npairs; ++p) {
    P->pairs[p].q = q[p];
    const int i = P->pairs[p].i, j = P->pairs[p].j;
    P->schwarz[(size_t)i * P->nsh + j] = q[p];
    P->schwarz[(size_t)j * P->nsh + i] = q[p];
  }
  return IGPU_OK;
}

}  // namespace

// ===================================================================== C ABI

extern "C" {

uint32_t igpu_abi_version(void) { return IGPU_ABI_VERSION; }

const char* igpu_last_error_string(void) { return g_err.c_str(); }

int igpu_plan_create(const igpu_shell* sh, size_t nsh, int engine, igpu_plan** out) {
  if (!out) return fail(IGPU_ERR_INVALID_ARGUMENT, "out is NULL");
  *out = nullptr;
  if (nsh > 0 && !sh) return fail(IGPU_ERR_INVALID_ARGUMENT, "shells is NULL");
  if (engine < 0 || engine > 2) return fail(IGPU_ERR_INVALID_ARGUMENT, "unknown engine");
  if (nsh > 65535) return fail(IGPU_ERR_INVALID_ARGUMENT, "at most 65535 shells");
  // validation order of Shell::with_kind (src/shell.rs:92-118)
  for (size_t s = 0; s < nsh; ++s) {
    if (sh[s].nprim <= 0) return fail(IGPU_ERR_EMPTY_CONTRACTION, "shell has no primitives");
    if (!sh[s].exps || !sh[s].coefs) return fail(IGPU_ERR_INVALID_ARGUMENT, "shell exponents/coefficients NULL");
    if (sh[s].l < 0) return fail(IGPU_ERR_INVALID_ARGUMENT, "negative angular momentum");
    if (sh[s].l > MAX_L) return fail(IGPU_ERR_ANGULAR_MOMENTUM, "angular momentum exceeds supported maximum 6");
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(IGPU_ERR_NO_DEVICE, "no CUDA device");
  }
  auto P = std::make_unique<igpu_plan>();
  CK(cudaGetDevice(&P->device));
  P->engine = engine;
  P->nsh = (int)nsh;
  int rc = ensure_constants(P->device);
  if (rc) return rc;
  // shells, offsets, atoms (shell.rs:193-262)
  std::vector<double> eff;
  std::vector<double> expv;
  int acc = 0;
  for (size_t s = 0; s < nsh; ++s) {
    DevShell d{};
    d.cx = sh[s].center[0];
    d.cy = sh[s].center[1];
    d.cz = sh[s].center[2];
    d.l = sh[s].l;
    d.nprim = sh[s].nprim;
    d.spherical = sh[s].spherical ? 1 : 0;
    d.nfunc = d.spherical ? 2 * d.l + 1 : (d.l + 1) * (d.l + 2) / 2;
    d.off = acc;
    acc += d.nfunc;
    d.prim_off = (int)expv.size();
    for (int p = 0; p < d.nprim; ++p) {
      expv.push_back(sh[s].exps[p]);
      eff.push_back(effective_coeff(sh[s].exps[p], sh[s].coefs[p], d.l));
    }
    int atom = -1;
    for (size_t a = 0; a < P->atoms.size(); ++a)
      if (P->atoms[a][0] == d.cx && P->atoms[a][1] == d.cy && P->atoms[a][2] == d.cz) atom = (int)a;
    if (atom < 0) {
      atom = (int)P->atoms.size();
      P->atoms.push_back({d.cx, d.cy, d.cz});
    }
    d.atom = atom;
    if (d.spherical) P->spherical_any = true;
    P->all_spherical = (s == 0 ? true : P->all_spherical) && d.spherical;
    P->shells.push_back(d);
  }
  P->nao = acc;
  P->natom = (int)P->atoms.size();
  int lmax = 0;
  for (auto& d : P->shells) lmax = std::max(lmax, d.l);
  if (lmax > KERNEL_MAX_L)
    return fail(IGPU_ERR_UNSUPPORTED, "shell angular momentum above the compiled GPU classes (l <= " +
                                          std::to_string(KERNEL_MAX_L) + ")");
  // c2s matrices (l <= GPU_MAX_L + 1)
  for (int l = 0; l <= GPU_MAX_L + 1; ++l) {
    P->c2s_off[l] = (int)P->c2s.size();
    auto m = c2s_effective(l);
    P->c2s.insert(P->c2s.end(), m.begin(), m.end());
  }
  P->c2s_off[GPU_MAX_L + 2] = (int)P->c2s.size();
  // canonical pairs (integrals.rs:1252-1260) and primitive-pair data in
  // evaluation orientation (l_a >= l_b), screened as os_eri.rs:211-244
  const int npc = pair_class(lmax, lmax) + 1;
  P->class_pairs.assign(npc, {});
  for (int i = 0; i < (int)nsh; ++i)
    for (int j = 0; j <= i; ++j) {
      const DevShell& si = P->shells[i];
      const DevShell& sj = P->shells[j];
      const bool keep = si.l >= sj.l;
      const DevShell& A = keep ? si : sj;
      const DevShell& B = keep ? sj : si;
      PairD pr{};
      pr.a = keep ? i : j;
      pr.b = keep ? j : i;
      pr.i = i;
      pr.j = j;
      pr.tri = i * (i + 1) / 2 + j;
      pr.cls = pair_class(A.l, B.l);
      pr.abx = A.cx - B.cx;
      pr.aby = A.cy - B.cy;
      pr.abz = A.cz - B.cz;
      pr.prim_off = (int)P->prims.size();
      const double d2 = pr.abx * pr.abx + pr.aby * pr.aby + pr.abz * pr.abz;
      for (int pa = 0; pa < A.nprim; ++pa)
        for (int pb = 0; pb < B.nprim; ++pb) {
          const double ea = expv[A.prim_off + pa], eb = expv[B.prim_off + pb];
          const double ca = eff[A.prim_off + pa], cb = eff[B.prim_off + pb];
          const double z = ea + eb;
          const double kappa = std::exp(-(ea * eb / z) * d2);
          if (kappa * std::fabs(ca * cb) < 1e-32) continue;
          PrimPairD q{};
          q.zeta = z;
          q.alpha = ea;
          q.beta = eb;
          q.px = (ea * A.cx + eb * B.cx) / z;
          q.py = (ea * A.cy + eb * B.cy) / z;
          q.pz = (ea * A.cz + eb * B.cz) / z;
          q.pax = q.px - A.cx;
          q.pay = q.py - A.cy;
          q.paz = q.pz - A.cz;
          q.e = kappa * ca * cb;
          P->prims.push_back(q);
        }
      pr.nprim = (int)P->prims.size() - pr.prim_off;
      P->pairs.push_back(pr);
      P->class_pairs[pr.cls].push_back((int)P->pairs.size() - 1);
    }
  P->npairs = (int)P->pairs.size();
  P->nprims_main = (int)P->prims.size();
  CK(cudaStreamCreateWithFlags(&P->stream, cudaStreamNonBlocking));
  CK(cudaEventCreate(&P->ev0));
  CK(cudaEventCreate(&P->ev1));
  CK(P->d_shells.upload(P->shells, P->stream));
  CK(P->d_pairs.upload(P->pairs, P->stream));
  CK(P->d_prims.upload(P->prims, P->stream));
  CK(P->d_c2s.upload(P->c2s, P->stream));
  CK(P->d_counters.ensure(1));
  // class lists (device) in pair order for the Schwarz pass
  {
    std::vector<int> flat;
    P->class_list_off.assign(npc, 0);
    for (int c = 0; c < npc; ++c) {
      P->class_list_off[c] = (int)flat.size();
      flat.insert(flat.end(), P->class_pairs[c].begin(), P->class_pairs[c].end());
    }
    CK(P->d_class_lists.upload(flat, P->stream));
  }
  rc = run_schwarz(P.get());
  if (rc) return rc;
  // re-sort every class by (primitive-pair count desc, Q desc, index) and
  // record the equal-count groups used to cut task segments
  {
    std::vector<int> flat;
    P->class_groups.assign(npc, {});
    for (int c = 0; c < npc; ++c) {
      auto& v = P->class_pairs[c];
      std::stable_sort(v.begin(), v.end(), [&](int x, int y) {
        if (P->pairs[x].nprim != P->pairs[y].nprim) return P->pairs[x].nprim > P->pairs[y].nprim;
        return P->pairs[x].q > P->pairs[y].q;
      });
      for (size_t a = 0; a < v.size();) {
        size_t b = a;
        while (b < v.size() && P->pairs[v[b]].nprim == P->pairs[v[a]].nprim) ++b;
        P->class_groups[c].push_back({a, b});
        a = b;
      }
      P->class_list_off[c] = (int)flat.size();
      flat.insert(flat.end(), v.begin(), v.end());
    }
    CK(P->d_pairs.upload(P->pairs, P->stream));
    CK(P->d_class_lists.upload(flat, P->stream));
    CK(cudaStreamSynchronize(P->stream));
  }
  *out = P.release();
  return IGPU_OK;
}

int igpu_plan_destroy(igpu_plan* plan) {
  if (!plan) return IGPU_OK;
  cudaStreamSynchronize(plan->stream);
  if (plan->ev0) cudaEventDestroy(plan->ev0);
  if (plan->ev1) cudaEventDestroy(plan->ev1);
  for (cudaEvent_t ev : plan->events) cudaEventDestroy(ev);
  cudaStream_t s = plan->stream;
  delete plan;
  if (s) cudaStreamDestroy(s);
  return IGPU_OK;
}

int igpu_plan_query(const igpu_plan* P, size_t* nao, size_t* natom, size_t* nbra, size_t* nsh) {
  if (!P) return fail(IGPU_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (nao) *nao = P->nao;
  if (natom) *natom = P->natom;
  if (nbra) *nbra = P->npairs;
  if (nsh) *nsh = P->nsh;
  return IGPU_OK;
}

int igpu_bra_pairs(const igpu_plan* P, uint32_t* out) {
  if (!P || !out) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  for (int p = 0; p < P->npairs; ++p) {
    out[2 * p] = P->pairs[p].i;
    out[2 * p + 1] = P->pairs[p].j;
  }
  return IGPU_OK;
}

int igpu_atoms(const igpu_plan* P, double* xyz) {
  if (!P || !xyz) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  for (int a = 0; a < P->natom; ++a)
    for (int c = 0; c < 3; ++c) xyz[3 * a + c] = P->atoms[a][c];
  return IGPU_OK;
}

int igpu_schwarz(const igpu_plan* P, double* q) {
  if (!P || !q) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  std::memcpy(q, P->schwarz.data(), P->schwarz.size() * sizeof(double));
  return IGPU_OK;
}

int igpu_set_erf_omega(igpu_plan* P, double omega) {
  // check_erf_omega (src/integrals.rs:316-321): finite and > 0; 0 = Coulomb
  if (!P) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  if (!(omega == 0.0 || (omega > 0.0 && std::isfinite(omega))))
    return fail(IGPU_ERR_INVALID_ARGUMENT, "EriKernel::Erf requires a finite omega > 0");
  P->erf_omega = omega;
  return IGPU_OK;
}

int igpu_set_mixed_cutoff(igpu_plan* P, double cutoff) {
  if (!P || !(cutoff >= 0.0)) return fail(IGPU_ERR_INVALID_ARGUMENT, "invalid cutoff");
  P->mixed_cutoff = cutoff;
  return IGPU_OK;
}

int igpu_density_shell_bounds(const igpu_plan* Pc, const double* dens, int ndens, double* bounds) {
  igpu_plan* P = const_cast<igpu_plan*>(Pc);
  if (!P || !dens || !bounds) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  if (ndens < 1 || ndens > MAX_DENS) return fail(IGPU_ERR_DENSITY_COUNT, "1..64 densities");
  const size_t n2 = (size_t)P->nao * P->nao;
  CK(P->d_D.ensure(n2 * ndens));
  CK(P->d_bounds.ensure((size_t)P->nsh * P->nsh * ndens));
  CK(cudaMemcpyAsync(P->d_D.p, dens, n2 * ndens * sizeof(double), cudaMemcpyHostToDevice, P->stream));
  CK(launch_shell_block_max(P->d_D.p, ndens, P->d_shells.p, P->nsh, P->nao, 0, P->d_bounds.p, P->stream));
  CK(cudaMemcpyAsync(bounds, P->d_bounds.p, (size_t)P->nsh * P->nsh * ndens * sizeof(double),
                     cudaMemcpyDeviceToHost, P->stream));
  CK(cudaStreamSynchronize(P->stream));
  return IGPU_OK;
}

int igpu_jk_device(igpu_plan* P, const double* d_dens, int ndens, const uint32_t* bra_subset, size_t nsub,
                   double threshold, int want_k, int precision, double* d_J, double* d_K, void* stream) {
  if (!P || !d_dens || !d_J) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  if (ndens < 1 || ndens > MAX_DENS) return fail(IGPU_ERR_DENSITY_COUNT, "1..64 densities");
  if (want_k && !d_K) return fail(IGPU_ERR_INVALID_ARGUMENT, "exchange buffer required");
  if (precision != IGPU_PRECISION_FP64 && precision != IGPU_PRECISION_MIXED)
    return fail(IGPU_ERR_INVALID_ARGUMENT, "unknown precision");
  if (std::isnan(threshold)) return fail(IGPU_ERR_INVALID_ARGUMENT, "threshold is NaN");
  cudaStream_t s = stream ? (cudaStream_t)stream : P->stream;
  std::vector<unsigned> bitmap;
  if (bra_subset) {
    int rc = check_bra_subset(P, bra_subset, nsub, bitmap);
    if (rc) return rc;
    CK(P->d_bitmap.ensure(bitmap.size()));
    CK(cudaMemcpyAsync(P->d_bitmap.p, bitmap.data(), bitmap.size() * sizeof(unsigned), cudaMemcpyHostToDevice, s));
  }
  const size_t nn = (size_t)P->nsh * P->nsh;
  CK(P->d_bounds.ensure(nn * ndens));
  CK(P->d_flag.ensure(1));
  CK(cudaMemsetAsync(P->d_flag.p, 0, sizeof(unsigned long long), s));
  CK(launch_shell_block_max(d_dens, ndens, P->d_shells.p, P->nsh, P->nao, 0, P->d_bounds.p, s));
  CK(launch_asym_count(d_dens, ndens, P->nao, P->d_flag.p, s));
  unsigned long long asym = 0;
  CK(cudaMemcpyAsync(&asym, P->d_flag.p, sizeof(asym), cudaMemcpyDeviceToHost, s));
  CK(cudaMemsetAsync(P->d_counters.p, 0, sizeof(Counters), s));
  // FP64 part: Q_bra*Q_ket*max|D| >= cutoff (the bounds' global max)
  double fp64_cut = 0.0;
  if (precision == IGPU_PRECISION_MIXED) {
    std::vector<double> hb(nn * ndens);
    CK(cudaMemcpyAsync(hb.data(), P->d_bounds.p, hb.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    double dmax = 0.0;
    for (double v : hb) dmax = std::max(dmax, v);
    fp64_cut = dmax > 0.0 ? P->mixed_cutoff / dmax : std::numeric_limits<double>::infinity();
    if (fp64_cut <= 0.0) fp64_cut = std::numeric_limits<double>::min();
  } else {
    CK(cudaStreamSynchronize(s));
  }
  int trc;
  TaskSet* tasks = cached_tasks(P, threshold, fp64_cut, trc);
  if (!tasks) return trc;
  KernelArgs A = base_args(P);
  A.mode = MODE_JK;
  A.jk.D = d_dens;
  A.jk.bounds = P->d_bounds.p;
  A.jk.ndens = ndens;
  A.jk.want_k = want_k ? 1 : 0;
  A.jk.symmetric = asym == 0 ? 1 : 0;
  A.jk.threshold = threshold;
  A.bra_bitmap = bra_subset ? P->d_bitmap.p : nullptr;
  const size_t n2 = (size_t)P->nao * P->nao * ndens;
  if (A.jk.symmetric) {
    // one-orientation accumulators, symmetrised into the caller's J/K below
    CK(P->d_Jh.ensure(n2));
    CK(cudaMemsetAsync(P->d_Jh.p, 0, n2 * sizeof(double), s));
    A.jk.J = P->d_Jh.p;
    if (want_k) {
      CK(P->d_Kh.ensure(n2));
      CK(cudaMemsetAsync(P->d_Kh.p, 0, n2 * sizeof(double), s));
      A.jk.K = P->d_Kh.p;
    }
  } else {
    A.jk.J = d_J;
    A.jk.K = want_k ? d_K : nullptr;
  }
  uint32_t launches = 3;
  int rc = run_tasks(P, *tasks, A, s, launches);
  if (rc) return rc;
  if (A.jk.symmetric) {
    CK(launch_symmetrize_add(P->d_Jh.p, d_J, ndens, P->nao, s));
    if (want_k) CK(launch_symmetrize_add(P->d_Kh.p, d_K, ndens, P->nao, s));
  }
  CK(cudaStreamSynchronize(s));
  return collect_profile(P, ndens, true);
}

int igpu_autotune_jk(igpu_plan* P, const double* d_dens, int ndens, double threshold, int precision, void* stream) {
  if (!P || !d_dens) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  if (ndens < 1 || ndens > MAX_DENS) return fail(IGPU_ERR_DENSITY_COUNT, "1..64 densities");
  const size_t n2 = (size_t)P->nao * P->nao * ndens;
  DevBuf<double> tj, tk;
  CK(tj.ensure(n2));
  CK(tk.ensure(n2));
  const int cand[] = {4, 8, 16, 32, 64};
  std::map<int, std::map<int, float>> best;  // class key -> chunk -> shortest time
  for (int rep = 0; rep < 2; ++rep)
    for (int m : cand) {
      P->tune_mult = m;
      int rc = igpu_jk_device(P, d_dens, ndens, nullptr, 0, threshold, 1, precision, tj.p, tk.p, stream);
      P->tune_mult = 0;
      if (rc) return rc;
      for (const igpu_launch_record& r : P->profile) {
        const int key = tune_key(pair_class(r.la, r.lb), pair_class(r.lc, r.ld), r.fp32 != 0);
        auto& slot = best[key];
        auto it = slot.find(m);
        if (it == slot.end() || r.ms < it->second) slot[m] = r.ms;
      }
    }
  for (const auto& kv : best) {
    int pick = 16;
    float t = std::numeric_limits<float>::infinity();
    for (const auto& mt : kv.second)
      if (mt.second < t) {
        t = mt.second;
        pick = mt.first;
      }
    P->tuned_mult[kv.first] = pick;
  }
  return IGPU_OK;
}

int igpu_jk(igpu_plan* P, const double* dens, int ndens, const uint32_t* bra_subset, size_t nsub, double threshold,
            int want_k, int precision, double* J, double* K) {
  if (!P || !dens || !J) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  if (ndens < 1 || ndens > MAX_DENS) return fail(IGPU_ERR_DENSITY_COUNT, "1..64 densities");
  if (want_k && !K) return fail(IGPU_ERR_INVALID_ARGUMENT, "exchange buffer required");
  const size_t n2 = (size_t)P->nao * P->nao * ndens;
  CK(P->d_D.ensure(n2));
  CK(P->d_J.ensure(n2));
  if (want_k) CK(P->d_K.ensure(n2));
  CK(cudaMemcpyAsync(P->d_D.p, dens, n2 * sizeof(double), cudaMemcpyHostToDevice, P->stream));
  CK(cudaMemsetAsync(P->d_J.p, 0, n2 * sizeof(double), P->stream));
  if (want_k) CK(cudaMemsetAsync(P->d_K.p, 0, n2 * sizeof(double), P->stream));
  int rc = igpu_jk_device(P, P->d_D.p, ndens, bra_subset, nsub, threshold, want_k, precision, P->d_J.p,
                          want_k ? P->d_K.p : nullptr, P->stream);
  if (rc) return rc;
  std::vector<double> tj(n2), tk(want_k ? n2 : 0);
  CK(cudaMemcpyAsync(tj.data(), P->d_J.p, n2 * sizeof(double), cudaMemcpyDeviceToHost, P->stream));
  if (want_k) CK(cudaMemcpyAsync(tk.data(), P->d_K.p, n2 * sizeof(double), cudaMemcpyDeviceToHost, P->stream));
  CK(cudaStreamSynchronize(P->stream));
  for (size_t e = 0; e < n2; ++e) J[e] += tj[e];
  if (want_k)
    for (size_t e = 0; e < n2; ++e) K[e] += tk[e];
  return IGPU_OK;
}

int igpu_jk_device_static(igpu_plan* P, const double* d_dens, int ndens, double threshold, int want_k,
                          double* d_J, double* d_K, void* stream) {
  if (!P || !d_dens || !d_J) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  if (ndens < 1 || ndens > MAX_DENS) return fail(IGPU_ERR_DENSITY_COUNT, "1..64 densities");
  if (want_k && !d_K) return fail(IGPU_ERR_INVALID_ARGUMENT, "exchange buffer required");
  if (std::isnan(threshold)) return fail(IGPU_ERR_INVALID_ARGUMENT, "threshold is NaN");
  // the FP64 task list of this threshold must already exist (igpu_jk /
  // igpu_jk_device with the same threshold build and cache it)
  auto it = P->jk_tasks.find(std::make_pair(threshold, 0.0));
  if (it == P->jk_tasks.end())
    return fail(IGPU_ERR_INVALID_ARGUMENT,
                "no FP64 task list for this threshold: call igpu_jk or igpu_jk_device with it once first");
  StaticBufs sb;
  CK(static_buffers(&sb));
  const size_t nb = (size_t)ndens * P->nsh * P->nsh;
  if (nb > sb.bounds_doubles)
    return fail(IGPU_ERR_UNSUPPORTED, "ndens * nsh^2 exceeds the static bounds storage (" +
                                          std::to_string(sb.bounds_doubles) + " doubles)");
  TaskSet& ts = *it->second;
  const size_t nl = ts.launches.size();
  if (nl > (size_t)sb.max_launches) return fail(IGPU_ERR_UNSUPPORTED, "too many class launches for static storage");
  for (auto& L : ts.launches) {
    if (L->total == 0) continue;
    const KernelEntry* e = kernel_entry(L->pcb, L->pck);
    if (!e) return fail(IGPU_ERR_UNSUPPORTED, "angular class not compiled for the GPU");
    if ((size_t)(128 / e->team) * e->slot > sb.scratch_doubles)
      return fail(IGPU_ERR_UNSUPPORTED, "class scratch exceeds the static scratch storage");
  }
  cudaStream_t s = stream ? (cudaStream_t)stream : P->stream;
  CK(launch_shell_block_max(d_dens, ndens, P->d_shells.p, P->nsh, P->nao, 0, sb.bounds, s));
  // the work counters must start at zero; the scratch slots are written
  // before they are read (general image path: no running accumulators)
  CK(cudaMemsetAsync(sb.work, 0, nl * sizeof(unsigned long long), s));
  KernelArgs A = base_args(P);
  A.mode = MODE_JK;
  A.counters = nullptr;
  A.jk.D = d_dens;
  A.jk.bounds = sb.bounds;
  A.jk.ndens = ndens;
  A.jk.want_k = want_k ? 1 : 0;
  A.jk.symmetric = 0;
  A.jk.threshold = threshold;
  A.jk.J = d_J;
  A.jk.K = want_k ? d_K : nullptr;
  A.scratch = sb.scratch;
  for (size_t li = 0; li < nl; ++li) {
    Launch* L = ts.launches[li].get();
    if (L->total == 0) continue;
    const KernelEntry* e = kernel_entry(L->pcb, L->pck);
    const size_t teams = 128 / e->team;
    const size_t cap = sb.scratch_doubles / (teams * e->slot);
    const size_t grid = std::min(grid_for(e, false, L->total), cap);
    A.slot_doubles = e->slot;
    A.acc_offset = e->slot;
    A.work_counter = sb.work + li;
    A.chunk = (unsigned long long)(32 / e->team) * 16;
    A.task.bra_pair = L->bra_pair.p;
    A.task.ket_pairs = L->ket_list;
    A.task.prefix = L->prefix.p;
    A.task.ket_start = L->ket_start.n ? L->ket_start.p : nullptr;
    A.task.nbra = L->nbra;
    A.task.total = L->total;
    A.fp32 = 0;
    A.builder_swap = 0;
    CK(launch_quartets(e, false, (int)grid, A, s));
  }
  return IGPU_OK;
}

namespace {

// One launch whose ket list is owned by the launch: bra b runs kets
// kets[0 .. nket[b]-1].
std::unique_ptr<Launch> owned_launch(igpu_plan* P, int pcb, int pck, const std::vector<int>& bras,
                                     const std::vector<int>& nket, const std::vector<int>& kets, int& rc) {
  auto L = make_launch(P, pcb, pck, false, bras, nket, {}, nullptr, 0, P->stream, rc);
  if (!L) return nullptr;
  cudaError_t e = L->own_kets.upload(kets, P->stream);
  if (e != cudaSuccess) {
    rc = cuda_fail(e, "ket list upload");
    return nullptr;
  }
  L->ket_list = L->own_kets.p;
  return L;
}

// Runs a density-fitting task set into d_dense (len doubles) and checks the
// writers' fault flag.
int run_df(igpu_plan* P, TaskSet& ts, int mode, size_t len) {
  CK(P->d_fault.ensure(1));
  CK(cudaMemsetAsync(P->d_fault.p, 0, sizeof(unsigned), P->stream));
  KernelArgs A = base_args(P);
  A.mode = mode;
  A.dense = P->d_dense.p;
  A.dense_len = len;
  A.naux = P->naux;
  A.store_fault = P->d_fault.p;
  A.counters = nullptr;
  uint32_t launches = 0;
  int rc = run_tasks(P, ts, A, P->stream, launches);
  if (rc) return rc;
  unsigned fault = 0;
  CK(cudaMemcpyAsync(&fault, P->d_fault.p, sizeof(unsigned), cudaMemcpyDeviceToHost, P->stream));
  CK(cudaStreamSynchronize(P->stream));
  if (fault) return fail(IGPU_ERR_CUDA, "internal: density-fitting store outside the output");
  P->last = igpu_stats{};
  P->last.launches = launches;
  return IGPU_OK;
}

}  // namespace

// Dense tensor (MODE_DENSE: every canonical quartet, or with tau > -inf the
// quartets with Q_ij*Q_kl >= tau) or the EriBuilder fill (MODE_BUILDER,
// every ket for the requested bras).
static int dense_like(igpu_plan* P, bool builder, const uint32_t* sub, size_t nsub, double* out,
                      double tau = -std::numeric_limits<double>::infinity()) {
  if (!P || !out) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  const size_t n = (size_t)P->nao;
  const size_t n4 = n * n * n * n;
  CK(P->d_dense.ensure(n4));
  if (builder)
    CK(cudaMemcpyAsync(P->d_dense.p, out, n4 * sizeof(double), cudaMemcpyHostToDevice, P->stream));
  else
    CK(cudaMemsetAsync(P->d_dense.p, 0, n4 * sizeof(double), P->stream));
  TaskSet local;
  TaskSet* ts = &local;
  const int npc = (int)P->class_pairs.size();
  int rc = IGPU_OK;
  if (!builder && tau > -std::numeric_limits<double>::infinity()) {
    ts = cached_tasks(P, tau, 0.0, rc);
    if (!ts) return rc;
  } else if (!builder) {
    if (!P->dense_tasks) {
      P->dense_tasks = std::make_unique<TaskSet>();
      rc = build_jk_tasks(P, -std::numeric_limits<double>::infinity(), 0.0, *P->dense_tasks);
      if (rc) return rc;
    }
    ts = P->dense_tasks.get();
  } else {
    std::vector<char> want(P->npairs, sub ? 0 : 1);
    for (size_t x = 0; sub && x < nsub; ++x) {
      if (sub[x] >= (uint32_t)P->npairs) return fail(IGPU_ERR_NONCANONICAL_BRA, "bra pair index out of range");
      want[sub[x]] = 1;
    }
    for (int ca = 0; ca < npc; ++ca)
      for (int cb = 0; cb <= ca; ++cb) {
        const auto& A = P->class_pairs[ca];
        const auto& B = P->class_pairs[cb];
        if (A.empty() || B.empty()) continue;
        // requested bras of class ca, every ket of class cb
        std::vector<int> bras, nk;
        for (int p : A)
          if (want[p]) {
            bras.push_back(p);
            nk.push_back((int)B.size());
          }
        auto L = make_launch(P, ca, cb, false, bras, nk, {}, P->d_class_lists.p + P->class_list_off[cb], 0,
                             P->stream, rc);
        if (!L) return rc;
        local.launches.push_back(std::move(L));
        if (ca != cb) {
          // requested bras of class cb: evaluated as (ket of ca | bra)
          std::vector<int> reqs;
          for (int p : B)
            if (want[p]) reqs.push_back(p);
          if (reqs.empty()) continue;
          auto L2 = std::make_unique<Launch>();
          L2->pcb = ca;
          L2->pck = cb;
          L2->builder_swap = 1;
          std::vector<int> br(A.begin(), A.end());
          std::vector<unsigned long long> pre(1, 0);
          for (size_t x = 0; x < br.size(); ++x) pre.push_back(pre.back() + reqs.size());
          L2->nbra = (int)br.size();
          L2->total = pre.back();
          CK(L2->bra_pair.upload(br, P->stream));
          CK(L2->prefix.upload(pre, P->stream));
          // ket list = the requested bras (device copy owned by the launch)
          CK(L2->own_kets.upload(reqs, P->stream));
          L2->ket_list = L2->own_kets.p;
          local.launches.push_back(std::move(L2));
        }
      }
  }
  KernelArgs A = base_args(P);
  A.mode = builder ? MODE_BUILDER : MODE_DENSE;
  A.dense = P->d_dense.p;
  uint32_t launches = 0;
  rc = run_tasks(P, *ts, A, P->stream, launches);
  if (rc) return rc;
  CK(cudaMemcpyAsync(out, P->d_dense.p, n4 * sizeof(double), cudaMemcpyDeviceToHost, P->stream));
  CK(cudaStreamSynchronize(P->stream));
  // per-launch device times and quartet counts (igpu_last_stats / _profile)
  return collect_profile(P, 0, false);
}

int igpu_eri_dense(igpu_plan* P, double* out) { return dense_like(P, false, nullptr, 0, out); }

int igpu_eri_builder_fill(igpu_plan* P, const uint32_t* sub, size_t nsub, double* out) {
  return dense_like(P, true, sub, nsub, out);
}

int igpu_eri_screened(igpu_plan* P, double tau, double* out, uint64_t* total, uint64_t* skipped) {
  if (!P || !out) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  if (std::isnan(tau)) return fail(IGPU_ERR_INVALID_ARGUMENT, "tau is NaN");
  int rc = dense_like(P, false, nullptr, 0, out, tau);
  if (rc) return rc;
  // canonical quartets i >= j, k >= l, ij >= kl (integrals.rs:897-910)
  const uint64_t all = (uint64_t)P->npairs * ((uint64_t)P->npairs + 1) / 2;
  if (total) *total = all;
  if (skipped) *skipped = all - P->last.quartets;
  return IGPU_OK;
}

int igpu_eri_block(igpu_plan* P, int i, int j, int k, int l, double* out) {
  if (!P || !out) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  const int sh4[4] = {i, j, k, l};
  for (int x : sh4)
    if (x < 0 || x >= P->nsh) return fail(IGPU_ERR_INVALID_ARGUMENT, "shell index out of range");
  const int pb = std::max(i, j) * (std::max(i, j) + 1) / 2 + std::min(i, j);
  const int pk = std::max(k, l) * (std::max(k, l) + 1) / 2 + std::min(k, l);
  size_t len = 1;
  KernelArgs A = base_args(P);
  for (int x = 0; x < 4; ++x) {
    A.blk_shells[x] = sh4[x];
    A.blk_dims[x] = P->shells[sh4[x]].nfunc;
    len *= (size_t)A.blk_dims[x];
  }
  CK(P->d_dense.ensure(len));
  CK(cudaMemsetAsync(P->d_dense.p, 0, len * sizeof(double), P->stream));
  CK(P->d_fault.ensure(1));
  CK(cudaMemsetAsync(P->d_fault.p, 0, sizeof(unsigned), P->stream));
  // the larger pair class is the evaluation bra
  const int cb = P->pairs[pb].cls, ck = P->pairs[pk].cls;
  const bool swap = ck > cb;
  TaskSet ts;
  int rc;
  auto L = owned_launch(P, swap ? ck : cb, swap ? cb : ck, {swap ? pk : pb}, {1}, {swap ? pb : pk}, rc);
  if (!L) return rc;
  ts.launches.push_back(std::move(L));
  A.mode = MODE_BLOCK;
  A.dense = P->d_dense.p;
  A.dense_len = len;
  A.store_fault = P->d_fault.p;
  A.counters = nullptr;
  uint32_t launches = 0;
  rc = run_tasks(P, ts, A, P->stream, launches);
  if (rc) return rc;
  unsigned fault = 0;
  CK(cudaMemcpyAsync(&fault, P->d_fault.p, sizeof(unsigned), cudaMemcpyDeviceToHost, P->stream));
  CK(cudaMemcpyAsync(out, P->d_dense.p, len * sizeof(double), cudaMemcpyDeviceToHost, P->stream));
  CK(cudaStreamSynchronize(P->stream));
  if (fault) return fail(IGPU_ERR_CUDA, "internal: block store outside the output");
  P->last = igpu_stats{};
  P->last.launches = launches;
  return IGPU_OK;
}

int igpu_eri_packed(igpu_plan* P, double threshold, const uint32_t* sub, size_t nsub, double* out) {
  if (!P || !out) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  if (std::isnan(threshold)) return fail(IGPU_ERR_INVALID_ARGUMENT, "threshold is NaN");
  // shell-pair blocked AO-pair numbering (packed_eri.rs:103-114)
  std::vector<long long> start(P->npairs + 1, 0);
  for (int p = 0; p < P->npairs; ++p) {
    const int ni = P->shells[P->pairs[p].i].nfunc, nj = P->shells[P->pairs[p].j].nfunc;
    start[p + 1] = start[p] + (P->pairs[p].i == P->pairs[p].j ? (long long)ni * (ni + 1) / 2 : (long long)ni * nj);
  }
  const size_t m = (size_t)start[P->npairs];
  const size_t len = m * (m + 1) / 2;
  std::vector<unsigned> bitmap;
  if (sub) {
    int rc = check_bra_subset(P, sub, nsub, bitmap);
    if (rc) return rc;
  }
  cudaStream_t s = P->stream;
  CK(P->d_packed_start.upload(start, s));
  if (P->d_dense.ensure(len) != cudaSuccess) {
    cudaGetLastError();
    return fail(IGPU_ERR_OUT_OF_MEMORY, "packed tensor of " + std::to_string(len) + " doubles does not fit");
  }
  // the caller's buffer is the initial content: rows of other bras stay
  CK(cudaMemcpyAsync(P->d_dense.p, out, len * sizeof(double), cudaMemcpyHostToDevice, s));
  if (sub) {
    CK(P->d_bitmap.ensure(bitmap.size()));
    CK(cudaMemcpyAsync(P->d_bitmap.p, bitmap.data(), bitmap.size() * sizeof(unsigned), cudaMemcpyHostToDevice, s));
  }
  // threshold > 0: skip Q_ij*Q_kl < threshold (packed_eri.rs:184-187);
  // otherwise every canonical quartet
  TaskSet* ts = nullptr;
  int rc = IGPU_OK;
  if (threshold > 0.0) {
    ts = cached_tasks(P, threshold, 0.0, rc);
    if (!ts) return rc;
  } else {
    if (!P->dense_tasks) {
      P->dense_tasks = std::make_unique<TaskSet>();
      rc = build_jk_tasks(P, -std::numeric_limits<double>::infinity(), 0.0, *P->dense_tasks);
      if (rc) return rc;
    }
    ts = P->dense_tasks.get();
  }
  KernelArgs A = base_args(P);
  A.mode = MODE_PACKED;
  A.dense = P->d_dense.p;
  A.packed_start = P->d_packed_start.p;
  A.bra_bitmap = sub ? P->d_bitmap.p : nullptr;
  A.counters = nullptr;
  uint32_t launches = 0;
  rc = run_tasks(P, *ts, A, s, launches);
  if (rc) return rc;
  CK(cudaMemcpyAsync(out, P->d_dense.p, len * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  P->last = igpu_stats{};
  P->last.launches = launches;
  return IGPU_OK;
}

// ===================================================== density fitting (df.rs)

int igpu_plan_attach_aux(igpu_plan* P, const igpu_shell* aux, size_t naux_sh) {
  if (!P) return fail(IGPU_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (naux_sh > 0 && !aux) return fail(IGPU_ERR_INVALID_ARGUMENT, "aux shells is NULL");
  if (naux_sh > 65535) return fail(IGPU_ERR_INVALID_ARGUMENT, "at most 65535 aux shells");
  // validation order of Shell::with_kind (src/shell.rs:92-118)
  for (size_t s = 0; s < naux_sh; ++s) {
    if (aux[s].nprim <= 0) return fail(IGPU_ERR_EMPTY_CONTRACTION, "aux shell has no primitives");
    if (!aux[s].exps || !aux[s].coefs) return fail(IGPU_ERR_INVALID_ARGUMENT, "aux exponents/coefficients NULL");
    if (aux[s].l < 0) return fail(IGPU_ERR_INVALID_ARGUMENT, "negative angular momentum");
    if (aux[s].l > MAX_L) return fail(IGPU_ERR_ANGULAR_MOMENTUM, "angular momentum exceeds supported maximum 6");
    if (aux[s].l > KERNEL_MAX_L)
      return fail(IGPU_ERR_UNSUPPORTED, "aux shell angular momentum above the compiled GPU classes (l <= " +
                                            std::to_string(KERNEL_MAX_L) + ")");
  }
  // an earlier aux basis is replaced
  P->shells.resize(P->nsh);
  P->pairs.resize(P->npairs);
  P->prims.resize(P->nprims_main);
  P->has_aux = false;
  P->aux_class_pairs.assign(pair_class(KERNEL_MAX_L, 0) + 1, {});
  P->aux_q.assign(naux_sh, 0.0);
  // aux shells (offsets within the aux basis), then the unit s dummy: one
  // zero-exponent primitive of coefficient 1 (src/df.rs:33-38)
  const int dummy = P->nsh + (int)naux_sh;
  int acc = 0;
  for (size_t s = 0; s < naux_sh; ++s) {
    DevShell d{};
    d.cx = aux[s].center[0];
    d.cy = aux[s].center[1];
    d.cz = aux[s].center[2];
    d.l = aux[s].l;
    d.nprim = aux[s].nprim;
    d.spherical = aux[s].spherical ? 1 : 0;
    d.nfunc = d.spherical ? 2 * d.l + 1 : (d.l + 1) * (d.l + 2) / 2;
    d.off = acc;
    acc += d.nfunc;
    d.atom = -1;
    d.prim_off = -1;
    P->shells.push_back(d);
  }
  {
    DevShell d{};
    d.l = 0;
    d.nprim = 1;
    d.nfunc = 1;
    d.atom = -1;
    d.prim_off = -1;
    P->shells.push_back(d);
  }
  // one pair (aux shell, dummy) per aux shell: zeta = alpha, P = the aux
  // centre, kappa = 1, coefficient product = the aux effective coefficient
  // times 1, under the 1e-32 pair screen of build_pairs (os_eri.rs:211-244)
  for (size_t s = 0; s < naux_sh; ++s) {
    const DevShell& a = P->shells[P->nsh + s];
    PairD pr{};
    pr.a = P->nsh + (int)s;
    pr.b = dummy;
    pr.i = (int)s;
    pr.j = -1;
    pr.tri = -1;
    pr.cls = pair_class(a.l, 0);
    pr.prim_off = (int)P->prims.size();
    for (int k = 0; k < a.nprim; ++k) {
      const double ea = aux[s].exps[k];
      const double ca = effective_coeff(ea, aux[s].coefs[k], a.l);
      if (std::fabs(ca) < 1e-32) continue;
      PrimPairD q{};
      q.zeta = ea;
      q.alpha = ea;
      q.beta = 0.0;
      q.px = a.cx;
      q.py = a.cy;
      q.pz = a.cz;
      q.e = ca;
      P->prims.push_back(q);
    }
    pr.nprim = (int)P->prims.size() - pr.prim_off;
    P->pairs.push_back(pr);
    P->aux_class_pairs[pr.cls].push_back((int)P->pairs.size() - 1);
  }
  P->naux_sh = (int)naux_sh;
  P->naux = acc;
  CK(P->d_shells.upload(P->shells, P->stream));
  CK(P->d_pairs.upload(P->pairs, P->stream));
  CK(P->d_prims.upload(P->prims, P->stream));
  // aux Schwarz factors (Basis::schwarz_aux_bounds, src/df.rs:250-286): one
  // (P s|P s) quartet per aux shell, Coulomb operator
  {
    std::vector<int> flat;
    std::vector<int> off;
    for (const auto& v : P->aux_class_pairs) {
      off.push_back((int)flat.size());
      flat.insert(flat.end(), v.begin(), v.end());
    }
    CK(P->d_aux_lists.upload(flat, P->stream));
    TaskSet ts;
    for (size_t c = 0; c < P->aux_class_pairs.size(); ++c) {
      const auto& B = P->aux_class_pairs[c];
      if (B.empty()) continue;
      std::vector<int> nk(B.size(), 1), ks(B.size());
      std::iota(ks.begin(), ks.end(), 0);
      int rc;
      auto L = make_launch(P, (int)c, (int)c, false, B, nk, ks, P->d_aux_lists.p + off[c], 0, P->stream, rc);
      if (!L) return rc;
      ts.launches.push_back(std::move(L));
    }
    CK(P->d_schwarz_pair.ensure(P->pairs.size()));
    KernelArgs A = base_args(P);
    A.mode = MODE_SCHWARZ;
    A.omega = 0.0;
    A.schwarz_out = P->d_schwarz_pair.p;
    A.counters = nullptr;
    uint32_t launches = 0;
    int rc = run_tasks(P, ts, A, P->stream, launches);
    if (rc) return rc;
    std::vector<double> q(P->pairs.size());
    CK(cudaMemcpyAsync(q.data(), P->d_schwarz_pair.p, q.size() * sizeof(double), cudaMemcpyDeviceToHost,
                       P->stream));
    CK(cudaStreamSynchronize(P->stream));
    for (size_t s = 0; s < naux_sh; ++s) {
      const size_t pi = (size_t)P->npairs + s;
      P->pairs[pi].q = q[pi];
      P->aux_q[s] = q[pi];
    }
    for (auto& v : P->aux_class_pairs)
      std::stable_sort(v.begin(), v.end(), [&](int x, int y) {
        if (P->pairs[x].nprim != P->pairs[y].nprim) return P->pairs[x].nprim > P->pairs[y].nprim;
        return P->pairs[x].q > P->pairs[y].q;
      });
    CK(P->d_pairs.upload(P->pairs, P->stream));
    CK(cudaStreamSynchronize(P->stream));
  }
  P->has_aux = true;
  return IGPU_OK;
}

int igpu_aux_query(const igpu_plan* P, size_t* naux, size_t* naux_sh) {
  if (!P) return fail(IGPU_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (!P->has_aux) return fail(IGPU_ERR_INVALID_ARGUMENT, "no auxiliary basis attached");
  if (naux) *naux = P->naux;
  if (naux_sh) *naux_sh = P->naux_sh;
  return IGPU_OK;
}

int igpu_schwarz_aux(const igpu_plan* P, double* qp) {
  if (!P || !qp) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  if (!P->has_aux) return fail(IGPU_ERR_INVALID_ARGUMENT, "no auxiliary basis attached");
  if (!P->aux_q.empty()) std::memcpy(qp, P->aux_q.data(), P->aux_q.size() * sizeof(double));
  return IGPU_OK;
}

int igpu_eri_2c(igpu_plan* P, double* out) {
  if (!P || !out) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  if (!P->has_aux) return fail(IGPU_ERR_INVALID_ARGUMENT, "no auxiliary basis attached");
  const size_t len = (size_t)P->naux * P->naux;
  if (P->d_dense.ensure(len) != cudaSuccess) {
    cudaGetLastError();
    return fail(IGPU_ERR_OUT_OF_MEMORY, "metric of " + std::to_string(len) + " doubles does not fit");
  }
  CK(cudaMemsetAsync(P->d_dense.p, 0, len * sizeof(double), P->stream));
  // every unordered aux shell pair once: classes ca >= cb, and within one
  // class the kets at list positions <= the bra's
  TaskSet ts;
  const int nac = (int)P->aux_class_pairs.size();
  for (int ca = 0; ca < nac; ++ca)
    for (int cb = 0; cb <= ca; ++cb) {
      const auto& B = P->aux_class_pairs[ca];
      const auto& K = P->aux_class_pairs[cb];
      if (B.empty() || K.empty()) continue;
      std::vector<int> nk(B.size());
      for (size_t x = 0; x < B.size(); ++x) nk[x] = ca == cb ? (int)x + 1 : (int)K.size();
      int rc;
      auto L = owned_launch(P, ca, cb, B, nk, K, rc);
      if (!L) return rc;
      ts.launches.push_back(std::move(L));
    }
  int rc = run_df(P, ts, MODE_DF2, len);
  if (rc) return rc;
  CK(cudaMemcpyAsync(out, P->d_dense.p, len * sizeof(double), cudaMemcpyDeviceToHost, P->stream));
  CK(cudaStreamSynchronize(P->stream));
  return IGPU_OK;
}

int igpu_eri_3c(igpu_plan* P, const uint32_t* sub, size_t nsub, const uint8_t* keep, double* out) {
  if (!P || !out) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  if (!P->has_aux) return fail(IGPU_ERR_INVALID_ARGUMENT, "no auxiliary basis attached");
  if (nsub > 0 && !sub) return fail(IGPU_ERR_INVALID_ARGUMENT, "bra subset is NULL");
  const size_t len = (size_t)P->nao * P->nao * P->naux;
  std::vector<char> want(P->npairs, sub ? 0 : 1);
  for (size_t x = 0; sub && x < nsub; ++x) {
    if (sub[x] >= (uint32_t)P->npairs) return fail(IGPU_ERR_NONCANONICAL_BRA, "bra pair index out of range");
    want[sub[x]] = 1;
  }
  if (P->d_dense.ensure(len) != cudaSuccess) {
    cudaGetLastError();
    return fail(IGPU_ERR_OUT_OF_MEMORY, "3-centre tensor of " + std::to_string(len) + " doubles does not fit");
  }
  // slots outside the requested bands, and of skipped aux shells, keep the
  // caller's content
  if (!sub && !keep)
    CK(cudaMemsetAsync(P->d_dense.p, 0, len * sizeof(double), P->stream));
  else
    CK(cudaMemcpyAsync(P->d_dense.p, out, len * sizeof(double), cudaMemcpyHostToDevice, P->stream));
  TaskSet ts;
  const int npc = (int)P->class_pairs.size();
  const int nac = (int)P->aux_class_pairs.size();
  for (int cm = 0; cm < npc; ++cm) {
    std::vector<int> mains;
    for (int p : P->class_pairs[cm])
      if (want[p]) mains.push_back(p);
    if (mains.empty()) continue;
    for (int ca = 0; ca < nac; ++ca) {
      std::vector<int> auxs;
      for (int p : P->aux_class_pairs[ca])
        if (!keep || keep[P->pairs[p].i]) auxs.push_back(p);
      if (auxs.empty()) continue;
      int rc;
      std::unique_ptr<Launch> L;
      // the larger pair class is the evaluation bra
      if (cm >= ca)
        L = owned_launch(P, cm, ca, mains, std::vector<int>(mains.size(), (int)auxs.size()), auxs, rc);
      else
        L = owned_launch(P, ca, cm, auxs, std::vector<int>(auxs.size(), (int)mains.size()), mains, rc);
      if (!L) return rc;
      ts.launches.push_back(std::move(L));
    }
  }
  int rc = run_df(P, ts, MODE_DF3, len);
  if (rc) return rc;
  CK(cudaMemcpyAsync(out, P->d_dense.p, len * sizeof(double), cudaMemcpyDeviceToHost, P->stream));
  CK(cudaStreamSynchronize(P->stream));
  return IGPU_OK;
}

int igpu_last_stats(const igpu_plan* P, igpu_stats* st) {
  if (!P || !st) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  *st = P->last;
  return IGPU_OK;
}

int igpu_last_profile(const igpu_plan* P, igpu_launch_record* out, size_t cap, size_t* n) {
  if (!P || !n) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  *n = P->profile.size();
  for (size_t k = 0; k < P->profile.size() && k < cap && out; ++k) out[k] = P->profile[k];
  return IGPU_OK;
}

int igpu_grad_device(igpu_plan* P, const igpu_term* coulomb, int ncoul, const igpu_term* exchange, int nexch,
                     const uint32_t* bra_subset, size_t nsub, double threshold, int precision, double* d_out,
                     void* stream) {
  if (!P || !d_out) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  if (ncoul < 0 || nexch < 0 || (ncoul > 0 && !coulomb) || (nexch > 0 && !exchange))
    return fail(IGPU_ERR_INVALID_ARGUMENT, "invalid term list");
  for (int t = 0; t < ncoul; ++t)
    if (!coulomb[t].left || !coulomb[t].right) return fail(IGPU_ERR_INVALID_ARGUMENT, "term matrix is NULL");
  for (int t = 0; t < nexch; ++t)
    if (!exchange[t].left || !exchange[t].right) return fail(IGPU_ERR_INVALID_ARGUMENT, "term matrix is NULL");
  if (precision != IGPU_PRECISION_FP64 && precision != IGPU_PRECISION_MIXED)
    return fail(IGPU_ERR_INVALID_ARGUMENT, "unknown precision");
  if (std::isnan(threshold)) return fail(IGPU_ERR_INVALID_ARGUMENT, "threshold is NaN");
  // DirectGradContractor::new (src/direct_grad.rs:181-186), main shells only
  for (int sh = 0; sh < P->nsh; ++sh) {
    const DevShell& d = P->shells[sh];
    if (d.l > MAX_GRAD_L)
      return fail(IGPU_ERR_ANGULAR_MOMENTUM_GRAD, "angular momentum too high for the gradient (l <= 5)");
    if (d.l > GRAD_KERNEL_MAX_L)
      return fail(IGPU_ERR_UNSUPPORTED, "shell angular momentum above the compiled gradient classes (l <= " +
                                            std::to_string(GRAD_KERNEL_MAX_L) + ")");
  }
  cudaStream_t s = stream ? (cudaStream_t)stream : P->stream;
  std::vector<unsigned> bitmap;
  if (bra_subset) {
    int rc = check_bra_subset(P, bra_subset, nsub, bitmap);
    if (rc) return rc;
    CK(P->d_bitmap.ensure(bitmap.size()));
    CK(cudaMemcpyAsync(P->d_bitmap.p, bitmap.data(), bitmap.size() * sizeof(unsigned), cudaMemcpyHostToDevice, s));
  }
  // symmetrised shell-block maxima of every distinct matrix (direct_grad.rs:
  // 272-312), one pass per matrix
  std::vector<const double*> mats;
  auto index_of = [&mats](const double* m) {
    for (size_t q = 0; q < mats.size(); ++q)
      if (mats[q] == m) return (int)q;
    mats.push_back(m);
    return (int)mats.size() - 1;
  };
  std::vector<int> ci(2 * ncoul), xi(2 * nexch);
  for (int t = 0; t < ncoul; ++t) {
    ci[2 * t] = index_of(coulomb[t].left);
    ci[2 * t + 1] = index_of(coulomb[t].right);
  }
  for (int t = 0; t < nexch; ++t) {
    xi[2 * t] = index_of(exchange[t].left);
    xi[2 * t + 1] = index_of(exchange[t].right);
  }
  const size_t nn = (size_t)P->nsh * P->nsh;
  CK(P->d_gmax.ensure(nn * std::max<size_t>(1, mats.size())));
  for (size_t m = 0; m < mats.size(); ++m)
    CK(launch_shell_block_max(mats[m], 1, P->d_shells.p, P->nsh, P->nao, 1, P->d_gmax.p + m * nn, s));
  // pointer table: cl, cr, cl_max, cr_max (ncoul each), then xl, xr, xl_max, xr_max
  std::vector<const double*> ptr(4 * (size_t)ncoul + 4 * (size_t)nexch);
  std::vector<double> fac(ncoul + nexch);
  for (int t = 0; t < ncoul; ++t) {
    ptr[t] = coulomb[t].left;
    ptr[ncoul + t] = coulomb[t].right;
    ptr[2 * ncoul + t] = P->d_gmax.p + ci[2 * t] * nn;
    ptr[3 * ncoul + t] = P->d_gmax.p + ci[2 * t + 1] * nn;
    fac[t] = coulomb[t].factor;
  }
  const size_t xo = 4 * (size_t)ncoul;
  for (int t = 0; t < nexch; ++t) {
    ptr[xo + t] = exchange[t].left;
    ptr[xo + nexch + t] = exchange[t].right;
    ptr[xo + 2 * nexch + t] = P->d_gmax.p + xi[2 * t] * nn;
    ptr[xo + 3 * nexch + t] = P->d_gmax.p + xi[2 * t + 1] * nn;
    fac[ncoul + t] = exchange[t].factor;
  }
  CK(P->d_gptr.ensure(ptr.size()));
  if (!ptr.empty())
    CK(cudaMemcpyAsync(P->d_gptr.p, ptr.data(), ptr.size() * sizeof(const double*), cudaMemcpyHostToDevice, s));
  CK(P->d_gfac.ensure(fac.size()));
  if (!fac.empty())
    CK(cudaMemcpyAsync(P->d_gfac.p, fac.data(), fac.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  // FP64 part of MIXED: Q_bra*Q_ket*max|block| >= cutoff
  double fp64_cut = 0.0;
  if (precision == IGPU_PRECISION_MIXED) {
    std::vector<double> hb(nn * mats.size());
    if (!hb.empty())
      CK(cudaMemcpyAsync(hb.data(), P->d_gmax.p, hb.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    double dmax = 0.0;
    for (double v : hb) dmax = std::max(dmax, v);
    fp64_cut = dmax > 0.0 ? P->mixed_cutoff / dmax : std::numeric_limits<double>::infinity();
    if (fp64_cut <= 0.0) fp64_cut = std::numeric_limits<double>::min();
  } else {
    CK(cudaStreamSynchronize(s));
  }
  int trc;
  TaskSet* tasks = cached_tasks(P, threshold, fp64_cut, trc);
  if (!tasks) return trc;
  KernelArgs A = base_args(P);
  A.mode = MODE_GRAD;
  const double* const* dp = P->d_gptr.p;
  A.grad.cl = dp;
  A.grad.cr = dp + ncoul;
  A.grad.cl_max = dp + 2 * ncoul;
  A.grad.cr_max = dp + 3 * ncoul;
  A.grad.cf = P->d_gfac.p;
  A.grad.xl = dp + xo;
  A.grad.xr = dp + xo + nexch;
  A.grad.xl_max = dp + xo + 2 * nexch;
  A.grad.xr_max = dp + xo + 3 * nexch;
  A.grad.xf = P->d_gfac.p + ncoul;
  A.grad.ncoul = ncoul;
  A.grad.nexch = nexch;
  A.grad.threshold = threshold;
  A.grad.out = d_out;
  A.bra_bitmap = bra_subset ? P->d_bitmap.p : nullptr;
  uint32_t launches = (uint32_t)mats.size();
  int rc = run_tasks(P, *tasks, A, s, launches);
  if (rc) return rc;
  CK(cudaStreamSynchronize(s));
  return collect_profile(P, 0, false, ncoul, nexch);
}

int igpu_grad(igpu_plan* P, const igpu_term* coulomb, int ncoul, const igpu_term* exchange, int nexch,
              const uint32_t* bra_subset, size_t nsub, double threshold, int precision, double* out) {
  if (!P || !out) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  if (ncoul < 0 || nexch < 0 || (ncoul > 0 && !coulomb) || (nexch > 0 && !exchange))
    return fail(IGPU_ERR_INVALID_ARGUMENT, "invalid term list");
  // distinct host matrices to the device once each
  std::vector<const double*> host;
  auto index_of = [&host](const double* m) {
    for (size_t q = 0; q < host.size(); ++q)
      if (host[q] == m) return (int)q;
    host.push_back(m);
    return (int)host.size() - 1;
  };
  std::vector<igpu_term> dc(coulomb, coulomb + ncoul), dx(exchange, exchange + nexch);
  std::vector<int> idx;
  for (auto* v : {&dc, &dx})
    for (auto& t : *v) {
      if (!t.left || !t.right) return fail(IGPU_ERR_INVALID_ARGUMENT, "term matrix is NULL");
      idx.push_back(index_of(t.left));
      idx.push_back(index_of(t.right));
    }
  const size_t n2 = (size_t)P->nao * P->nao;
  CK(P->d_gmat.ensure(n2 * std::max<size_t>(1, host.size())));
  for (size_t m = 0; m < host.size(); ++m)
    CK(cudaMemcpyAsync(P->d_gmat.p + m * n2, host[m], n2 * sizeof(double), cudaMemcpyHostToDevice, P->stream));
  size_t q = 0;
  for (auto* v : {&dc, &dx})
    for (auto& t : *v) {
      t.left = P->d_gmat.p + idx[q++] * n2;
      t.right = P->d_gmat.p + idx[q++] * n2;
    }
  const size_t no = (size_t)P->natom * 3;
  CK(P->d_gout.ensure(no));
  CK(cudaMemsetAsync(P->d_gout.p, 0, no * sizeof(double), P->stream));
  int rc = igpu_grad_device(P, dc.data(), ncoul, dx.data(), nexch, bra_subset, nsub, threshold, precision,
                            P->d_gout.p, P->stream);
  if (rc) return rc;
  std::vector<double> g(no);
  CK(cudaMemcpyAsync(g.data(), P->d_gout.p, no * sizeof(double), cudaMemcpyDeviceToHost, P->stream));
  CK(cudaStreamSynchronize(P->stream));
  for (size_t e = 0; e < no; ++e) out[e] += g[e];
  return IGPU_OK;
}

}  // extern "C"
