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
#include "plan_internal.hpp"

namespace igpu {
namespace host {

thread_local std::string g_err;

namespace {
std::mutex g_const_mutex;
std::vector<int> g_const_ready;  // per device
}  // namespace

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

// SM count of the current device, looked up once per device.
static int sm_count() {
  static std::mutex m;
  static std::vector<int> count;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(m);
  if ((int)count.size() <= dev) count.resize(dev + 1, 0);
  if (!count[dev]) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    count[dev] = n > 0 ? n : 1;
  }
  return count[dev];
}

size_t grid_for(const KernelEntry* e, bool fp32, unsigned long long total, int bps_cap) {
  const int nsm = sm_count();
  const int teams_per_block = 128 / e->team;
  const unsigned long long need = (total + teams_per_block - 1) / teams_per_block;
  int bps = blocks_per_sm(e, fp32);
  if (bps_cap > 0 && bps_cap < bps) bps = bps_cap;
  const unsigned long long cap = (unsigned long long)bps * nsm;
  return (size_t)std::max<unsigned long long>(1, std::min(need, cap));
}

KernelArgs base_args(igpu_plan* P) {
  KernelArgs A;
  std::memset(&A, 0, sizeof(A));
  A.shells = P->d_shells.p;
  A.pairs = P->d_pairs.p;
  A.prims = P->d_prims.p;
  A.primsf = P->d_primsf.p;
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

// Q_bra * Q_ket at or above which a quartet of the MIXED path runs in FP64:
// the plan's cutoff over max|D| rounded up to a power of two.  Rounding up
// keeps every quartet with Q_bra * Q_ket * max|D| >= cutoff in FP64, and
// the densities of successive SCF iterations, whose maxima rarely leave
// their binade, then share one cached task list.
double mixed_split(double cutoff, double dmax) {
  if (!(dmax > 0.0)) return std::numeric_limits<double>::infinity();
  int e = 0;
  const double m = std::frexp(dmax, &e);
  const double up = m == 0.5 ? dmax : std::ldexp(1.0, e);
  const double cut = cutoff / up;
  return cut > 0.0 ? cut : std::numeric_limits<double>::min();
}

// Key of a launch class in the tuned-chunk table; gradient classes have
// their own keys.
int tune_key(int pcb, int pck, bool fp32, bool grad) {
  return ((pcb * 64 + pck) * 2 + (fp32 ? 1 : 0)) | (grad ? (1 << 20) : 0);
}

// Tuning: note every launch time of the last call made with candidate m
// (a chunk multiplier, or a blocks-per-SM cap), then keep per class the
// candidate of the shortest time.
void tune_record(igpu_plan* P, int m, bool grad, std::map<int, std::map<int, float>>& best) {
  for (const igpu_launch_record& r : P->log.profile) {
    auto& slot = best[tune_key(pair_class(r.la, r.lb), pair_class(r.lc, r.ld), r.fp32 != 0, grad)];
    auto it = slot.find(m);
    if (it == slot.end() || r.ms < it->second) slot[m] = r.ms;
  }
}
void tune_keep(igpu_plan* P, const std::map<int, std::map<int, float>>& best, bool bps) {
  for (const auto& kv : best) {
    int pick = bps ? 0 : 16;
    float t = std::numeric_limits<float>::infinity();
    for (const auto& mt : kv.second)
      if (mt.second < t) {
        t = mt.second;
        pick = mt.first;
      }
    if (bps)
      P->tuned_bps[kv.first] = pick;
    else
      P->tuned_mult[kv.first] = pick;
  }
}

// The two-stage tuner of igpu_autotune_jk / igpu_autotune_grad: `run` makes
// one build; stage one times every chunk multiplier (tasks a warp claims per
// grab, in units of its teams) at the occupancy grid, stage two every
// blocks-per-SM cap of the grid with the chosen chunks; each twice over.
int tune_two_stage(igpu_plan* P, bool grad, const std::function<int()>& run) {
  const int mults[] = {4, 8, 16, 32, 64};
  std::map<int, std::map<int, float>> best;
  for (int rep = 0; rep < 2; ++rep)
    for (int m : mults) {
      P->tune_mult = m;
      const int rc = run();
      P->tune_mult = 0;
      if (rc) return rc;
      tune_record(P, m, grad, best);
    }
  tune_keep(P, best, false);
  // cap 0 is the occupancy limit itself
  const int caps[] = {1, 2, 3, 4, 0};
  std::map<int, std::map<int, float>> best_bps;
  for (int rep = 0; rep < 2; ++rep)
    for (int c : caps) {
      P->tune_bps = c > 0 ? c : -1;
      const int rc = run();
      P->tune_bps = 0;
      if (rc) return rc;
      tune_record(P, c, grad, best_bps);
    }
  tune_keep(P, best_bps, true);
  return IGPU_OK;
}

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
    if (A.mode == MODE_JK && L->fp32 && !A.jk.Df)
      return fail(IGPU_ERR_INVALID_ARGUMENT, "FP32 J/K launch without the FP32 densities");
    need = std::max(need, grid_for(e, L->fp32, L->total) * (128 / e->team) * slot_with_acc(e, L->pcb, A));
  }
  CK(P->d_scratch.ensure(need));
  const size_t nl = ts.launches.size();
  LaunchLog& lg = *P->cur_log;
  CK(lg.counters.ensure(nl));
  CK(cudaMemsetAsync(lg.counters.p, 0, nl * sizeof(Counters), s));
  CK(lg.work.ensure(nl));
  CK(cudaMemsetAsync(lg.work.p, 0, nl * sizeof(unsigned long long), s));
  while (lg.events.size() < 2 * nl) {
    cudaEvent_t ev;
    CK(cudaEventCreate(&ev));
    lg.events.push_back(ev);
  }
  lg.profile.clear();
  lg.profile_launch.clear();
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(s, &cap));
  const bool capturing = cap == cudaStreamCaptureStatusActive;
  const double prim_cut0 = A.prim_cut;
  for (size_t li = 0; li < nl; ++li) {
    Launch* L = ts.launches[li].get();
    if (L->total == 0) continue;
    const KernelEntry* e = entry(L->pcb, L->pck);
    const int key = tune_key(L->pcb, L->pck, L->fp32, A.mode == MODE_GRAD);
    int cap = 0;  // blocks-per-SM cap of the grid (0: the occupancy limit)
    if (P->tune_bps) {
      cap = P->tune_bps > 0 ? P->tune_bps : 0;
    } else if (A.mode == MODE_JK || A.mode == MODE_GRAD) {
      auto t = P->tuned_bps.find(key);
      if (t != P->tuned_bps.end()) cap = t->second;
    }
    const size_t grid = grid_for(e, L->fp32, L->total, cap);
    A.scratch = P->d_scratch.p;
    A.slot_doubles = slot_with_acc(e, L->pcb, A);
    A.acc_offset = e->slot;
    A.work_counter = lg.work.p + li;
    // tasks a warp claims per grab: (32 / team) x mult.  Untuned, mult is 16,
    // or less when the launch has so few tasks that 16 would leave warps of
    // the grid without work: every warp should find at least four grabs,
    // which matters for classes of few, heavy quartets (g shells, small
    // molecules)
    const unsigned long long warps = (unsigned long long)grid * 4;
    const unsigned long long fill = L->total / (4 * warps * (unsigned long long)(32 / e->team));
    int mult = (int)std::max<unsigned long long>(1, std::min<unsigned long long>(16, fill));
    if (P->tune_mult) {
      mult = P->tune_mult;
    } else if (A.mode == MODE_JK || A.mode == MODE_GRAD) {
      auto t = P->tuned_mult.find(key);
      if (t != P->tuned_mult.end()) mult = t->second;
    }
    A.chunk = (unsigned long long)(32 / e->team) * mult;
    if (A.counters) A.counters = lg.counters.p + li;
    A.task.bra_pair = L->bra_pair.p;
    A.task.ket_pairs = L->ket_list;
    A.task.prefix = L->prefix.p;
    A.task.ket_start = L->ket_start.n ? L->ket_start.p : nullptr;
    A.task.nbra = L->nbra;
    A.task.total = L->total;
    A.fp32 = L->fp32 ? 1 : 0;
    A.prim_cut = prim_cut0 / fp32_class_scale(class_lmax(L->pcb, L->pck));
    A.builder_swap = L->builder_swap;
    // under stream capture the records are external nodes, so that the
    // graph records them on every replay (the flag is only valid there)
    CK(capturing ? cudaEventRecordWithFlags(lg.events[2 * li], s, cudaEventRecordExternal)
                 : cudaEventRecord(lg.events[2 * li], s));
    CK(launch_quartets(e, L->fp32, (int)grid, A, s));
    CK(capturing ? cudaEventRecordWithFlags(lg.events[2 * li + 1], s, cudaEventRecordExternal)
                 : cudaEventRecord(lg.events[2 * li + 1], s));
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
    lg.profile.push_back(r);
    lg.profile_launch.push_back(li);
  }
  return IGPU_OK;
}

// After the stream is synchronised: per-launch times, counters, model flops.
int collect_profile(igpu_plan* P, int ndens, bool jk, int grad_terms_c, int grad_terms_x) {
  LaunchLog& lg = *P->cur_log;
  const size_t nl = lg.profile.empty() ? 0 : lg.profile_launch.back() + 1;
  std::vector<Counters> c(nl);
  if (nl) CK(cudaMemcpy(c.data(), lg.counters.p, nl * sizeof(Counters), cudaMemcpyDeviceToHost));
  P->last = igpu_stats{};
  for (size_t k = 0; k < lg.profile.size(); ++k) {
    igpu_launch_record& r = lg.profile[k];
    const size_t li = lg.profile_launch[k];
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, lg.events[2 * li], lg.events[2 * li + 1]) != cudaSuccess) {
      cudaGetLastError();  // a launch without a usable record: no time, no sticky error
      ms = 0.f;
    }
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
  P->last.launches = (uint32_t)lg.profile.size();
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

// How much smaller a class's FP32 cutoffs are than the plan's, by the
// largest angular momentum of its four shells: the recurrences' cancellation
// amplifies FP32 rounding more at high l, and on spread molecules with f and
// g shells the mixed energy error per unit of cutoff grew about 100-fold per
// unit of l above 2.  So f classes take a quartet into FP32 below 1/100 of
// the cutoff (and skip primitive quartets below 1/100 of the primitive
// cutoff), g classes below 1/10^4.
double fp32_class_scale(int lmax) { return lmax <= 2 ? 1.0 : std::pow(100.0, lmax - 2); }

int class_lmax(int pca, int pcb) {
  const int a = pc_la_host(pca), b = pca - a * (a + 1) / 2;
  const int c = pc_la_host(pcb), d = pcb - c * (c + 1) / 2;
  return std::max(std::max(a, b), std::max(c, d));
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
      // the class's own FP32 cutoff (fp32_class_scale)
      const double cut_c = fp64_cut / fp32_class_scale(class_lmax(ca, cb));
      std::vector<double> qk(K.size());
      for (size_t x = 0; x < K.size(); ++x) qk[x] = P->pairs[K[x]].q;
      // One segment per (bra, ket group of equal primitive-pair count): the
      // lanes of a warp then run equal primitive loops.  Within a group the
      // kets are Q-descending, so the accepted kets are a prefix.
      const auto& groups = P->class_groups[cb];
      std::vector<int> bras, n64, n32, st64, st32;
      for (size_t bp = 0; bp < B.size(); ++bp) {
        const double qb = P->pairs[B[bp]].q;
        // a batch pairs a bra with the kets of its own molecule only
        size_t g0 = 0, g1 = groups.size();
        if (P->batch) {
          const auto& r = P->class_mol_groups[cb][P->shells[P->pairs[B[bp]].i].pad];
          g0 = (size_t)r.first;
          g1 = (size_t)r.second;
        }
        for (size_t gi = g0; gi < g1; ++gi) {
          const size_t gs = groups[gi].first, ge = groups[gi].second;
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
              if (qb * qk[mid] >= cut_c)
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
// FP64 lists (cutoff 0, one per threshold) stay.  Every entry point that
// builds or evicts a list synchronises before it returns, so an evicted
// list has no launch in flight; igpu_jk_device_static only reads FP64
// lists, which are never evicted.
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

// Bitmap of a bra-pair subset.  Entry points that accumulate (J/K, the
// gradient) pass accumulate = true: a repeated index would count once here
// but twice through the reference's per-bra calls, so it is rejected.
int check_bra_subset(igpu_plan* P, const uint32_t* sub, size_t nsub, std::vector<unsigned>& bitmap,
                     bool accumulate) {
  bitmap.assign(((size_t)P->npairs + 31) / 32, 0u);
  for (size_t x = 0; x < nsub; ++x) {
    if (sub[x] >= (uint32_t)P->npairs) return fail(IGPU_ERR_NONCANONICAL_BRA, "bra pair index out of range");
    const unsigned bit = 1u << (sub[x] % 32);
    if (accumulate && (bitmap[sub[x] / 32] & bit))
      return fail(IGPU_ERR_INVALID_ARGUMENT, "bra pair " + std::to_string(sub[x]) + " repeated in the subset");
    bitmap[sub[x] / 32] |= bit;
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
  if (!P->batch) P->schwarz.assign((size_t)P->nsh * P->nsh, 0.0);
  for (int p = 0; p < P->npairs; ++p) {
    P->pairs[p].q = q[p];
    if (P->batch) continue;  // a batch keeps its bounds per pair only
    const int i = P->pairs[p].i, j = P->pairs[p].j;
    P->schwarz[(size_t)i * P->nsh + j] = q[p];
    P->schwarz[(size_t)j * P->nsh + i] = q[p];
  }
  return IGPU_OK;
}

// The reference's Schwarz bounds of the listed ordered shell pairs (i, j)
// wherever its Auto policy evaluates (ij|ij) with OS/HGP, on the device with
// the shared bit-exact evaluation (schwarz_core.cuh): one launch per class
// (l_i, l_j), one thread or one warp per pair.  done[x] = 1 where q[x] was set.
int exact_schwarz_pairs(igpu_plan* P, const std::vector<std::pair<int, int>>& pairs, std::vector<double>& q,
                        std::vector<unsigned char>& done) {
  q.assign(pairs.size(), 0.0);
  done.assign(pairs.size(), 0);
  const int nsh = (int)P->sshells.size();
  std::map<std::pair<int, int>, std::vector<int>> by_class;
  for (size_t x = 0; x < pairs.size(); ++x) {
    const SchwarzShell& a = P->sshells[pairs[x].first];
    const SchwarzShell& b = P->sshells[pairs[x].second];
    const long long np = (long long)a.exps.size() * (long long)b.exps.size();
    if (auto_picks_os(a.l + b.l, a.l + b.l, np * np)) by_class[{a.l, b.l}].push_back((int)x);
  }
  if (by_class.empty()) return IGPU_OK;
  cudaStream_t s = P->stream;
  // shell data and the Boys table
  std::vector<double> centers(3 * (size_t)nsh), exps, coefs;
  std::vector<int> nprim(nsh), prim_off(nsh), c2s_off(nsh, -1);
  for (int k = 0; k < nsh; ++k) {
    const SchwarzShell& sh = P->sshells[k];
    for (int c = 0; c < 3; ++c) centers[3 * k + c] = sh.center[c];
    nprim[k] = (int)sh.exps.size();
    prim_off[k] = (int)exps.size();
    exps.insert(exps.end(), sh.exps.begin(), sh.exps.end());
    coefs.insert(coefs.end(), sh.coefs.begin(), sh.coefs.end());
    if (sh.c2s) c2s_off[k] = (int)(sh.c2s - P->c2s.data());
  }
  DevBuf<double> d_centers, d_exps, d_coefs, d_boys, d_kappa, d_q, d_scratch;
  DevBuf<int> d_nprim, d_prim_off, d_c2s_off, d_pi, d_pj, d_eoff;
  DevBuf<long long> d_kappa_off;
  CK(d_centers.upload(centers, s));
  CK(d_exps.upload(exps, s));
  CK(d_coefs.upload(coefs, s));
  CK(d_nprim.upload(nprim, s));
  CK(d_prim_off.upload(prim_off, s));
  CK(d_c2s_off.upload(c2s_off, s));
  CK(d_boys.upload(schwarz_boys_table(), s));
  sc::BoysDev B = schwarz_boys_view();
  B.tab = d_boys.p;
  const size_t budget = (size_t)2 << 30;  // scratch bytes per class launch
  for (const auto& kv : by_class) {
    const std::vector<int>& xs = kv.second;
    std::vector<int> pi(xs.size()), pj(xs.size());
    std::vector<long long> koff(xs.size());
    std::vector<double> kap;
    int maxpp = 1;
    for (size_t t = 0; t < xs.size(); ++t) {
      const SchwarzShell& a = P->sshells[pairs[xs[t]].first];
      const SchwarzShell& b = P->sshells[pairs[xs[t]].second];
      pi[t] = pairs[xs[t]].first;
      pj[t] = pairs[xs[t]].second;
      koff[t] = (long long)kap.size();
      kap.resize(kap.size() + a.exps.size() * b.exps.size());
      schwarz_kappa(a, b, kap.data() + koff[t]);
      maxpp = std::max(maxpp, (int)(a.exps.size() * b.exps.size()));
    }
    std::vector<int> eoff;
    sc::SClass C = schwarz_class_layout(kv.first.first, kv.first.second, maxpp, eoff);
    CK(d_eoff.upload(eoff, s));
    C.eoff = d_eoff.p;
    // classes from l_i + l_j = 4 up run a warp per pair (their recurrence
    // levels have hundreds of elements), the smaller ones a thread per pair
    const int team = kv.first.first + kv.first.second >= 4 ? 32 : 1;
    const size_t per_block_pairs = 128 / team;
    const size_t per_block = per_block_pairs * C.total * sizeof(double);
    const size_t want = (xs.size() + per_block_pairs - 1) / per_block_pairs;
    const int grid = (int)std::max<size_t>(1, std::min(want, std::max<size_t>(1, budget / per_block)));
    CK(d_scratch.ensure((size_t)grid * per_block_pairs * C.total));
    CK(d_pi.upload(pi, s));
    CK(d_pj.upload(pj, s));
    CK(d_kappa_off.upload(koff, s));
    CK(d_kappa.upload(kap, s));
    CK(d_q.ensure(xs.size()));
    SchwarzPairsDev in{(int)xs.size(), d_pi.p, d_pj.p, d_centers.p, d_nprim.p, d_prim_off.p, d_exps.p, d_coefs.p,
                       d_c2s_off.p, P->d_c2s.p, d_kappa_off.p, d_kappa.p};
    CK(launch_schwarz_exact(B, C, in, d_scratch.p, grid, team, d_q.p, s));
    std::vector<double> hq(xs.size());
    CK(cudaMemcpyAsync(hq.data(), d_q.p, hq.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    // the host vectors above are read by queued copies: finish this class
    CK(cudaStreamSynchronize(s));
    for (size_t t = 0; t < xs.size(); ++t) {
      q[xs[t]] = hq[t];
      done[xs[t]] = 1;
    }
  }
  return IGPU_OK;
}

// Replace the device (P|P) Q of every canonical pair for which the
// reference's Auto policy picks OS/HGP by its bit-exact evaluation in the
// reference orientation (shell i, shell j), so that every threshold
// comparison of the screening is the reference's.
int exact_schwarz(igpu_plan* P) {
  std::vector<std::pair<int, int>> ij(P->npairs);
  for (int p = 0; p < P->npairs; ++p) ij[p] = {P->pairs[p].i, P->pairs[p].j};
  std::vector<double> q;
  std::vector<unsigned char> done;
  const int rc = exact_schwarz_pairs(P, ij, q, done);
  if (rc) return rc;
  P->schwarz_exact_pairs = 0;
  for (int p = 0; p < P->npairs; ++p) {
    if (!done[p]) continue;
    ++P->schwarz_exact_pairs;
    P->pairs[p].q = q[p];
    if (P->batch) continue;
    const int i = P->pairs[p].i, j = P->pairs[p].j;
    P->schwarz[(size_t)i * P->nsh + j] = q[p];
    P->schwarz[(size_t)j * P->nsh + i] = q[p];
  }
  return IGPU_OK;
}

// The primitive pairs and their FP32 copy to the device.
cudaError_t upload_prims(igpu_plan* P) {
  std::vector<PrimPairF> f(P->prims.size());
  for (size_t k = 0; k < f.size(); ++k) {
    const PrimPairD& d = P->prims[k];
    f[k] = PrimPairF{(float)d.zeta, (float)d.e, (float)d.pax, (float)d.pay, (float)d.paz,
                     (float)d.alpha, (float)d.beta, 0.f};
  }
  cudaError_t e = P->d_prims.upload(P->prims, P->stream);
  if (e != cudaSuccess) return e;
  e = P->d_primsf.upload(f, P->stream);
  if (e != cudaSuccess) return e;
  // the host copy goes out of scope: finish the transfer
  return cudaStreamSynchronize(P->stream);
}

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

}  // namespace host
}  // namespace igpu

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
    SchwarzShell ss;
    ss.l = d.l;
    ss.center[0] = d.cx;
    ss.center[1] = d.cy;
    ss.center[2] = d.cz;
    ss.exps.assign(expv.end() - d.nprim, expv.end());
    ss.coefs.assign(eff.end() - d.nprim, eff.end());
    P->sshells.push_back(std::move(ss));
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
  for (int s = 0; s < (int)nsh; ++s)
    if (P->shells[s].spherical) P->sshells[s].c2s = P->c2s.data() + P->c2s_off[P->shells[s].l];
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
  CK(upload_prims(P.get()));
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
  rc = exact_schwarz(P.get());
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

int igpu_schwarz(const igpu_plan* Pc, double* q) {
  if (!Pc || !q) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  igpu_plan* P = const_cast<igpu_plan*>(Pc);
  if (!P->schwarz_upper_done) {
    // Q[j][i], j < i, is the reference's own evaluation of (j i|j i) (it
    // computes every ordered pair), which may differ from Q[i][j] in the
    // last bit
    std::vector<std::pair<int, int>> ji;
    for (int p = 0; p < P->npairs; ++p)
      if (P->pairs[p].i != P->pairs[p].j) ji.push_back({P->pairs[p].j, P->pairs[p].i});
    std::vector<double> v;
    std::vector<unsigned char> done;
    const int rc = exact_schwarz_pairs(P, ji, v, done);
    if (rc) return rc;
    for (size_t x = 0; x < ji.size(); ++x)
      if (done[x]) P->schwarz[(size_t)ji[x].first * P->nsh + ji[x].second] = v[x];
    P->schwarz_upper_done = true;
  }
  std::memcpy(q, P->schwarz.data(), P->schwarz.size() * sizeof(double));
  return IGPU_OK;
}

int igpu_schwarz_bounds(const igpu_shell* sh, size_t nsh, double* q, size_t* n_rys) {
  if (nsh > 0 && (!sh || !q)) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  if (n_rys) *n_rys = 0;
  std::vector<SchwarzShell> ss(nsh);
  for (size_t s = 0; s < nsh; ++s) {
    // validation order of Shell::with_kind (src/shell.rs:92-118)
    if (sh[s].nprim <= 0) return fail(IGPU_ERR_EMPTY_CONTRACTION, "shell has no primitives");
    if (!sh[s].exps || !sh[s].coefs) return fail(IGPU_ERR_INVALID_ARGUMENT, "shell exponents/coefficients NULL");
    if (sh[s].l < 0) return fail(IGPU_ERR_INVALID_ARGUMENT, "negative angular momentum");
    if (sh[s].l > MAX_L) return fail(IGPU_ERR_ANGULAR_MOMENTUM, "angular momentum exceeds supported maximum 6");
    ss[s].l = sh[s].l;
    for (int c = 0; c < 3; ++c) ss[s].center[c] = sh[s].center[c];
    for (int p = 0; p < sh[s].nprim; ++p) {
      ss[s].exps.push_back(sh[s].exps[p]);
      ss[s].coefs.push_back(effective_coeff(sh[s].exps[p], sh[s].coefs[p], sh[s].l));
    }
  }
  std::vector<std::vector<double>> mats(MAX_L + 1);
  for (size_t s = 0; s < nsh; ++s)
    if (sh[s].spherical) {
      if (mats[sh[s].l].empty()) mats[sh[s].l] = c2s_effective(sh[s].l);
      ss[s].c2s = mats[sh[s].l].data();
    }
  std::vector<std::pair<int, int>> all;
  for (int i = 0; i < (int)nsh; ++i)
    for (int j = 0; j < (int)nsh; ++j) all.push_back({i, j});
  std::vector<double> v;
  std::vector<unsigned char> done;
  schwarz_exact_many(ss, all, v, done, 0);
  size_t rys = 0;
  for (size_t x = 0; x < all.size(); ++x) {
    q[x] = done[x] ? v[x] : std::numeric_limits<double>::quiet_NaN();
    rys += done[x] ? 0 : 1;
  }
  if (n_rys) *n_rys = rys;
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

int igpu_get_mixed_cutoffs(const igpu_plan* P, double* cutoff, double* prim_eps) {
  if (!P) return fail(IGPU_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (cutoff) *cutoff = P->mixed_cutoff;
  if (prim_eps) *prim_eps = P->mixed_prim_cut;
  return IGPU_OK;
}

int igpu_set_mixed_prim_cutoff(igpu_plan* P, double eps) {
  if (!P || !(eps >= 0.0) || std::isinf(eps)) return fail(IGPU_ERR_INVALID_ARGUMENT, "invalid primitive cutoff");
  P->mixed_prim_cut = eps;
  return IGPU_OK;
}

int igpu_last_stats(const igpu_plan* P, igpu_stats* st) {
  if (!P || !st) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  *st = P->last;
  return IGPU_OK;
}

int igpu_last_profile(const igpu_plan* P, igpu_launch_record* out, size_t cap, size_t* n) {
  if (!P || !n) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  *n = P->log.profile.size();
  for (size_t k = 0; k < P->log.profile.size() && k < cap && out; ++k) out[k] = P->log.profile[k];
  return IGPU_OK;
}

}  // extern "C"
