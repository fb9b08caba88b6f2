// Direct J/K entry points (DirectContractor, src/direct.rs): density shell
// bounds, the J/K build on host or device buffers, the chunk autotuner and
// the allocation-free FP64 entry.
#include "plan_internal.hpp"

extern "C" {

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
    int rc = check_bra_subset(P, bra_subset, nsub, bitmap, true);
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
  double fp64_cut = 0.0, prim_cut = 0.0;
  if (precision == IGPU_PRECISION_MIXED) {
    std::vector<double> hb(nn * ndens);
    CK(cudaMemcpyAsync(hb.data(), P->d_bounds.p, hb.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    double dmax = 0.0;
    for (double v : hb) dmax = std::max(dmax, v);
    fp64_cut = mixed_split(P->mixed_cutoff, dmax);
    if (dmax > 0.0) prim_cut = P->mixed_prim_cut / dmax;
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
  A.prim_cut = prim_cut;
  A.bra_bitmap = bra_subset ? P->d_bitmap.p : nullptr;
  const size_t n2 = (size_t)P->nao * P->nao * ndens;
  A.jk.Df = nullptr;
  if (precision == IGPU_PRECISION_MIXED) {
    CK(P->d_Df.ensure(n2));
    CK(launch_to_float(d_dens, P->d_Df.p, n2, s));
    A.jk.Df = P->d_Df.p;
  }
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
  return tune_two_stage(P, false, [&] {
    return igpu_jk_device(P, d_dens, ndens, nullptr, 0, threshold, 1, precision, tj.p, tk.p, stream);
  });
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
  // the plan's buffers live on P->device; the static arrays are looked up
  // on the current device, so the two must agree
  int cur_dev = -1;
  CK(cudaGetDevice(&cur_dev));
  if (cur_dev != P->device)
    return fail(IGPU_ERR_INVALID_ARGUMENT, "current device " + std::to_string(cur_dev) +
                                               " is not the plan's device " + std::to_string(P->device));
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
    const auto tuned = P->tuned_mult.find(tune_key(L->pcb, L->pck, L->fp32, false));
    A.chunk = (unsigned long long)(32 / e->team) * (tuned == P->tuned_mult.end() ? 16 : tuned->second);
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
  // on the plan's private stream the caller has nothing to wait on: finish
  // here, as the other entry points do; on a caller stream the work stays
  // queued there
  if (!stream) CK(cudaStreamSynchronize(s));
  return IGPU_OK;
}

}  // extern "C"
