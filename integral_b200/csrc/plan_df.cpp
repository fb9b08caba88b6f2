// Density-fitting entry points (src/df.rs): the auxiliary basis attached
// to a plan, the 3-centre tensor, the 2-centre metric and the aux Schwarz
// factors.
#include "plan_internal.hpp"

namespace {

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

extern "C" {

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
  CK(upload_prims(P));
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

}  // extern "C"
