// Molecule batches: one direct J/K build and one density-direct gradient for
// each of many independent molecules of uneven size, every angular class of
// every molecule in one persistent launch per class, the whole sequence
// captured once into a CUDA graph and replayed.
//
// The reference runs such a workload as a caller-side loop over one
// DirectContractor / DirectGradContractor per molecule
// (src/direct.rs:19-21, src/direct_grad.rs:140-142); the per-molecule
// screening, integrals and contractions here are exactly those of a plan of
// that molecule alone.
//
// Layout (the trick that leaves every kernel unchanged): with S the largest
// shell count and P the largest AO count of the batch, shell `local` of
// molecule m is global shell m*S + local and its AOs start at m*P + local
// offset.  A kernel forming the row-major index (row)*P + col of two AOs of
// molecule m then lands at m*P*(P+1) + local_row*P + local_col, so molecule
// m's matrices occupy their own block [m*P*(P+1), m*P*(P+1) + P*P) of one
// flat array; the shell-block bounds likewise occupy m*S*(S+1) with row
// stride S.  Pairs and quartets are formed inside a molecule only.
#include "plan_internal.hpp"

struct igpu_batch {
  std::unique_ptr<igpu_plan> plan;
  int nmol = 0, S = 0, Pd = 0;
  std::vector<int> mol_nsh, mol_nao, mol_natom, mol_atom0;
  size_t natom = 0;
  // device: densities, J, K (and their one-orientation accumulators), shell
  // bounds, gradient block maxima and output, gradient term tables
  DevBuf<double> d_D, d_J, d_K, d_Jh, d_Kh, d_bounds, d_gmax, d_gout, d_gfac;
  DevBuf<float> d_Df;  // FP32 copy of the densities (mixed steps)
  DevBuf<const double*> d_gptr;
  // the captured sequence and the arguments it was captured for
  cudaGraphExec_t exec = nullptr;
  bool have_key = false;
  double key_thr = 0.0, key_cut = 0.0, key_prim = 0.0, key_cf = 0.0, key_xf = 0.0;
  int key_want_k = 0, key_grad = 0, key_sym = 0, key_mixed = 0;
  ~igpu_batch() {
    if (exec) cudaGraphExecDestroy(exec);
  }
};

namespace {

size_t mat_len(const igpu_batch* b) { return (size_t)b->nmol * b->Pd * (b->Pd + 1); }
size_t blk_len(const igpu_batch* b) { return (size_t)b->nmol * b->S * (b->S + 1); }

// The launches of one batch step on stream s, with no host synchronisation
// and no allocation once the buffers exist (so that it can be captured).
int enqueue(igpu_batch* b, TaskSet& ts, double threshold, int mixed, double prim_cut, int want_k, int want_grad,
            int sym, double cf, double xf, cudaStream_t s, uint32_t& launches) {
  igpu_plan* P = b->plan.get();
  const size_t ml = mat_len(b);
  CK(cudaMemsetAsync(b->d_J.p, 0, ml * sizeof(double), s));
  if (want_k) CK(cudaMemsetAsync(b->d_K.p, 0, ml * sizeof(double), s));
  CK(launch_batch_block_max(b->d_D.p, P->d_shells.p, b->nmol, b->S, b->Pd, 0, b->d_bounds.p, s));
  KernelArgs A = base_args(P);
  A.mode = MODE_JK;
  A.jk.D = b->d_D.p;
  A.jk.bounds = b->d_bounds.p;
  A.jk.ndens = 1;
  A.jk.want_k = want_k;
  A.jk.symmetric = sym;
  A.jk.threshold = threshold;
  A.prim_cut = prim_cut;
  if (mixed) {
    // the FP32 launches read the FP32 copy of the densities
    CK(launch_to_float(b->d_D.p, b->d_Df.p, ml, s));
    A.jk.Df = b->d_Df.p;
    ++launches;
  }
  if (sym) {
    CK(cudaMemsetAsync(b->d_Jh.p, 0, ml * sizeof(double), s));
    if (want_k) CK(cudaMemsetAsync(b->d_Kh.p, 0, ml * sizeof(double), s));
    A.jk.J = b->d_Jh.p;
    A.jk.K = want_k ? b->d_Kh.p : nullptr;
  } else {
    A.jk.J = b->d_J.p;
    A.jk.K = want_k ? b->d_K.p : nullptr;
  }
  P->cur_log = &P->log;
  int rc = run_tasks(P, ts, A, s, launches);
  if (rc) return rc;
  if (sym) {
    CK(launch_batch_symmetrize_add(b->d_Jh.p, b->d_J.p, b->nmol, b->Pd, s));
    if (want_k) CK(launch_batch_symmetrize_add(b->d_Kh.p, b->d_K.p, b->nmol, b->Pd, s));
  }
  launches += 2 + (sym ? 1 + want_k : 0);
  if (!want_grad) return IGPU_OK;
  // gradient: Coulomb (cf, D, D) and exchange (xf, D, D), the density's
  // symmetrised shell-block maxima for the screening (src/direct_grad.rs:272-312)
  CK(launch_batch_block_max(b->d_D.p, P->d_shells.p, b->nmol, b->S, b->Pd, 1, b->d_gmax.p, s));
  CK(cudaMemsetAsync(b->d_gout.p, 0, b->natom * 3 * sizeof(double), s));
  KernelArgs G = base_args(P);
  G.mode = MODE_GRAD;
  const double* const* dp = b->d_gptr.p;
  G.grad.cl = dp;
  G.grad.cr = dp + 1;
  G.grad.cl_max = dp + 2;
  G.grad.cr_max = dp + 3;
  G.grad.cf = b->d_gfac.p;
  G.grad.xl = dp + 4;
  G.grad.xr = dp + 5;
  G.grad.xl_max = dp + 6;
  G.grad.xr_max = dp + 7;
  G.grad.xf = b->d_gfac.p + 1;
  G.grad.ncoul = cf != 0.0 ? 1 : 0;
  G.grad.nexch = xf != 0.0 ? 1 : 0;
  G.grad.threshold = threshold;
  G.grad.out = b->d_gout.p;
  P->cur_log = &P->log2;
  rc = run_tasks(P, ts, G, s, launches);
  P->cur_log = &P->log;
  launches += 2;
  return rc;
}

}  // namespace

extern "C" {

int igpu_batch_create(const igpu_shell* sh, const size_t* mol_nsh, size_t nmol, igpu_batch** out) {
  if (!out) return fail(IGPU_ERR_INVALID_ARGUMENT, "out is NULL");
  *out = nullptr;
  if (nmol == 0 || !mol_nsh) return fail(IGPU_ERR_INVALID_ARGUMENT, "no molecules");
  size_t nsh_total = 0;
  for (size_t m = 0; m < nmol; ++m) {
    if (mol_nsh[m] == 0) return fail(IGPU_ERR_INVALID_ARGUMENT, "molecule without shells");
    nsh_total += mol_nsh[m];
  }
  if (!sh) return fail(IGPU_ERR_INVALID_ARGUMENT, "shells is NULL");
  for (size_t s = 0; s < nsh_total; ++s) {
    // validation order of Shell::with_kind (src/shell.rs:92-118)
    if (sh[s].nprim <= 0) return fail(IGPU_ERR_EMPTY_CONTRACTION, "shell has no primitives");
    if (!sh[s].exps || !sh[s].coefs) return fail(IGPU_ERR_INVALID_ARGUMENT, "shell exponents/coefficients NULL");
    if (sh[s].l < 0) return fail(IGPU_ERR_INVALID_ARGUMENT, "negative angular momentum");
    if (sh[s].l > MAX_L) return fail(IGPU_ERR_ANGULAR_MOMENTUM, "angular momentum exceeds supported maximum 6");
    if (sh[s].l > KERNEL_MAX_L)
      return fail(IGPU_ERR_UNSUPPORTED, "shell angular momentum above the compiled GPU classes (l <= " +
                                            std::to_string(KERNEL_MAX_L) + ")");
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(IGPU_ERR_NO_DEVICE, "no CUDA device");
  }
  auto b = std::make_unique<igpu_batch>();
  b->plan = std::make_unique<igpu_plan>();
  igpu_plan* P = b->plan.get();
  P->batch = true;
  CK(cudaGetDevice(&P->device));
  int rc = ensure_constants(P->device);
  if (rc) return rc;
  b->nmol = (int)nmol;
  // per-molecule sizes and the padded strides
  size_t s0 = 0;
  for (size_t m = 0; m < nmol; ++m) {
    int nao = 0;
    for (size_t s = s0; s < s0 + mol_nsh[m]; ++s)
      nao += sh[s].spherical ? 2 * sh[s].l + 1 : (sh[s].l + 1) * (sh[s].l + 2) / 2;
    b->mol_nsh.push_back((int)mol_nsh[m]);
    b->mol_nao.push_back(nao);
    b->S = std::max(b->S, (int)mol_nsh[m]);
    b->Pd = std::max(b->Pd, nao);
    s0 += mol_nsh[m];
  }
  if ((size_t)b->S * nmol > (size_t)1 << 24) return fail(IGPU_ERR_INVALID_ARGUMENT, "batch too large");
  P->nsh = b->S;
  P->nao = b->Pd;
  // shells at m*S + local (padding entries have no functions and no pairs),
  // atoms by bitwise-equal centre inside each molecule (src/shell.rs:250-258)
  P->shells.assign((size_t)b->S * nmol, DevShell{});
  P->sshells.assign((size_t)b->S * nmol, SchwarzShell{});
  std::vector<double> expv, eff;
  int lmax = 0;
  s0 = 0;
  for (size_t m = 0; m < nmol; ++m) {
    b->mol_atom0.push_back((int)P->atoms.size());
    const size_t a0 = P->atoms.size();
    int acc = 0;
    for (size_t q = 0; q < mol_nsh[m]; ++q) {
      const igpu_shell& in = sh[s0 + q];
      DevShell d{};
      d.cx = in.center[0];
      d.cy = in.center[1];
      d.cz = in.center[2];
      d.l = in.l;
      d.nprim = in.nprim;
      d.spherical = in.spherical ? 1 : 0;
      d.nfunc = d.spherical ? 2 * d.l + 1 : (d.l + 1) * (d.l + 2) / 2;
      d.off = (int)m * b->Pd + acc;
      acc += d.nfunc;
      d.prim_off = (int)expv.size();
      d.pad = (int)m;  // molecule of the shell
      for (int p = 0; p < d.nprim; ++p) {
        expv.push_back(in.exps[p]);
        eff.push_back(effective_coeff(in.exps[p], in.coefs[p], d.l));
      }
      int atom = -1;
      for (size_t a = a0; a < P->atoms.size(); ++a)
        if (P->atoms[a][0] == d.cx && P->atoms[a][1] == d.cy && P->atoms[a][2] == d.cz) atom = (int)a;
      if (atom < 0) {
        atom = (int)P->atoms.size();
        P->atoms.push_back({d.cx, d.cy, d.cz});
      }
      d.atom = atom;
      if (d.spherical) P->spherical_any = true;
      lmax = std::max(lmax, d.l);
      const size_t g = m * b->S + q;
      P->shells[g] = d;
      SchwarzShell& ss = P->sshells[g];
      ss.l = d.l;
      ss.center[0] = d.cx;
      ss.center[1] = d.cy;
      ss.center[2] = d.cz;
      ss.exps.assign(expv.end() - d.nprim, expv.end());
      ss.coefs.assign(eff.end() - d.nprim, eff.end());
    }
    b->mol_natom.push_back((int)(P->atoms.size() - a0));
    s0 += mol_nsh[m];
  }
  b->natom = P->atoms.size();
  P->natom = (int)b->natom;
  bool all_sph = true;
  for (size_t m = 0; m < nmol; ++m)
    for (int q = 0; q < b->mol_nsh[m]; ++q) all_sph = all_sph && P->shells[m * b->S + q].spherical;
  P->all_spherical = all_sph;
  for (int l = 0; l <= GPU_MAX_L + 1; ++l) {
    P->c2s_off[l] = (int)P->c2s.size();
    auto mm = c2s_effective(l);
    P->c2s.insert(P->c2s.end(), mm.begin(), mm.end());
  }
  P->c2s_off[GPU_MAX_L + 2] = (int)P->c2s.size();
  for (size_t g = 0; g < P->shells.size(); ++g)
    if (P->shells[g].nfunc && P->shells[g].spherical) P->sshells[g].c2s = P->c2s.data() + P->c2s_off[P->shells[g].l];
  // canonical pairs inside each molecule (integrals.rs:1252-1260, local
  // order) with their primitive pairs in evaluation orientation
  // (os_eri.rs:211-244); tri is the local canonical index, which orders the
  // pairs of one molecule as the reference does
  const int npc = pair_class(lmax, lmax) + 1;
  P->class_pairs.assign(npc, {});
  for (size_t m = 0; m < nmol; ++m)
    for (int li = 0; li < b->mol_nsh[m]; ++li)
      for (int lj = 0; lj <= li; ++lj) {
        const int i = (int)m * b->S + li, j = (int)m * b->S + lj;
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
        pr.tri = li * (li + 1) / 2 + lj;
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
  CK(upload_prims(P));
  CK(P->d_c2s.upload(P->c2s, P->stream));
  CK(P->d_counters.ensure(1));
  {
    std::vector<int> flat;
    P->class_list_off.assign(npc, 0);
    for (int c = 0; c < npc; ++c) {
      P->class_list_off[c] = (int)flat.size();
      flat.insert(flat.end(), P->class_pairs[c].begin(), P->class_pairs[c].end());
    }
    CK(P->d_class_lists.upload(flat, P->stream));
  }
  rc = run_schwarz(P);
  if (rc) return rc;
  rc = exact_schwarz(P);
  if (rc) return rc;
  // every class sorted by (molecule, primitive-pair count desc, Q desc);
  // groups are the runs of equal (molecule, count), indexed per molecule
  {
    std::vector<int> flat;
    P->class_groups.assign(npc, {});
    P->class_mol_groups.assign(npc, std::vector<std::pair<int, int>>(nmol, {0, 0}));
    for (int c = 0; c < npc; ++c) {
      auto& v = P->class_pairs[c];
      auto mol = [&](int x) { return P->shells[P->pairs[x].i].pad; };
      std::stable_sort(v.begin(), v.end(), [&](int x, int y) {
        if (mol(x) != mol(y)) return mol(x) < mol(y);
        if (P->pairs[x].nprim != P->pairs[y].nprim) return P->pairs[x].nprim > P->pairs[y].nprim;
        return P->pairs[x].q > P->pairs[y].q;
      });
      for (size_t a = 0; a < v.size();) {
        size_t e = a;
        while (e < v.size() && P->pairs[v[e]].nprim == P->pairs[v[a]].nprim && mol(v[e]) == mol(v[a])) ++e;
        const int g = (int)P->class_groups[c].size();
        auto& r = P->class_mol_groups[c][mol(v[a])];
        if (r.first == r.second) r.first = g;
        r.second = g + 1;
        P->class_groups[c].push_back({a, e});
        a = e;
      }
      P->class_list_off[c] = (int)flat.size();
      flat.insert(flat.end(), v.begin(), v.end());
    }
    CK(P->d_pairs.upload(P->pairs, P->stream));
    CK(P->d_class_lists.upload(flat, P->stream));
  }
  // batch buffers
  const size_t ml = mat_len(b.get()), bl = blk_len(b.get());
  CK(b->d_D.ensure(ml));
  CK(b->d_Df.ensure(ml));
  CK(b->d_J.ensure(ml));
  CK(b->d_K.ensure(ml));
  CK(b->d_bounds.ensure(bl));
  CK(cudaMemsetAsync(b->d_D.p, 0, ml * sizeof(double), P->stream));
  CK(cudaStreamSynchronize(P->stream));
  *out = b.release();
  return IGPU_OK;
}

int igpu_batch_destroy(igpu_batch* b) {
  if (!b) return IGPU_OK;
  if (b->plan && b->plan->stream) cudaStreamSynchronize(b->plan->stream);
  cudaStream_t s = b->plan ? b->plan->stream : nullptr;
  if (b->plan) {
    if (b->plan->ev0) cudaEventDestroy(b->plan->ev0);
    if (b->plan->ev1) cudaEventDestroy(b->plan->ev1);
  }
  delete b;
  if (s) cudaStreamDestroy(s);
  return IGPU_OK;
}

int igpu_batch_query(const igpu_batch* b, size_t mol, size_t* nao, size_t* natom, size_t* nsh) {
  if (!b) return fail(IGPU_ERR_INVALID_ARGUMENT, "batch is NULL");
  if (mol >= (size_t)b->nmol) return fail(IGPU_ERR_INVALID_ARGUMENT, "molecule index out of range");
  if (nao) *nao = b->mol_nao[mol];
  if (natom) *natom = b->mol_natom[mol];
  if (nsh) *nsh = b->mol_nsh[mol];
  return IGPU_OK;
}

int igpu_batch_jk_grad(igpu_batch* b, const double* dens, double threshold, int precision, int want_k,
                       int want_grad, double coul_factor, double exch_factor, double* J, double* K, double* grad,
                       igpu_stats* stats) {
  if (!b || !dens || !J) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  if (want_k && !K) return fail(IGPU_ERR_INVALID_ARGUMENT, "exchange buffer required");
  if (want_grad && !grad) return fail(IGPU_ERR_INVALID_ARGUMENT, "gradient buffer required");
  if (precision != IGPU_PRECISION_FP64 && precision != IGPU_PRECISION_MIXED)
    return fail(IGPU_ERR_INVALID_ARGUMENT, "unknown precision");
  if (std::isnan(threshold)) return fail(IGPU_ERR_INVALID_ARGUMENT, "threshold is NaN");
  if (want_grad && coul_factor == 0.0 && exch_factor == 0.0) want_grad = 0;
  igpu_plan* P = b->plan.get();
  if (want_grad)
    for (const DevShell& d : P->shells)
      if (d.nfunc && d.l > GRAD_KERNEL_MAX_L)
        return fail(IGPU_ERR_UNSUPPORTED, "shell angular momentum above the compiled gradient classes (l <= " +
                                              std::to_string(GRAD_KERNEL_MAX_L) + ")");
  cudaStream_t s = P->stream;
  // densities into their molecule blocks; max |D| and bitwise symmetry on
  // the host (they select the task lists and the accumulation path)
  double dmax = 0.0;
  int sym = 1;
  size_t o = 0;
  for (int m = 0; m < b->nmol; ++m) {
    const int n = b->mol_nao[m];
    const double* Dm = dens + o;
    for (int r = 0; r < n; ++r)
      for (int c = 0; c < n; ++c) {
        dmax = std::max(dmax, std::fabs(Dm[(size_t)r * n + c]));
        if (c > r && std::memcmp(Dm + (size_t)r * n + c, Dm + (size_t)c * n + r, sizeof(double)) != 0) sym = 0;
      }
    CK(cudaMemcpy2DAsync(b->d_D.p + (size_t)m * b->Pd * (b->Pd + 1), (size_t)b->Pd * sizeof(double), Dm,
                         (size_t)n * sizeof(double), (size_t)n * sizeof(double), n, cudaMemcpyHostToDevice, s));
    o += (size_t)n * n;
  }
  const double fp64_cut = precision == IGPU_PRECISION_MIXED ? mixed_split(P->mixed_cutoff, dmax) : 0.0;
  const double prim_cut = precision == IGPU_PRECISION_MIXED && dmax > 0.0 ? P->mixed_prim_cut / dmax : 0.0;
  int trc;
  TaskSet* tasks = cached_tasks(P, threshold, fp64_cut, trc);
  if (!tasks) return trc;
  const int mixed = precision == IGPU_PRECISION_MIXED ? 1 : 0;
  const bool same = b->have_key && b->key_thr == threshold && b->key_cut == fp64_cut && b->key_prim == prim_cut &&
                    b->key_mixed == mixed && b->key_want_k == want_k &&
                    b->key_grad == want_grad && b->key_sym == sym && b->key_cf == coul_factor &&
                    b->key_xf == exch_factor && b->exec;
  uint32_t launches = 0;
  if (!same) {
    if (b->exec) {
      CK(cudaGraphExecDestroy(b->exec));
      b->exec = nullptr;
    }
    const size_t ml = mat_len(b);
    if (sym) {
      CK(b->d_Jh.ensure(ml));
      if (want_k) CK(b->d_Kh.ensure(ml));
    }
    if (want_grad) {
      CK(b->d_gmax.ensure(blk_len(b)));
      CK(b->d_gout.ensure(b->natom * 3));
      // Coulomb term (cl, cr, cl_max, cr_max) then exchange term, each the
      // density and its symmetrised block maxima
      std::vector<const double*> ptr = {b->d_D.p, b->d_D.p, b->d_gmax.p, b->d_gmax.p,
                                        b->d_D.p, b->d_D.p, b->d_gmax.p, b->d_gmax.p};
      CK(b->d_gptr.upload(ptr, s));
      std::vector<double> fac = {coul_factor, exch_factor};
      CK(b->d_gfac.upload(fac, s));
    }
    // one plain run allocates every scratch buffer; then the same sequence
    // is captured (no allocation or host synchronisation inside it)
    int rc = enqueue(b, *tasks, threshold, mixed, prim_cut, want_k, want_grad, sym, coul_factor, exch_factor, s,
                     launches);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s));
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    uint32_t l2 = 0;
    rc = enqueue(b, *tasks, threshold, mixed, prim_cut, want_k, want_grad, sym, coul_factor, exch_factor, s, l2);
    cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    CK(ce);
    ce = cudaGraphInstantiate(&b->exec, graph, 0);
    cudaGraphDestroy(graph);
    CK(ce);
    b->have_key = true;
    b->key_thr = threshold;
    b->key_cut = fp64_cut;
    b->key_prim = prim_cut;
    b->key_mixed = mixed;
    b->key_want_k = want_k;
    b->key_grad = want_grad;
    b->key_sym = sym;
    b->key_cf = coul_factor;
    b->key_xf = exch_factor;
  }
  CK(cudaEventRecord(P->ev0, s));
  CK(cudaGraphLaunch(b->exec, s));
  CK(cudaEventRecord(P->ev1, s));
  // results: every molecule's block back into the caller's concatenated
  // layout (accumulated, as the reference's outputs are)
  std::vector<double> hj(o), hk(want_k ? o : 0), hg(want_grad ? b->natom * 3 : 0);
  size_t q = 0;
  for (int m = 0; m < b->nmol; ++m) {
    const int n = b->mol_nao[m];
    const size_t base = (size_t)m * b->Pd * (b->Pd + 1);
    CK(cudaMemcpy2DAsync(hj.data() + q, (size_t)n * sizeof(double), b->d_J.p + base, (size_t)b->Pd * sizeof(double),
                         (size_t)n * sizeof(double), n, cudaMemcpyDeviceToHost, s));
    if (want_k)
      CK(cudaMemcpy2DAsync(hk.data() + q, (size_t)n * sizeof(double), b->d_K.p + base,
                           (size_t)b->Pd * sizeof(double), (size_t)n * sizeof(double), n, cudaMemcpyDeviceToHost, s));
    q += (size_t)n * n;
  }
  if (want_grad)
    CK(cudaMemcpyAsync(hg.data(), b->d_gout.p, hg.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  for (size_t e = 0; e < o; ++e) J[e] += hj[e];
  if (want_k)
    for (size_t e = 0; e < o; ++e) K[e] += hk[e];
  if (want_grad)
    for (size_t e = 0; e < hg.size(); ++e) grad[e] += hg[e];
  // counters of the replayed graph: J/K phase in log, gradient in log2
  igpu_stats st{};
  for (int ph = 0; ph < (want_grad ? 2 : 1); ++ph) {
    P->cur_log = ph ? &P->log2 : &P->log;
    int rc = ph ? collect_profile(P, 0, false, coul_factor != 0.0 ? 1 : 0, exch_factor != 0.0 ? 1 : 0)
                : collect_profile(P, 1, true);
    if (rc) return rc;
    st.quartets += P->last.quartets;
    st.quartet_hash += P->last.quartet_hash;
    st.quartets_fp32 += P->last.quartets_fp32;
    st.prim_quartets += P->last.prim_quartets;
    st.model_flops += P->last.model_flops;
    st.launches += P->last.launches;
  }
  P->cur_log = &P->log;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, P->ev0, P->ev1) != cudaSuccess) {
    cudaGetLastError();
    ms = 0.f;
  }
  st.kernel_ms = ms;
  P->last = st;
  if (stats) *stats = st;
  return IGPU_OK;
}

int igpu_batch_last_stats(const igpu_batch* b, igpu_stats* stats) {
  if (!b || !stats) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  *stats = b->plan->last;
  return IGPU_OK;
}

int igpu_batch_set_mixed_cutoff(igpu_batch* b, double cutoff) {
  if (!b) return fail(IGPU_ERR_INVALID_ARGUMENT, "batch is NULL");
  return igpu_set_mixed_cutoff(b->plan.get(), cutoff);
}

}  // extern "C"
