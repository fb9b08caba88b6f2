// Density-direct gradient entry points (DirectGradContractor,
// src/direct_grad.rs): host and device term matrices.
#include "plan_internal.hpp"

extern "C" {

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
    int rc = check_bra_subset(P, bra_subset, nsub, bitmap, true);
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
    fp64_cut = mixed_split(P->mixed_cutoff, dmax);
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

int igpu_autotune_grad(igpu_plan* P, const igpu_term* coulomb, int ncoul, const igpu_term* exchange, int nexch,
                       double threshold, int precision) {
  if (!P) return fail(IGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  std::vector<double> out((size_t)P->natom * 3);
  return tune_two_stage(P, true, [&] {
    return igpu_grad(P, coulomb, ncoul, exchange, nexch, nullptr, 0, threshold, precision, out.data());
  });
}

}  // extern "C"
