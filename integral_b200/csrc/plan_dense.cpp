// Dense-tensor entry points: Basis::eri / eri_screened / eri_block,
// EriBuilder fills and the packed symmetry-unique tensor
// (src/integrals.rs, src/eri_builder.rs, src/packed_eri.rs).
#include "plan_internal.hpp"

extern "C" {

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
    int rc = check_bra_subset(P, sub, nsub, bitmap, false);
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

}  // extern "C"
