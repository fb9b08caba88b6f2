// Exact Schwarz bounds: the host side.
//
// The screened quartet list is decided by comparisons Q_ij * Q_kl (* max|D|)
// against a threshold, so the list equals the reference's bit for bit only if
// every Q is the reference's bit for bit.  The reference takes Q from its own
// FP64 engines (Basis::schwarz_bounds, src/integrals.rs:842-862) under the
// Auto policy (src/integrals.rs:374-388), which picks the Obara-Saika /
// Head-Gordon-Pople engine for every diagonal quartet of a contracted basis.
// schwarz_core.cuh evaluates those diagonal quartets with the same
// arithmetic in the same order; this file builds its inputs (the Boys table
// of src/math/boys.rs:122-136, the kappa of every primitive combination, the
// per-class layout of the work arrays) and runs it on the host threads.  The
// device runs the same code (schwarz_dev.cu).  The build compiles both
// without floating-point contraction, so every product and sum rounds as in
// Rust; libm's exp and pow are the reference's own (same library on the same
// host), sqrt and division are correctly rounded everywhere.
#include "host_schwarz.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <thread>

#include "host_math.hpp"

namespace igpu {
namespace {

// Table of F_0..F_32 and e^{-T0} on the grid T0 = 0.1 i, i = 0..930
// (src/math/boys.rs:122-136), built once from the positive series or the
// large-T closed form with the downward recurrence.
class BoysTable {
 public:
  static const BoysTable& get() {
    static const BoysTable b;
    return b;
  }
  sc::BoysDev view() const {
    sc::BoysDev v;
    v.tab = tab_.data();
    v.tmax = tmax_;
    v.h = h_;
    for (int k = 0; k <= sc::kBoysTaylor; ++k) v.inv_fact[k] = inv_fact_[k];
    for (int m = 0; m <= sc::kBoysMaxM; ++m) v.inv_odd[m] = inv_odd_[m];
    return v;
  }
  const std::vector<double>& table() const { return tab_; }

 private:
  BoysTable() {
    inv_fact_[0] = 1.0;
    for (int k = 1; k <= sc::kBoysTaylor; ++k) inv_fact_[k] = inv_fact_[k - 1] / (double)k;
    inv_odd_[0] = 1.0;
    for (int m = 1; m <= sc::kBoysMaxM; ++m) inv_odd_[m] = 1.0 / (double)(2 * m - 1);
    tmax_ = 33.0 + 2.5 * (double)sc::kBoysMaxM;
    const size_t ngrid = (size_t)(tmax_ / h_);
    tab_.assign((ngrid + 1) * sc::kBoysRow, 0.0);
    for (size_t i = 0; i <= ngrid; ++i) {
      const double t0 = (double)i * h_;
      double* row = tab_.data() + i * sc::kBoysRow;
      reference(sc::kBoysOrders - 1, t0, row);
      row[sc::kBoysOrders] = std::exp(-t0);
    }
  }
  // Top order by the positive series below the asymptotic boundary
  // 33 + 2.5 m, else the large-T closed form; then the downward recurrence.
  static void reference(int mmax, double t, double* f) {
    const double et = std::exp(-t);
    if (t < 33.0 + 2.5 * (double)mmax) {
      const double two_t = 2.0 * t;
      double term = 1.0 / (double)(2 * mmax + 1);
      double sum = term;
      for (int k = 1;; ++k) {
        term *= two_t / (double)(2 * mmax + 2 * k + 1);
        sum += term;
        if (term <= sum * 1e-17 || k + 1 >= 1000) break;
      }
      f[mmax] = et * sum;
    } else {
      double v = 0.5 * std::sqrt(sc::kPi / t);
      const double two_t = 2.0 * t;
      for (int k = 1; k <= mmax; ++k) v *= (double)(2 * k - 1) / two_t;
      f[mmax] = v;
    }
    for (int m = mmax; m > 0; --m) f[m - 1] = (2.0 * t * f[m] + et) / (double)(2 * m - 1);
  }

  double h_ = 0.1;
  double tmax_ = 0.0;
  double inv_fact_[sc::kBoysTaylor + 1];
  double inv_odd_[sc::kBoysMaxM + 1];
  std::vector<double> tab_;
};

int ncart_of(int l) { return (l + 1) * (l + 2) / 2; }

}  // namespace

sc::BoysDev schwarz_boys_view() { return BoysTable::get().view(); }
const std::vector<double>& schwarz_boys_table() { return BoysTable::get().table(); }

sc::SClass schwarz_class_layout(int li, int lj, int maxpp, std::vector<int>& eoff) {
  sc::SClass C{};
  C.li = li;
  C.lj = lj;
  C.ne = li + lj;
  C.nf = li + lj;
  C.lt = C.ne + C.nf;
  C.n_e = (C.ne + 1) * (C.ne + 2) * (C.ne + 3) / 6;
  C.n_f = C.n_e;
  // the reference's packed window: for ket level k an e of degree de keeps
  // m = 0 .. l_total - de - k (src/engine/os_eri.rs:600-620)
  eoff.assign((size_t)(C.nf + 1) * C.n_e, 0);
  C.maxlevel = 1;
  for (int k = 0; k <= C.nf; ++k) {
    int run = 0, ae = 0;
    for (int de = 0; de <= C.ne; ++de) {
      const int mlen = C.lt - de - k + 1;
      for (int c = 0; c < ncart_of(de); ++c) {
        eoff[(size_t)k * C.n_e + ae] = run;
        ++ae;
        run += mlen;
      }
    }
    C.slab[k] = run;
    C.maxlevel = std::max(C.maxlevel, ncart_of(k) * run);
  }
  const int na = ncart_of(li), nb = ncart_of(lj);
  const int nfr = C.n_f - li * (li + 1) * (li + 2) / 6;
  size_t o = 0;
  C.o_prims = o;
  o += (size_t)11 * std::max(1, maxpp);
  C.o_lev = o;
  o += (size_t)3 * C.maxlevel;
  C.o_cef = o;
  o += (size_t)C.n_e * C.n_f;
  C.o_bra = o;
  o += (size_t)na * nb * nfr;
  C.o_prev = o;
  o += (size_t)nb * C.n_e;
  C.o_cur = o;
  o += (size_t)nb * C.n_e;
  C.o_kprev = o;
  o += (size_t)nb * C.n_f;
  C.o_kcur = o;
  o += (size_t)nb * C.n_f;
  C.o_blk = o;
  o += (size_t)na * nb * na * nb;
  C.o_tmp = o;
  o += (size_t)na * nb * na * nb;
  C.total = o;
  return C;
}

void schwarz_kappa(const SchwarzShell& si, const SchwarzShell& sj, double* out) {
  const double d2 = (si.center[0] - sj.center[0]) * (si.center[0] - sj.center[0]) +
                    (si.center[1] - sj.center[1]) * (si.center[1] - sj.center[1]) +
                    (si.center[2] - sj.center[2]) * (si.center[2] - sj.center[2]);
  for (size_t a = 0; a < si.exps.size(); ++a)
    for (size_t b = 0; b < sj.exps.size(); ++b) {
      const double e1 = si.exps[a], e2 = sj.exps[b];
      const double z = e1 + e2;
      out[a * sj.exps.size() + b] = std::exp(-(e1 * e2 / z) * d2);
    }
}

// Auto engine of src/integrals.rs:374-388.
bool auto_picks_os(int ne, int nf, long long degree) {
  const int lt = ne + nf;
  if (lt > 16) return false;
  const long long thr = lt <= 5 ? 1 : (std::max(ne, nf) <= 6 ? 3 : 16);
  return degree >= thr;
}

bool schwarz_exact(const SchwarzShell& si, const SchwarzShell& sj, double& q) {
  const long long np = (long long)si.exps.size() * (long long)sj.exps.size();
  if (!auto_picks_os(si.l + sj.l, si.l + sj.l, np * np)) return false;
  thread_local std::vector<double> work;
  thread_local std::vector<double> kap;
  thread_local std::vector<int> eoff;
  sc::SClass C = schwarz_class_layout(si.l, sj.l, (int)np, eoff);
  C.eoff = eoff.data();
  if (work.size() < C.total) work.resize(C.total);
  kap.resize((size_t)np);
  schwarz_kappa(si, sj, kap.data());
  const sc::BoysDev B = BoysTable::get().view();
  const sc::Slice W{work.data(), 1};
  q = sc::sc_schwarz(B, C, W, sc::Team{0, 1}, si.center, sj.center, (int)si.exps.size(), (int)sj.exps.size(), si.exps.data(),
                     si.coefs.data(), sj.exps.data(), sj.coefs.data(), kap.data(), si.c2s, sj.c2s);
  return true;
}

void schwarz_exact_many(const std::vector<SchwarzShell>& shells, const std::vector<std::pair<int, int>>& pairs,
                        std::vector<double>& q, std::vector<unsigned char>& done, int nthreads) {
  q.assign(pairs.size(), 0.0);
  done.assign(pairs.size(), 0);
  if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  nthreads = std::min(nthreads, 256);
  std::atomic<size_t> next{0};
  auto work = [&] {
    for (;;) {
      const size_t lo = next.fetch_add(64);
      if (lo >= pairs.size()) return;
      const size_t hi = std::min(pairs.size(), lo + 64);
      for (size_t x = lo; x < hi; ++x) {
        double v = 0.0;
        if (schwarz_exact(shells[pairs[x].first], shells[pairs[x].second], v)) {
          q[x] = v;
          done[x] = 1;
        }
      }
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nthreads; ++t) th.emplace_back(work);
  work();
  for (auto& t : th) t.join();
}

}  // namespace igpu
