// Exact Schwarz bounds on the host.
//
// The screened quartet list is decided by comparisons Q_ij * Q_kl (* max|D|)
// against a threshold, so the list equals the reference's bit for bit only if
// every Q is the reference's bit for bit.  The reference takes Q from its own
// FP64 engines (Basis::schwarz_bounds, src/integrals.rs:842-862) under the
// Auto policy (src/integrals.rs:374-388), which picks the Obara-Saika /
// Head-Gordon-Pople engine for every diagonal quartet of a contracted basis.
// This file evaluates those diagonal quartets with the same arithmetic in the
// same order: primitive pairs (src/engine/os_eri.rs:221-244), the Boys ladder
// from its interpolation table (src/math/boys.rs:63-431), the m-marching
// vertical recurrence (src/engine/os_eri.rs:2860-3020; the reference's
// specialised kernels are bit-identical to it, os_eri.rs:1007-1017), the
// contracted horizontal recurrence (os_eri.rs:3040-3143), the (ss|ss) fast
// path (os_eri.rs:500-536) and the per-axis c2s transform
// (src/spherical.rs:121-179).  The build compiles this file without
// floating-point contraction, so every product and sum rounds as in Rust.
// Only libm's exp and pow are shared with the reference (same library on the
// same host); sqrt and division are correctly rounded everywhere.
#include "host_schwarz.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <thread>

#include "host_math.hpp"

namespace igpu {
namespace {

constexpr double kPi = 3.14159265358979323846;
using V3 = std::array<double, 3>;

// ------------------------------------------------------------------ Boys

// Table of F_0..F_32 and e^{-T0} on the grid T0 = 0.1 i, i = 0..930, and the
// Taylor / downward-recurrence evaluation of the reference.
class Boys {
 public:
  static constexpr int kMaxM = 24;
  static constexpr int kTaylor = 8;
  static constexpr int kOrders = kMaxM + kTaylor + 1;  // orders stored per grid point
  static constexpr int kRow = kOrders + 1;             // plus e^{-T0}

  static const Boys& get() {
    static const Boys b;
    return b;
  }

  // F_0 .. F_mmax at t into f[0..mmax].
  void ladder(int mmax, double t, double* f) const {
    if (t < tmax_ && mmax + kTaylor < kOrders) {
      const size_t i = (size_t)std::round(t * (1.0 / h_));
      const double nd = (double)i * h_ - t;  // -(t - T0)
      const double* row = tab_.data() + i * kRow;
      double top = row[mmax + kTaylor] * inv_fact_[kTaylor];
      for (int k = kTaylor - 1; k >= 0; --k) top = top * nd + row[mmax + k] * inv_fact_[k];
      f[mmax] = top;
      if (mmax > 0) {
        double ep = inv_fact_[kTaylor];
        for (int k = kTaylor - 1; k >= 0; --k) ep = ep * nd + inv_fact_[k];
        const double et = row[kOrders] * ep;
        const double two_t = 2.0 * t;
        for (int m = mmax; m > 0; --m) f[m - 1] = (two_t * f[m] + et) * inv_odd_[m];
      }
      return;
    }
    reference(mmax, t, f);
  }

 private:
  Boys() {
    inv_fact_[0] = 1.0;
    for (int k = 1; k <= kTaylor; ++k) inv_fact_[k] = inv_fact_[k - 1] / (double)k;
    inv_odd_[0] = 1.0;
    for (int m = 1; m <= kMaxM; ++m) inv_odd_[m] = 1.0 / (double)(2 * m - 1);
    tmax_ = 33.0 + 2.5 * (double)kMaxM;
    const size_t ngrid = (size_t)(tmax_ / h_);
    tab_.assign((ngrid + 1) * kRow, 0.0);
    for (size_t i = 0; i <= ngrid; ++i) {
      const double t0 = (double)i * h_;
      double* row = tab_.data() + i * kRow;
      reference(kOrders - 1, t0, row);
      row[kOrders] = std::exp(-t0);
    }
  }

  static double boundary(int m) { return 33.0 + 2.5 * (double)m; }

  // Top order by the positive series below the asymptotic boundary, else the
  // large-T closed form; then the downward recurrence.
  static void reference(int mmax, double t, double* f) {
    const double et = std::exp(-t);
    if (t < boundary(mmax)) {
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
      double v = 0.5 * std::sqrt(kPi / t);
      const double two_t = 2.0 * t;
      for (int k = 1; k <= mmax; ++k) v *= (double)(2 * k - 1) / two_t;
      f[mmax] = v;
    }
    for (int m = mmax; m > 0; --m) f[m - 1] = (2.0 * t * f[m] + et) / (double)(2 * m - 1);
  }

  double h_ = 0.1;
  double tmax_ = 0.0;
  double inv_fact_[kTaylor + 1];
  double inv_odd_[kMaxM + 1];
  std::vector<double> tab_;
};

// ------------------------------------------------------ angular bookkeeping

struct Tri {
  int x, y, z;
  int operator[](int a) const { return a == 0 ? x : (a == 1 ? y : z); }
};
inline int deg_below(int d) { return d * (d + 1) * (d + 2) / 6; }
inline int ncart_of(int l) { return (l + 1) * (l + 2) / 2; }
inline int within(const Tri& t) {  // index inside its degree (x descending, then y)
  const int r = t.y + t.z;
  return r * (r + 1) / 2 + t.z;
}
inline int addr_of(const Tri& t) { return deg_below(t.x + t.y + t.z) + within(t); }
inline int low_axis(const Tri& t) { return t.x > 0 ? 0 : (t.y > 0 ? 1 : 2); }
inline Tri step(Tri t, int a, int d) {
  if (a == 0) t.x += d;
  if (a == 1) t.y += d;
  if (a == 2) t.z += d;
  return t;
}
// Cartesian triples by degree in the reference's order (src/math/am.rs:15-55).
const std::vector<std::vector<Tri>>& triples() {
  static const std::vector<std::vector<Tri>> T = [] {
    std::vector<std::vector<Tri>> v;
    for (int d = 0; d <= 4 * MAX_L + 2; ++d) {
      std::vector<Tri> row;
      for (auto& c : cart_comps(d)) row.push_back({c[0], c[1], c[2]});
      v.push_back(row);
    }
    return v;
  }();
  return T;
}

// ---------------------------------------------------------- primitive pairs

struct Prim2 {
  double zeta, kappa, c1, c2, inv2z;
  V3 P, PA;
};

std::vector<Prim2> prim_pairs(const SchwarzShell& s1, const SchwarzShell& s2) {
  std::vector<Prim2> out;
  const double d2 = (s1.center[0] - s2.center[0]) * (s1.center[0] - s2.center[0]) +
                    (s1.center[1] - s2.center[1]) * (s1.center[1] - s2.center[1]) +
                    (s1.center[2] - s2.center[2]) * (s1.center[2] - s2.center[2]);
  for (size_t a = 0; a < s1.exps.size(); ++a)
    for (size_t b = 0; b < s2.exps.size(); ++b) {
      const double e1 = s1.exps[a], e2 = s2.exps[b];
      const double c1 = s1.coefs[a], c2 = s2.coefs[b];
      const double z = e1 + e2;
      const double kappa = std::exp(-(e1 * e2 / z) * d2);
      if (kappa * std::fabs(c1 * c2) < 1e-32) continue;
      Prim2 p;
      p.zeta = z;
      p.kappa = kappa;
      p.c1 = c1;
      p.c2 = c2;
      p.inv2z = 0.5 / z;
      for (int k = 0; k < 3; ++k) {
        p.P[k] = (e1 * s1.center[k] + e2 * s2.center[k]) / z;
        p.PA[k] = p.P[k] - s1.center[k];
      }
      out.push_back(p);
    }
  return out;
}

// ------------------------------------------------------- OS/HGP shell quartet

// Per-thread work space of the vertical recurrence: level k (ket degree) holds
// [ncart(k)][n_e][mlen] values, m = 0..l_total - deg(e) - k.
struct Work {
  std::vector<std::vector<double>> lev;
  std::vector<double> cef, bra, prev, cur, kprev, kcur, blk, tmp;
};

void vrr_into(const Prim2& b, const Prim2& k, int ne, int nf, int lt, int n_e, int n_f, int mlen, double scale,
              Work& W, double* cef) {
  const auto& tri = triples();
  const double p = b.zeta, q = k.zeta;
  const double pq = p + q;
  const double rho = p * q / pq;
  const V3 d = {b.P[0] - k.P[0], b.P[1] - k.P[1], b.P[2] - k.P[2]};
  const double t = rho * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  V3 w;
  for (int a = 0; a < 3; ++a) w[a] = (p * b.P[a] + q * k.P[a]) / pq;
  const V3 wp = {w[0] - b.P[0], w[1] - b.P[1], w[2] - b.P[2]};
  const V3 wq = {w[0] - k.P[0], w[1] - k.P[1], w[2] - k.P[2]};
  const double pref = 2.0 * kPi * kPi * std::sqrt(kPi) / (p * q * std::sqrt(pq)) * b.kappa * k.kappa;
  double fm[4 * MAX_L + 3];
  Boys::get().ladder(lt, t, fm);
  auto at = [&](int kd, int lf, int ae) { return W.lev[kd].data() + ((size_t)lf * n_e + ae) * mlen; };
  {
    double* s0 = at(0, 0, 0);
    for (int m = 0; m <= lt; ++m) s0[m] = pref * fm[m];
  }
  const double inv2pq = 0.5 / pq, q_pq = q / pq, p_pq = p / pq;
  // bra ladder at ket degree 0
  for (int na = 1; na <= ne; ++na)
    for (const Tri& te : tri[na]) {
      const int i = low_axis(te);
      const double* s1 = at(0, 0, addr_of(step(te, i, -1)));
      const bool two = te[i] >= 2;
      const double c2 = (double)(te[i] - 1) * b.inv2z;
      const double* s2 = two ? at(0, 0, addr_of(step(step(te, i, -1), i, -1))) : nullptr;
      double* dst = at(0, 0, addr_of(te));
      for (int m = 0; m <= lt - na; ++m) {
        double v = b.PA[i] * s1[m] + wp[i] * s1[m + 1];
        if (two) v += c2 * (s2[m] - q_pq * s2[m + 1]);
        dst[m] = v;
      }
    }
  for (int ae = 0; ae < n_e; ++ae) cef[(size_t)ae * n_f] += scale * at(0, 0, ae)[0];
  // ket raise
  for (int kd = 1; kd <= nf; ++kd) {
    for (const Tri& tf : tri[kd]) {
      const int j = low_axis(tf);
      const Tri f1 = step(tf, j, -1);
      const int lf1 = within(f1);
      const bool two = tf[j] >= 2;
      const double c2 = (double)(tf[j] - 1) * k.inv2z;
      const int lf2 = two ? within(step(f1, j, -1)) : 0;
      const int lf = within(tf);
      for (int nd = 0; nd <= ne; ++nd)
        for (const Tri& te : tri[nd]) {
          const int ea = addr_of(te);
          const bool cross = te[j] >= 1;
          const double cc = cross ? (double)te[j] * inv2pq : 0.0;
          const double* sx = cross ? at(kd - 1, lf1, addr_of(step(te, j, -1))) : nullptr;
          const double* s1 = at(kd - 1, lf1, ea);
          const double* s2 = two ? at(kd - 2, lf2, ea) : nullptr;
          double* dst = at(kd, lf, ea);
          for (int m = 0; m <= lt - nd - kd; ++m) {
            double v = k.PA[j] * s1[m] + wq[j] * s1[m + 1];
            if (two) v += c2 * (s2[m] - p_pq * s2[m + 1]);
            if (cross) v += cc * sx[m + 1];
            dst[m] = v;
          }
        }
    }
    for (const Tri& tf : tri[kd]) {
      const int lf = within(tf), af = addr_of(tf);
      for (int ae = 0; ae < n_e; ++ae) cef[(size_t)ae * n_f + af] += scale * at(kd, lf, ae)[0];
    }
  }
}

// Contracted HRR, bra (A -> B) then ket (C -> D), into out[a][b][c][d]
// (zero on entry).
void hrr_into(int la, int lb, int lc, int ld, int n_f, const double* cef, const V3& ab, const V3& cd, Work& W,
              double* out) {
  const auto& tri = triples();
  const int na = ncart_of(la), nb = ncart_of(lb), nc = ncart_of(lc), nd = ncart_of(ld);
  const int ne = la + lb, nf = lc + ld;
  const int n_e = deg_below(ne + 1);
  const int fb = deg_below(lc);
  const int nfr = n_f - fb;
  W.bra.assign((size_t)na * nb * nfr, 0.0);
  W.prev.assign((size_t)nb * n_e, 0.0);
  W.cur.assign((size_t)nb * n_e, 0.0);
  for (int fg = fb; fg < n_f; ++fg) {
    for (int dg = la; dg <= ne; ++dg)
      for (const Tri& a : tri[dg]) W.prev[addr_of(a)] = cef[(size_t)addr_of(a) * n_f + fg];
    for (int kb = 1; kb <= lb; ++kb) {
      int ibw = 0;
      for (const Tri& bt : tri[kb]) {
        const int i = low_axis(bt);
        const int b1 = within(step(bt, i, -1));
        for (int dg = la; dg <= ne - kb; ++dg)
          for (const Tri& a : tri[dg]) {
            const int ae = addr_of(a);
            W.cur[(size_t)ibw * n_e + ae] =
                W.prev[(size_t)b1 * n_e + addr_of(step(a, i, 1))] + ab[i] * W.prev[(size_t)b1 * n_e + ae];
          }
        ++ibw;
      }
      std::swap(W.prev, W.cur);
    }
    int ib = 0;
    for (const Tri& bt : tri[lb]) {
      int ia = 0;
      for (const Tri& a : tri[la]) {
        W.bra[((size_t)ia * nb + ib) * nfr + (fg - fb)] = W.prev[(size_t)within(bt) * n_e + addr_of(a)];
        ++ia;
      }
      ++ib;
    }
  }
  W.kprev.assign((size_t)nd * n_f, 0.0);
  W.kcur.assign((size_t)nd * n_f, 0.0);
  for (int ia = 0; ia < na; ++ia)
    for (int ib = 0; ib < nb; ++ib) {
      const size_t row = ((size_t)ia * nb + ib) * nfr;
      for (int dg = lc; dg <= nf; ++dg)
        for (const Tri& c : tri[dg]) W.kprev[addr_of(c)] = W.bra[row + (addr_of(c) - fb)];
      for (int kd = 1; kd <= ld; ++kd) {
        int idw = 0;
        for (const Tri& dt : tri[kd]) {
          const int j = low_axis(dt);
          const int d1 = within(step(dt, j, -1));
          for (int dg = lc; dg <= nf - kd; ++dg)
            for (const Tri& c : tri[dg]) {
              const int ce = addr_of(c);
              W.kcur[(size_t)idw * n_f + ce] =
                  W.kprev[(size_t)d1 * n_f + addr_of(step(c, j, 1))] + cd[j] * W.kprev[(size_t)d1 * n_f + ce];
            }
          ++idw;
        }
        std::swap(W.kprev, W.kcur);
      }
      int ic = 0;
      for (const Tri& c : tri[lc]) {
        for (int id = 0; id < nd; ++id)
          out[(((size_t)ia * nb + ib) * nc + ic) * nd + id] += W.kprev[(size_t)id * n_f + addr_of(c)];
        ++ic;
      }
    }
}

// Cartesian block of (s1 s2 | s1 s2) into W.blk.
void diagonal_block(const SchwarzShell& s1, const SchwarzShell& s2, Work& W) {
  const int la = s1.l, lb = s2.l;
  const int ne = la + lb, nf = ne, lt = ne + nf;
  const std::vector<Prim2> pr = prim_pairs(s1, s2);
  const size_t nblk = (size_t)ncart_of(la) * ncart_of(lb) * ncart_of(la) * ncart_of(lb);
  W.blk.assign(nblk, 0.0);
  if (lt == 0) {
    const double two_pi_2_5 = 2.0 * kPi * kPi * std::sqrt(kPi);
    double acc = 0.0;
    for (const Prim2& b : pr) {
      const double bc = b.c1 * b.c2;
      const double p = b.zeta;
      for (const Prim2& k : pr) {
        const double q = k.zeta;
        const double pq = p + q;
        const double d2 = (b.P[0] - k.P[0]) * (b.P[0] - k.P[0]) + (b.P[1] - k.P[1]) * (b.P[1] - k.P[1]) +
                          (b.P[2] - k.P[2]) * (b.P[2] - k.P[2]);
        const double t = (p * q / pq) * d2;
        const double pref = two_pi_2_5 / (p * q * std::sqrt(pq)) * b.kappa * k.kappa;
        double f0;
        Boys::get().ladder(0, t, &f0);
        acc += (bc * k.c1) * k.c2 * (pref * f0);
      }
    }
    W.blk[0] += acc;
    return;
  }
  const int n_e = deg_below(ne + 1), n_f = deg_below(nf + 1), mlen = lt + 2;
  W.cef.assign((size_t)n_e * n_f, 0.0);
  if ((int)W.lev.size() < nf + 1) W.lev.resize(nf + 1);
  for (int kd = 0; kd <= nf; ++kd) {
    const size_t need = (size_t)ncart_of(kd) * n_e * mlen;
    if (W.lev[kd].size() < need) W.lev[kd].resize(need);
  }
  for (const Prim2& b : pr) {
    const double bc = b.c1 * b.c2;
    for (const Prim2& k : pr) vrr_into(b, k, ne, nf, lt, n_e, n_f, mlen, (bc * k.c1) * k.c2, W, W.cef.data());
  }
  const V3 ab = {s1.center[0] - s2.center[0], s1.center[1] - s2.center[1], s1.center[2] - s2.center[2]};
  hrr_into(la, lb, la, lb, n_f, W.cef.data(), ab, ab, W, W.blk.data());
}

// The reference's per-axis transform: axes 0..3 in order, zero matrix entries
// skipped, each output element accumulated over the input index in order.
void transform_axes(Work& W, int dims[4], const double* const mats[4], const int nout[4]) {
  for (int axis = 0; axis < 4; ++axis) {
    if (!mats[axis]) continue;
    const int n_in = dims[axis], n_o = nout[axis];
    size_t outer = 1, inner = 1;
    for (int q = 0; q < axis; ++q) outer *= dims[q];
    for (int q = axis + 1; q < 4; ++q) inner *= dims[q];
    W.tmp.assign(outer * n_o * inner, 0.0);
    const double* M = mats[axis];
    for (size_t o = 0; o < outer; ++o)
      for (int r = 0; r < n_o; ++r) {
        double* dst = W.tmp.data() + (o * n_o + r) * inner;
        for (int j = 0; j < n_in; ++j) {
          const double m = M[(size_t)r * n_in + j];
          if (m == 0.0) continue;
          const double* src = W.blk.data() + (o * n_in + j) * inner;
          for (size_t s = 0; s < inner; ++s) dst[s] += m * src[s];
        }
      }
    dims[axis] = n_o;
    std::swap(W.blk, W.tmp);
  }
}

}  // namespace

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
  thread_local Work W;
  diagonal_block(si, sj, W);
  int dims[4] = {ncart_of(si.l), ncart_of(sj.l), ncart_of(si.l), ncart_of(sj.l)};
  const double* mats[4] = {si.c2s, sj.c2s, si.c2s, sj.c2s};
  const int nout[4] = {2 * si.l + 1, 2 * sj.l + 1, 2 * si.l + 1, 2 * sj.l + 1};
  transform_axes(W, dims, mats, nout);
  const int ni = dims[0], nj = dims[1];
  double mx = 0.0;
  for (int mu = 0; mu < ni; ++mu)
    for (int nu = 0; nu < nj; ++nu) mx = std::fmax(mx, std::fabs(W.blk[(((size_t)mu * nj + nu) * ni + mu) * nj + nu]));
  q = std::sqrt(mx);
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
