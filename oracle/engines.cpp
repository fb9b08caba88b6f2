// ORACLE — test infrastructure only (see oracle.hpp).
// L1 engines: OS/HGP (generic m-marching VRR + contracted HRR) and Rys.
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "oracle.hpp"

namespace oracle {

static const double PI = 3.14159265358979323846;

namespace {
inline Vec3 sub(const Vec3& u, const Vec3& v) { return {u[0] - v[0], u[1] - v[1], u[2] - v[2]}; }
inline double norm2(const Vec3& u) { return u[0] * u[0] + u[1] * u[1] + u[2] * u[2]; }
inline double dist2(const Vec3& u, const Vec3& v) { return norm2(sub(u, v)); }
inline Vec3 combine(double a, const Vec3& ca, double b, const Vec3& cb, double p) {
  return {(a * ca[0] + b * cb[0]) / p, (a * ca[1] + b * cb[1]) / p, (a * ca[2] + b * cb[2]) / p};
}
// os_eri.rs:116-137
inline int n_addr(int lmax) { return (lmax + 1) * (lmax + 2) * (lmax + 3) / 6; }
inline int tri_below(int d) { return d * (d + 1) * (d + 2) / 6; }
inline int addr(const Tri& t) {
  int n = t[0] + t[1] + t[2];
  int base = n * (n + 1) * (n + 2) / 6;
  int within = (n - t[0]) * (n - t[0] + 1) / 2 + t[2];
  return base + within;
}
inline int lower_axis(const Tri& t) { return t[0] > 0 ? 0 : (t[1] > 0 ? 1 : 2); }
inline Tri dec(Tri t, int i) {
  t[i] -= 1;
  return t;
}
inline Tri inc(Tri t, int i) {
  t[i] += 1;
  return t;
}
const std::vector<std::vector<Tri>>& tri_all() {
  static std::vector<std::vector<Tri>> t = [] {
    std::vector<std::vector<Tri>> v;
    for (int d = 0; d <= 4 * MAX_L + 2; ++d) v.push_back(cart_components(d));
    return v;
  }();
  return t;
}
}  // namespace

// integrals.rs:374-388
Engine select_engine(int ne, int nf, int contraction_degree) {
  int l_total = ne + nf;
  bool has_fast_kernel = std::max(ne, nf) <= 6;
  int threshold;
  if (l_total <= 5)
    threshold = 1;
  else if (l_total <= 16)
    threshold = has_fast_kernel ? 3 : 16;
  else
    return Engine::Rys;
  return contraction_degree >= threshold ? Engine::OsHgp : Engine::Rys;
}

// os_eri.rs:221-244
std::vector<PrimPair> build_pairs(const Shell& s1, const double* c1, const Shell& s2,
                                  const double* c2) {
  std::vector<PrimPair> out;
  double d2 = dist2(s1.center, s2.center);
  for (int i = 0; i < s1.n_prim(); ++i) {
    double e1 = s1.exps[i];
    for (int j = 0; j < s2.n_prim(); ++j) {
      double e2 = s2.exps[j];
      double zeta = e1 + e2;
      double kappa = std::exp(-(e1 * e2 / zeta) * d2);
      if (kappa * std::fabs(c1[i] * c2[j]) < 1e-32) continue;
      PrimPair p;
      p.zeta = zeta;
      p.center = combine(e1, s1.center, e2, s2.center, zeta);
      p.kappa = kappa;
      p.c1 = c1[i];
      p.c2 = c2[j];
      p.inv_2zeta = 0.5 / zeta;
      p.r1 = sub(p.center, s1.center);
      out.push_back(p);
    }
  }
  return out;
}

namespace {

// Full-table storage of the VRR values the reference keeps in a rolling,
// triangle-packed window: L[k][lf][ae][m].  Only the storage differs; every
// value is produced by the same expression in the same order.
struct VrrScratch {
  std::vector<double> lv;
  int n_e = 0, mlen = 0;
  std::vector<size_t> koff;
  double& at(int k, int lf, int ae, int m) {
    return lv[koff[k] + ((size_t)lf * n_e + ae) * mlen + m];
  }
};

// os_eri.rs:2860-3020
void vrr_primitive(const PrimPair& bra, const PrimPair& ket, int ne, int nf, int l_total,
                   int n_e, int n_f, double scale, VrrScratch& S, double* c_ef) {
  const auto& tri = tri_all();
  double p = bra.zeta, q = ket.zeta;
  const Vec3& pc = bra.center;
  const Vec3& qc = ket.center;
  double pq = p + q;
  double rho = p * q / pq;
  Vec3 pq_vec = sub(pc, qc);
  double t = rho * norm2(pq_vec);
  Vec3 w = {(p * pc[0] + q * qc[0]) / pq, (p * pc[1] + q * qc[1]) / pq,
            (p * pc[2] + q * qc[2]) / pq};
  Vec3 wp = sub(w, pc);
  Vec3 wq = sub(w, qc);
  double pref = 2.0 * PI * PI * std::sqrt(PI) / (p * q * std::sqrt(pq)) * bra.kappa * ket.kappa;
  double fm[4 * MAX_L + 3];
  boys_array(l_total, t, fm);
  for (int m = 0; m <= l_total; ++m) S.at(0, 0, 0, m) = pref * fm[m];
  double inv_2p = bra.inv_2zeta, inv_2q = ket.inv_2zeta;
  double inv_2pq = 0.5 / pq;
  double q_over_pq = q / pq;
  double p_over_pq = p / pq;
  const Vec3& pa = bra.r1;
  const Vec3& qcen = ket.r1;

  // Phase A: bra ladder at f-degree 0.
  for (int na = 1; na <= ne; ++na) {
    for (const Tri& te : tri[na]) {
      int i = lower_axis(te);
      int s1a = addr(dec(te, i));
      int mmax = l_total - na;
      double coef2 = (double)(te[i] - 1) * inv_2p;
      bool has2 = te[i] >= 2;
      int s2a = has2 ? addr(dec(dec(te, i), i)) : 0;
      int dst = addr(te);
      for (int m = 0; m <= mmax; ++m) {
        double v = pa[i] * S.at(0, 0, s1a, m) + wp[i] * S.at(0, 0, s1a, m + 1);
        if (has2) v += coef2 * (S.at(0, 0, s2a, m) - q_over_pq * S.at(0, 0, s2a, m + 1));
        S.at(0, 0, dst, m) = v;
      }
    }
  }
  for (int ae = 0; ae < n_e; ++ae) c_ef[(size_t)ae * n_f] += scale * S.at(0, 0, ae, 0);

  // Phase B: ket raise over f-degree k.
  for (int k = 1; k <= nf; ++k) {
    for (const Tri& tf : tri[k]) {
      int j = lower_axis(tf);
      Tri f1 = dec(tf, j);
      int lf1 = cart_index(f1);
      double coef2 = (double)(tf[j] - 1) * inv_2q;
      bool has2 = tf[j] >= 2;
      int lf2 = has2 ? cart_index(dec(f1, j)) : 0;
      int lf = cart_index(tf);
      for (int nadeg = 0; nadeg <= ne; ++nadeg) {
        for (const Tri& te : tri[nadeg]) {
          int ea = addr(te);
          bool has_cross = te[j] >= 1;
          double cross_coef = has_cross ? (double)te[j] * inv_2pq : 0.0;
          int ce = has_cross ? addr(dec(te, j)) : 0;
          int mmax = l_total - nadeg - k;
          for (int m = 0; m <= mmax; ++m) {
            double v = qcen[j] * S.at(k - 1, lf1, ea, m) + wq[j] * S.at(k - 1, lf1, ea, m + 1);
            if (has2)
              v += coef2 * (S.at(k - 2, lf2, ea, m) - p_over_pq * S.at(k - 2, lf2, ea, m + 1));
            if (has_cross) v += cross_coef * S.at(k - 1, lf1, ce, m + 1);
            S.at(k, lf, ea, m) = v;
          }
        }
      }
    }
    for (const Tri& tf : tri[k]) {
      int lf = cart_index(tf);
      int af = addr(tf);
      for (int ae = 0; ae < n_e; ++ae) c_ef[(size_t)ae * n_f + af] += scale * S.at(k, lf, ae, 0);
    }
  }
}

// os_eri.rs:3040-3143
void hrr_and_scatter(int la, int lb, int lc, int ld, int n_f, const double* c_ef, const Vec3& ab,
                     const Vec3& cd, double* out) {
  const auto& tri = tri_all();
  int na = n_cart(la), nb = n_cart(lb), nc = n_cart(lc), nd = n_cart(ld);
  int ne = la + lb, nf = lc + ld;
  int n_e = n_addr(ne);
  int f_base = tri_below(lc);
  int nf_range = n_f - f_base;
  std::vector<double> bra((size_t)na * nb * nf_range, NAN);
  std::vector<double> prev((size_t)n_cart(lb) * n_e, NAN), cur((size_t)n_cart(lb) * n_e, NAN);
  for (int f_global = f_base; f_global < n_f; ++f_global) {
    int jf = f_global - f_base;
    for (int dg = la; dg <= ne; ++dg)
      for (const Tri& a : tri[dg]) {
        int ae = addr(a);
        prev[ae] = c_ef[(size_t)ae * n_f + f_global];
      }
    for (int kb = 1; kb <= lb; ++kb) {
      int ibw = 0;
      for (const Tri& b : tri[kb]) {
        int i = lower_axis(b);
        int b1w = cart_index(dec(b, i));
        for (int dg = la; dg <= ne - kb; ++dg)
          for (const Tri& a : tri[dg]) {
            int ae = addr(a);
            int a1e = addr(inc(a, i));
            cur[(size_t)ibw * n_e + ae] =
                prev[(size_t)b1w * n_e + a1e] + ab[i] * prev[(size_t)b1w * n_e + ae];
          }
        ++ibw;
      }
      std::swap(prev, cur);
    }
    int ib = 0;
    for (const Tri& b : tri[lb]) {
      int ibw = cart_index(b);
      int ia = 0;
      for (const Tri& a : tri[la]) {
        bra[((size_t)ia * nb + ib) * nf_range + jf] = prev[(size_t)ibw * n_e + addr(a)];
        ++ia;
      }
      ++ib;
    }
  }
  std::vector<double> kprev((size_t)n_cart(ld) * n_f, NAN), kcur((size_t)n_cart(ld) * n_f, NAN);
  for (int ia = 0; ia < na; ++ia)
    for (int ib = 0; ib < nb; ++ib) {
      size_t brarow = ((size_t)ia * nb + ib) * nf_range;
      for (int dg = lc; dg <= nf; ++dg)
        for (const Tri& c : tri[dg]) {
          int ce = addr(c);
          kprev[ce] = bra[brarow + (ce - f_base)];
        }
      for (int kd = 1; kd <= ld; ++kd) {
        int idw = 0;
        for (const Tri& d : tri[kd]) {
          int j = lower_axis(d);
          int d1w = cart_index(dec(d, j));
          for (int dg = lc; dg <= nf - kd; ++dg)
            for (const Tri& c : tri[dg]) {
              int ce = addr(c);
              int c1e = addr(inc(c, j));
              kcur[(size_t)idw * n_f + ce] =
                  kprev[(size_t)d1w * n_f + c1e] + cd[j] * kprev[(size_t)d1w * n_f + ce];
            }
          ++idw;
        }
        std::swap(kprev, kcur);
      }
      int ic = 0;
      for (const Tri& c : tri[lc]) {
        int ce = addr(c);
        for (int id = 0; id < nd; ++id)
          out[(((size_t)ia * nb + ib) * nc + ic) * nd + id] += kprev[(size_t)id * n_f + ce];
        ++ic;
      }
    }
}
}  // namespace

// os_eri.rs:455-697 (the specialised VRR kernels are bit-identical to the
// generic vrr_primitive, os_eri.rs:1007-1017, so only the generic one is
// restated).
void os_shell_quartet(const Shell& a, const Shell& b, const Shell& c, const Shell& d,
                      const std::vector<PrimPair>& bra_pairs,
                      const std::vector<PrimPair>& ket_pairs, int la, int lb, int lc, int ld,
                      double* out) {
  int ne = la + lb, nf = lc + ld, l_total = ne + nf;
  int n_e = n_addr(ne), n_f = n_addr(nf);
  if (l_total == 0) {
    // (ss|ss) fast path, os_eri.rs:500-536.
    double two_pi_2_5 = 2.0 * PI * PI * std::sqrt(PI);
    double acc = 0.0;
    double f0[1];
    for (const PrimPair& br : bra_pairs) {
      double bc = br.c1 * br.c2;
      double p = br.zeta;
      for (const PrimPair& k : ket_pairs) {
        double q = k.zeta;
        double pq = p + q;
        double t = (p * q / pq) * dist2(br.center, k.center);
        double pref = two_pi_2_5 / (p * q * std::sqrt(pq)) * br.kappa * k.kappa;
        boys_array(0, t, f0);
        acc += (bc * k.c1) * k.c2 * (pref * f0[0]);
      }
    }
    out[0] += acc;
    return;
  }
  std::vector<double> c_ef((size_t)n_e * n_f, 0.0);
  thread_local VrrScratch S;
  S.n_e = n_e;
  S.mlen = l_total + 2;
  S.koff.assign(nf + 1, 0);
  size_t tot = 0;
  for (int k = 0; k <= nf; ++k) {
    S.koff[k] = tot;
    tot += (size_t)n_cart(k) * n_e * S.mlen;
  }
  if (S.lv.size() < tot) S.lv.resize(tot);
  for (const PrimPair& br : bra_pairs) {
    double bra_coef = br.c1 * br.c2;
    for (const PrimPair& k : ket_pairs) {
      double scale = (bra_coef * k.c1) * k.c2;
      vrr_primitive(br, k, ne, nf, l_total, n_e, n_f, scale, S, c_ef.data());
    }
  }
  Vec3 ab = sub(a.center, b.center);
  Vec3 cd = sub(c.center, d.center);
  hrr_and_scatter(la, lb, lc, ld, n_f, c_ef.data(), ab, cd, out);
}

// ---------------------------------------------------------------- Rys
// engine/rys.rs:121-309
namespace {
constexpr int L1 = MAX_L + 2;      // one extra: gradient raises l by one
constexpr int LT1 = 2 * MAX_L + 3;
using Axis4 = double[L1][L1][L1][L1];

void build_axis(int la, int lb, int lc, int ld, double c00, double cp0, double b10, double b01,
                double b00, double ab, double cd, Axis4& out4) {
  int nbra = la + lb, nket = lc + ld;
  double g[LT1][LT1];
  g[0][0] = 1.0;
  if (nbra >= 1) g[1][0] = c00;
  for (int n = 1; n < nbra; ++n) g[n + 1][0] = c00 * g[n][0] + (double)n * b10 * g[n - 1][0];
  for (int m = 0; m < nket; ++m)
    for (int n = 0; n <= nbra; ++n) {
      double term = cp0 * g[n][m];
      if (m >= 1) term += (double)m * b01 * g[n][m - 1];
      if (n >= 1) term += (double)n * b00 * g[n - 1][m];
      g[n][m + 1] = term;
    }
  static thread_local double h[LT1][L1][LT1];
  for (int i = 0; i <= nbra; ++i)
    for (int m = 0; m <= nket; ++m) h[i][0][m] = g[i][m];
  for (int j = 1; j <= lb; ++j)
    for (int i = 0; i <= nbra - j; ++i)
      for (int m = 0; m <= nket; ++m) h[i][j][m] = h[i + 1][j - 1][m] + ab * h[i][j - 1][m];
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j <= lb; ++j) {
      double t[LT1][L1];
      for (int k = 0; k <= nket; ++k) t[k][0] = h[i][j][k];
      for (int l = 1; l <= ld; ++l)
        for (int k = 0; k <= nket - l; ++k) t[k][l] = t[k + 1][l - 1] + cd * t[k][l - 1];
      for (int k = 0; k <= lc; ++k)
        for (int l = 0; l <= ld; ++l) out4[i][j][k][l] = t[k][l];
    }
}
}  // namespace

namespace {
double g_rys_erf_omega = 0.0;
}
void set_rys_erf_omega(double omega) { g_rys_erf_omega = omega; }
double rys_erf_omega() { return g_rys_erf_omega; }

void rys_prim_quartet(double ea, const Vec3& A, int la, double eb, const Vec3& B, int lb,
                      double ec, const Vec3& C, int lc, double ed, const Vec3& D, int ld,
                      double scale, double* out) {
  int na = n_cart(la), nb = n_cart(lb), nc = n_cart(lc), nd = n_cart(ld);
  double p = ea + eb;
  double q = ec + ed;
  Vec3 p_ctr = combine(ea, A, eb, B, p);
  Vec3 q_ctr = combine(ec, C, ed, D, q);
  double kab = std::exp(-(ea * eb / p) * dist2(A, B));
  double kcd = std::exp(-(ec * ed / q) * dist2(C, D));
  double pq = p + q;
  double rho = p * q / pq;
  Vec3 pq_vec = sub(p_ctr, q_ctr);
  double t = rho * norm2(pq_vec);
  double pref = 2.0 * PI * PI * std::sqrt(PI) / (p * q * std::sqrt(pq)) * kab * kcd;
  int l_total = la + lb + lc + ld;
  int nroots = l_total / 2 + 1;
  double roots[MAX_RYS_ROOTS], wts[MAX_RYS_ROOTS];
  const double omega = rys_erf_omega();
  if (omega > 0.0) {
    // erf(omega r)/r (crates/integral/src/engine/rys.rs:163-175): quadrature at s*T, roots
    // scaled by s, weights by sqrt(s)
    double s = omega * omega / (rho + omega * omega);
    rys_roots_weights(nroots, s * t, roots, wts);
    double sqrt_s = std::sqrt(s);
    for (int r = 0; r < nroots; ++r) roots[r] *= s;
    for (int r = 0; r < nroots; ++r) wts[r] *= sqrt_s;
  } else {
    rys_roots_weights(nroots, t, roots, wts);
  }
  Vec3 pa = sub(p_ctr, A), qc = sub(q_ctr, C), ab = sub(A, B), cd = sub(C, D);
  const auto& tri = tri_all();
  const std::vector<Tri>&ca = tri[la], &cb = tri[lb], &cc = tri[lc], &cdv = tri[ld];
  static thread_local Axis4 ix, iy, iz;
  for (int r = 0; r < nroots; ++r) {
    double x = roots[r];
    double b00 = x / (2.0 * pq);
    double b10 = (1.0 - x * q / pq) / (2.0 * p);
    double b01 = (1.0 - x * p / pq) / (2.0 * q);
    double cq = x * q / pq;
    double cp = x * p / pq;
    Axis4* outs[3] = {&ix, &iy, &iz};
    for (int axis = 0; axis < 3; ++axis) {
      double c00 = pa[axis] - cq * pq_vec[axis];
      double cp0 = qc[axis] + cp * pq_vec[axis];
      build_axis(la, lb, lc, ld, c00, cp0, b10, b01, b00, ab[axis], cd[axis], *outs[axis]);
    }
    double pw = scale * pref * wts[r];
    for (int ia = 0; ia < na; ++ia)
      for (int ib = 0; ib < nb; ++ib)
        for (int ic = 0; ic < nc; ++ic)
          for (int id = 0; id < nd; ++id) {
            const Tri &a = ca[ia], &b = cb[ib], &c = cc[ic], &d = cdv[id];
            double v = ix[a[0]][b[0]][c[0]][d[0]] * iy[a[1]][b[1]][c[1]][d[1]] *
                       iz[a[2]][b[2]][c[2]][d[2]];
            out[(((size_t)ia * nb + ib) * nc + ic) * nd + id] += pw * v;
          }
  }
}

}  // namespace oracle
