// ORACLE — test infrastructure only (see oracle.hpp).
// L0 math: angular momentum, normalisation, Boys function, Rys roots/weights
// with the Chebyshev-table generator, and the Cartesian->spherical matrices.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <numeric>

#include "oracle.hpp"

namespace oracle {

static const double PI = 3.14159265358979323846;  // std::f64::consts::PI

// --- src/math/am.rs:23-31: lx descending outer, ly descending inner.
std::vector<Tri> cart_components(int l) {
  std::vector<Tri> out;
  for (int lx = l; lx >= 0; --lx)
    for (int ly = l - lx; ly >= 0; --ly) out.push_back({lx, ly, l - lx - ly});
  return out;
}

// --- src/math/am.rs:51-55
int cart_index(const Tri& c) {
  int l = c[0] + c[1] + c[2];
  int d = l - c[0];
  return d * (d + 1) / 2 + c[2];
}

// Rust `f64::powi` compiles to LLVM's `__powidf2`: square-and-multiply over
// the exponent bits, reciprocal for negative exponents.
double powi(double a, int b) {
  const bool recip = b < 0;
  double r = 1.0;
  for (;;) {
    if (b & 1) r *= a;
    b /= 2;
    if (b == 0) break;
    a *= a;
  }
  return recip ? 1.0 / r : r;
}

// --- src/math/norm.rs:30-38
double double_factorial(long n) {
  long k = n;
  double acc = 1.0;
  while (k > 1) {
    acc *= (double)k;
    k -= 2;
  }
  return acc;
}

// --- src/math/norm.rs:42-49
double cart_norm(double alpha, int lx, int ly, int lz) {
  int l = lx + ly + lz;
  double df = double_factorial(2L * lx - 1) * double_factorial(2L * ly - 1) *
              double_factorial(2L * lz - 1);
  double two_alpha_over_pi = 2.0 * alpha / PI;
  return std::pow(two_alpha_over_pi, 0.75) * std::sqrt(powi(4.0 * alpha, l)) / std::sqrt(df);
}

// --- src/shell.rs:182-187
double Shell::primitive_coeff(int i) const {
  if (exps[i] == 0.0) return coefs[i];
  return coefs[i] * cart_norm(exps[i], l, 0, 0);
}

// ============================================================ Boys function
// src/math/boys.rs:63-431

double asymptotic_boundary(int m) { return 33.0 + 2.5 * (double)m; }

namespace {
constexpr int BOYS_MAX_M = 24;
constexpr int BOYS_K = 8;
constexpr int BOYS_STRIDE = BOYS_MAX_M + BOYS_K + 1;  // 33
constexpr int BOYS_ROW = BOYS_STRIDE + 1;             // 34
constexpr double BOYS_H = 0.1;
const double BOYS_TABLE_TMAX = 33.0 + 2.5 * (double)BOYS_MAX_M;  // 93

struct BoysConsts {
  double inv_fact[BOYS_K + 1];
  double inv_odd[BOYS_MAX_M + 1];
  BoysConsts() {
    inv_fact[0] = 1.0;
    for (int k = 1; k <= BOYS_K; ++k) inv_fact[k] = inv_fact[k - 1] / (double)k;
    inv_odd[0] = 1.0;
    for (int m = 1; m <= BOYS_MAX_M; ++m) inv_odd[m] = 1.0 / (double)(2 * m - 1);
  }
};
const BoysConsts& bc() {
  static BoysConsts c;
  return c;
}

// boys.rs:386-406: non-alternating series for the top order.
double boys_series(int m, double t, double et) {
  double two_t = 2.0 * t;
  double term = 1.0 / (double)(2 * m + 1);
  double sum = term;
  int k = 1;
  for (;;) {
    term *= two_t / (double)(2 * m + 2 * k + 1);
    sum += term;
    if (term <= sum * 1e-17) break;
    k += 1;
    if (k >= 1000) break;
  }
  return et * sum;
}

// boys.rs:411-418
double boys_asymptotic(int m, double t) {
  double val = 0.5 * std::sqrt(PI / t);
  double two_t = 2.0 * t;
  for (int k = 1; k <= m; ++k) val *= (double)(2 * k - 1) / two_t;
  return val;
}
}  // namespace

// boys.rs:362-380
void boys_reference(int m_max, double t, double* out) {
  double et = std::exp(-t);
  out[m_max] = t < asymptotic_boundary(m_max) ? boys_series(m_max, t, et)
                                               : boys_asymptotic(m_max, t);
  for (int m = m_max; m > 0; --m) out[m - 1] = (2.0 * t * out[m] + et) / (double)(2 * m - 1);
}

// boys.rs:122-136: table built once from boys_reference plus libm exp.
const std::vector<double>& boys_table() {
  static std::vector<double> table;
  static std::once_flag once;
  std::call_once(once, [] {
    size_t ngrid = (size_t)(BOYS_TABLE_TMAX / BOYS_H);  // 930
    table.assign((ngrid + 1) * BOYS_ROW, 0.0);
    for (size_t i = 0; i <= ngrid; ++i) {
      double t0 = (double)i * BOYS_H;
      double* row = &table[i * BOYS_ROW];
      boys_reference(BOYS_STRIDE - 1, t0, row);
      row[BOYS_STRIDE] = std::exp(-t0);
    }
  });
  return table;
}

// boys.rs:146-193
void boys_array(int m_max, double t, double* out) {
  if (t < BOYS_TABLE_TMAX && m_max + BOYS_K < BOYS_STRIDE) {
    const std::vector<double>& table = boys_table();
    const BoysConsts& c = bc();
    size_t i = (size_t)std::round(t * (1.0 / BOYS_H));
    double neg_d = (double)i * BOYS_H - t;
    size_t row = i * BOYS_ROW;
    size_t base = row + (size_t)m_max;
    double top = table[base + BOYS_K] * c.inv_fact[BOYS_K];
    for (int k = BOYS_K - 1; k >= 0; --k) top = top * neg_d + table[base + k] * c.inv_fact[k];
    out[m_max] = top;
    if (m_max > 0) {
      double ep = c.inv_fact[BOYS_K];
      for (int k = BOYS_K - 1; k >= 0; --k) ep = ep * neg_d + c.inv_fact[k];
      double et = table[row + BOYS_STRIDE] * ep;
      double two_t = 2.0 * t;
      for (int m = m_max; m > 0; --m) out[m - 1] = (two_t * out[m] + et) * c.inv_odd[m];
    }
  } else {
    boys_reference(m_max, t, out);
  }
}

// ============================================================ Rys quadrature
// src/math/rys.rs

namespace {
constexpr int GL_POINTS = 128;

// rys.rs:409-469: implicit-shift QL on a symmetric tridiagonal matrix,
// accumulating only the first eigenvector row.
void tridiagonal_ql(double* d, double* e, double* z0, int n) {
  if (n <= 1) return;
  const int MAX_ITER = 60;
  const double EPS = 2.220446049250313e-16;
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    for (;;) {
      int m = l;
      while (m < n - 1) {
        double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= EPS * dd) break;
        m += 1;
      }
      if (m == l) break;
      iter += 1;
      if (iter > MAX_ITER) break;
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = std::hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + std::copysign(r, g));
      double s = 1.0, c = 1.0, p = 0.0;
      bool underflow = false;
      int i = m;
      while (i > l) {
        i -= 1;
        double f = s * e[i];
        double b = c * e[i];
        double r2 = std::hypot(f, g);
        e[i + 1] = r2;
        if (r2 == 0.0) {
          d[i + 1] -= p;
          e[m] = 0.0;
          underflow = true;
          break;
        }
        s = f / r2;
        c = g / r2;
        double dd = d[i + 1] - p;
        double r3 = (d[i] - dd) * s + 2.0 * c * b;
        p = s * r3;
        d[i + 1] = dd + p;
        g = c * r3 - b;
        f = z0[i + 1];
        z0[i + 1] = s * z0[i] + c * f;
        z0[i] = c * z0[i] - s * f;
      }
      if (underflow) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
}

// Stable ascending order of indices by value (Rust `sort_by` is stable).
void sort_idx(const double* d, int n, int* idx) {
  for (int i = 0; i < n; ++i) idx[i] = i;
  std::stable_sort(idx, idx + n, [&](int a, int b) { return d[a] < d[b]; });
}

// rys.rs:318-342: cached 128-point Gauss-Legendre rule on [0,1].
struct GLRule {
  double nodes[GL_POINTS];
  double wts[GL_POINTS];
  GLRule() {
    const int n = GL_POINTS;
    double d[GL_POINTS], e[GL_POINTS], z0[GL_POINTS];
    for (int i = 0; i < n; ++i) {
      d[i] = 0.5;
      e[i] = 0.0;
      z0[i] = 0.0;
    }
    z0[0] = 1.0;
    for (int i = 1; i < n; ++i) {
      double l = (double)i;
      double b = 0.25 * l * l / (4.0 * l * l - 1.0);
      e[i - 1] = std::sqrt(b);
    }
    e[n - 1] = 0.0;
    tridiagonal_ql(d, e, z0, n);
    int idx[GL_POINTS];
    sort_idx(d, n, idx);
    for (int o = 0; o < n; ++o) {
      nodes[o] = d[idx[o]];
      wts[o] = z0[idx[o]] * z0[idx[o]];
    }
  }
};
const GLRule& gauss_legendre_01() {
  static GLRule rule;
  return rule;
}

// rys.rs:348-401: Golub-Welsch.
void golub_welsch(const double* alpha, const double* beta, int n, double* roots,
                  double* weights) {
  double mu0 = beta[0];
  if (n == 1) {
    roots[0] = alpha[0];
    weights[0] = mu0;
    return;
  }
  double d[MAX_RYS_ROOTS], e[MAX_RYS_ROOTS], z0[MAX_RYS_ROOTS];
  for (int i = 0; i < n; ++i) {
    d[i] = alpha[i];
    z0[i] = 0.0;
  }
  z0[0] = 1.0;
  for (int i = 1; i < n; ++i) e[i - 1] = std::sqrt(std::max(beta[i], 0.0));
  e[n - 1] = 0.0;
  tridiagonal_ql(d, e, z0, n);
  int idx[MAX_RYS_ROOTS];
  sort_idx(d, n, idx);
  for (int o = 0; o < n; ++o) {
    roots[o] = d[idx[o]];
    weights[o] = mu0 * z0[idx[o]] * z0[idx[o]];
  }
}

// rys.rs:256-310: discretized Stieltjes procedure (f64).
void stieltjes(int n, const double* x, const double* w, double* alpha, double* beta) {
  const int m = GL_POINTS;
  double p_prev[GL_POINTS], p_curr[GL_POINTS], p_next[GL_POINTS];
  auto moments = [&](const double* p, double& norm, double& xnorm) {
    norm = 0.0;
    xnorm = 0.0;
    for (int i = 0; i < m; ++i) {
      double wp = w[i] * p[i] * p[i];
      norm = norm + wp;
      xnorm = xnorm + x[i] * wp;
    }
  };
  for (int i = 0; i < m; ++i) {
    p_prev[i] = 0.0;
    p_curr[i] = 1.0;
  }
  double norm, xnorm;
  moments(p_curr, norm, xnorm);
  beta[0] = norm;
  alpha[0] = xnorm / norm;
  for (int k = 1; k < n; ++k) {
    double a_km1 = alpha[k - 1], b_km1 = beta[k - 1];
    for (int i = 0; i < m; ++i) p_next[i] = (x[i] - a_km1) * p_curr[i] - b_km1 * p_prev[i];
    double nn, xn;
    moments(p_next, nn, xn);
    alpha[k] = xn / nn;
    beta[k] = nn / norm;
    norm = nn;
    for (int i = 0; i < m; ++i) {
      p_prev[i] = p_curr[i];
      p_curr[i] = p_next[i];
    }
  }
}

// rys.rs:232-252
void finite_branch(int n, double t, double* roots, double* weights) {
  const GLRule& gl = gauss_legendre_01();
  double x[GL_POINTS], w[GL_POINTS];
  for (int m = 0; m < GL_POINTS; ++m) {
    double u = gl.nodes[m];
    double xm = u * u;
    x[m] = xm;
    w[m] = gl.wts[m] * std::exp(-t * xm);
  }
  double alpha[MAX_RYS_ROOTS] = {0}, beta[MAX_RYS_ROOTS] = {0};
  stieltjes(n, x, w, alpha, beta);
  golub_welsch(alpha, beta, n, roots, weights);
}

// rys.rs:540-571: T-independent generalized Gauss-Laguerre(-1/2) nodes.
struct LaguerreCache {
  double xi[MAX_RYS_ROOTS][MAX_RYS_ROOTS];
  double om[MAX_RYS_ROOTS][MAX_RYS_ROOTS];
  LaguerreCache() {
    for (int m = 1; m <= MAX_RYS_ROOTS; ++m) {
      double alpha_param = -0.5;
      double a[MAX_RYS_ROOTS] = {0}, b[MAX_RYS_ROOTS] = {0};
      for (int k = 0; k < m; ++k) {
        double kf = (double)k;
        a[k] = 2.0 * kf + alpha_param + 1.0;
        b[k] = kf * (kf + alpha_param);
      }
      b[0] = std::sqrt(PI);
      golub_welsch(a, b, m, xi[m - 1], om[m - 1]);
    }
  }
};
const LaguerreCache& laguerre() {
  static LaguerreCache c;
  return c;
}

// rys.rs:524-533
void laguerre_half_branch(int n, double t, double* roots, double* weights) {
  const LaguerreCache& c = laguerre();
  double inv_t = 1.0 / t;
  double scale = 0.5 / std::sqrt(t);
  for (int i = 0; i < n; ++i) {
    roots[i] = c.xi[n - 1][i] * inv_t;
    weights[i] = c.om[n - 1][i] * scale;
  }
}

// rys.rs:218-229 (and the identical Clenshaw in gen_rys_tables.rs)
double chebev(const double* c, double xi) {
  double two_xi = 2.0 * xi;
  double d = 0.0, dd = 0.0;
  for (int k = RYS_NC - 1; k >= 1; --k) {
    double sv = d;
    d = two_xi * d - dd + c[k];
    dd = sv;
  }
  return xi * d - dd + 0.5 * c[0];
}

// gen_rys_tables.rs:164-193 (NR chebft at the 17 Chebyshev nodes).
void fit_cell(int n, double a, double b, std::vector<double>& rs, std::vector<double>& ws) {
  const int NC = RYS_NC;
  double bma = 0.5 * (b - a);
  double bpa = 0.5 * (b + a);
  double node_r[NC][MAX_RYS_ROOTS], node_w[NC][MAX_RYS_ROOTS];
  double r[MAX_RYS_ROOTS], w[MAX_RYS_ROOTS];
  for (int j = 0; j < NC; ++j) {
    double y = std::cos((PI * ((double)j + 0.5)) / (double)NC);
    double t = y * bma + bpa;
    rys_finite_reference(n, t, r, w);
    for (int i = 0; i < n; ++i) {
      node_r[j][i] = r[i];
      node_w[j][i] = w[i];
    }
  }
  rs.assign((size_t)n * NC, 0.0);
  ws.assign((size_t)n * NC, 0.0);
  double fac = 2.0 / (double)NC;
  for (int k = 0; k < NC; ++k) {
    for (int j = 0; j < NC; ++j) {
      double cos_kj = std::cos((PI * (double)k * ((double)j + 0.5)) / (double)NC);
      for (int i = 0; i < n; ++i) {
        rs[(size_t)i * NC + k] += fac * node_r[j][i] * cos_kj;
        ws[(size_t)i * NC + k] += fac * node_w[j][i] * cos_kj;
      }
    }
  }
}

// gen_rys_tables.rs:136-161
double max_error(int n, double t_hi, int n_sub) {
  const int CHECK_PER_CELL = 33;
  double width = t_hi / (double)n_sub;
  double worst = 0.0;
  double rr[MAX_RYS_ROOTS], rw[MAX_RYS_ROOTS];
  std::vector<double> rc, wc;
  for (int s = 0; s < n_sub; ++s) {
    double a = (double)s * width;
    double b = a + width;
    fit_cell(n, a, b, rc, wc);
    for (int j = 0; j < CHECK_PER_CELL; ++j) {
      double frac = (double)j / (double)(CHECK_PER_CELL - 1);
      double t = a + frac * (b - a);
      rys_finite_reference(n, t, rr, rw);
      double xi = (2.0 * t - (a + b)) / (b - a);
      for (int i = 0; i < n; ++i) {
        worst = std::max(worst, std::fabs(chebev(&rc[(size_t)i * RYS_NC], xi) - rr[i]));
        worst = std::max(worst, std::fabs(chebev(&wc[(size_t)i * RYS_NC], xi) - rw[i]));
      }
    }
  }
  return worst;
}
}  // namespace

void rys_finite_reference(int n, double t, double* roots, double* weights) {
  finite_branch(n, t, roots, weights);
}

// gen_rys_tables.rs:44-92, 124-133: the adaptive n_sub search and the fits.
const std::vector<RysTable>& rys_tables_regenerated() {
  static std::vector<RysTable> tables;
  static std::once_flag once;
  std::call_once(once, [] {
    const double FIT_TOL = 2e-14;
    const int MAX_SUB = 256;
    tables.resize(MAX_RYS_ROOTS);
    for (int n = 1; n <= MAX_RYS_ROOTS; ++n) {
      double t_hi = asymptotic_boundary(2 * n - 1);
      int n_sub = 1;
      double worst;
      for (;;) {
        worst = max_error(n, t_hi, n_sub);
        if (worst <= FIT_TOL || n_sub >= MAX_SUB) break;
        n_sub += 1;
      }
      RysTable& tb = tables[n - 1];
      tb.n = n;
      tb.n_sub = n_sub;
      tb.worst = worst;
      double width = t_hi / (double)n_sub;
      std::vector<double> rc, wc;
      for (int s = 0; s < n_sub; ++s) {
        double a = (double)s * width;
        double b = a + width;
        fit_cell(n, a, b, rc, wc);
        tb.root.insert(tb.root.end(), rc.begin(), rc.end());
        tb.weight.insert(tb.weight.end(), wc.begin(), wc.end());
      }
    }
  });
  return tables;
}

#ifdef ORACLE_HAVE_REF_TABLES
#include "_ref/rys_tables.inc"
bool rys_tables_are_reference_literals() { return true; }
// The literal coefficients the reference interpolates at run time
// (src/math/rys_tables.rs), extracted at build time.
const std::vector<RysTable>& rys_tables() {
  static std::vector<RysTable> tables;
  static std::once_flag once;
  std::call_once(once, [] {
    tables.resize(MAX_RYS_ROOTS);
    for (int n = 1; n <= MAX_RYS_ROOTS; ++n) {
      RysTable& tb = tables[n - 1];
      tb.n = n;
      tb.n_sub = REF_NSUB[n - 1];
      size_t len = (size_t)tb.n_sub * n * RYS_NC;
      tb.root.assign(REF_ROOT[n - 1], REF_ROOT[n - 1] + len);
      tb.weight.assign(REF_WEIGHT[n - 1], REF_WEIGHT[n - 1] + len);
    }
  });
  return tables;
}
#else
bool rys_tables_are_reference_literals() { return false; }
const std::vector<RysTable>& rys_tables() { return rys_tables_regenerated(); }
#endif

// rys.rs:174-186, 193-215
void rys_roots_weights(int n, double t, double* roots, double* weights) {
  if (t >= asymptotic_boundary(2 * n - 1)) {
    laguerre_half_branch(n, t, roots, weights);
    return;
  }
  const RysTable& tb = rys_tables()[n - 1];
  double t_hi = asymptotic_boundary(2 * n - 1);
  int n_sub = tb.n_sub;
  double width = t_hi / (double)n_sub;
  size_t s = (size_t)(t / width);
  if (s >= (size_t)n_sub) s = (size_t)n_sub - 1;
  double a = (double)s * width;
  double b = a + width;
  double xi = (2.0 * t - (a + b)) / (b - a);
  size_t base = s * (size_t)n;
  for (int i = 0; i < n; ++i) {
    roots[i] = chebev(&tb.root[(base + i) * RYS_NC], xi);
    weights[i] = chebev(&tb.weight[(base + i) * RYS_NC], xi);
  }
}

// ============================================================ c2s
// src/math/solid_harmonics.rs

namespace {
double factorial(int n) {
  double acc = 1.0;
  for (int k = 1; k <= n; ++k) acc *= (double)k;
  return acc;
}
double binom(long n, long k) {
  if (k < 0 || k > n || n < 0) return 0.0;
  return factorial((int)n) / (factorial((int)k) * factorial((int)(n - k)));
}
double cos_half_pi(long n) {
  long r = ((n % 4) + 4) % 4;
  return r == 0 ? 1.0 : (r == 2 ? -1.0 : 0.0);
}
double sin_half_pi(long n) {
  long r = ((n % 4) + 4) % 4;
  return r == 1 ? 1.0 : (r == 3 ? -1.0 : 0.0);
}

// solid_harmonics.rs:87-147
double racah_coeff(int l, long m, int lx, int ly, int lz) {
  int big_m = (int)(m < 0 ? -m : m);
  if (big_m > l) return 0.0;
  bool cosine = m >= 0;
  double norm = big_m == 0 ? std::sqrt(factorial(l - big_m) / factorial(l + big_m))
                           : std::sqrt(2.0 * factorial(l - big_m) / factorial(l + big_m));
  double acc = 0.0;
  int kmax = (l - big_m) / 2;
  for (int k = 0; k <= kmax; ++k) {
    int zpow = l - 2 * k - big_m;
    double gamma = (k % 2 == 0 ? 1.0 : -1.0) * powi(2.0, -l) * binom(l, k) *
                   binom(2L * l - 2L * k, l) * factorial(l - 2 * k) /
                   factorial(l - 2 * k - big_m);
    if (gamma == 0.0) continue;
    for (int a = 0; a <= k; ++a)
      for (int b = 0; b <= k - a; ++b) {
        int c = k - a - b;
        for (int p = 0; p <= big_m; ++p) {
          int q = big_m - p;
          int tx = 2 * a + p, ty = 2 * b + q, tz = 2 * c + zpow;
          if (tx != lx || ty != ly || tz != lz) continue;
          double trig = cosine ? cos_half_pi(q) : sin_half_pi(q);
          if (trig == 0.0) continue;
          double multinomial = factorial(k) / (factorial(a) * factorial(b) * factorial(c));
          acc += gamma * multinomial * binom(big_m, p) * trig;
        }
      }
  }
  return norm * acc;
}

std::vector<long> m_order(int l) {
  if (l == 1) return {1, -1, 0};
  std::vector<long> v;
  for (long m = -l; m <= l; ++m) v.push_back(m);
  return v;
}

// solid_harmonics.rs:175-200
double gaussian_moment_1d(int n, double beta) {
  if (n % 2 == 1) return 0.0;
  double dfac = double_factorial((long)n - 1);
  return dfac / powi(2.0 * beta, n / 2) * std::sqrt(PI / beta);
}
double raw_self_overlap(int l, const Tri& ci, const Tri& cj) {
  double beta = 2.0;
  double bare = gaussian_moment_1d(ci[0] + cj[0], beta) * gaussian_moment_1d(ci[1] + cj[1], beta) *
                gaussian_moment_1d(ci[2] + cj[2], beta);
  double n_mono = cart_norm(1.0, l, 0, 0);
  double raw_shell = powi(monomial_to_raw_factor(l), 2);
  return raw_shell * n_mono * n_mono * bare;
}
}  // namespace

double monomial_to_raw_factor(int l) {
  if (l < 2) return 1.0;
  return std::sqrt(4.0 * PI / (double)(2 * l + 1));
}

// solid_harmonics.rs:218-247
std::vector<double> c2s_matrix(int l) {
  std::vector<Tri> comps = cart_components(l);
  int ncart = n_cart(l);
  std::vector<long> ms = m_order(l);
  std::vector<double> mat(ms.size() * (size_t)ncart, 0.0);
  for (size_t row = 0; row < ms.size(); ++row) {
    long m = ms[row];
    std::vector<double> coeffs(ncart, 0.0);
    for (int i = 0; i < ncart; ++i) coeffs[i] = racah_coeff(l, m, comps[i][0], comps[i][1], comps[i][2]);
    double q = 0.0;
    for (int i = 0; i < ncart; ++i) {
      if (coeffs[i] == 0.0) continue;
      for (int j = 0; j < ncart; ++j) {
        if (coeffs[j] == 0.0) continue;
        q += coeffs[i] * coeffs[j] * raw_self_overlap(l, comps[i], comps[j]);
      }
    }
    double kappa = 1.0 / std::sqrt(q);
    for (int i = 0; i < ncart; ++i) mat[row * ncart + i] = kappa * coeffs[i];
  }
  return mat;
}

}  // namespace oracle
