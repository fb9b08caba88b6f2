// Host-side math of the plan: primitive normalisation, the Cartesian ->
// real-solid-harmonic matrices, and the Rys Chebyshev tables the device
// interpolates.  These are plan-construction steps (the reference also builds
// its tables lazily at first use, src/math/boys.rs:122-136); no quartet is
// evaluated here.
#include "host_math.hpp"

#include <algorithm>
#include <cmath>
#include <mutex>

namespace igpu {

static const double PI = 3.14159265358979323846;

// Square-and-multiply integer power (the lowering of Rust's f64::powi).
double ipow(double a, int b) {
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

static double dfact(long n) {
  double acc = 1.0;
  for (long k = n; k > 1; k -= 2) acc *= (double)k;
  return acc;
}

// N(alpha; l,0,0) = (2 alpha/pi)^{3/4} sqrt((4 alpha)^l) / sqrt((2l-1)!!)
// (src/math/norm.rs:42-49).
double shell_norm(double alpha, int l) {
  return std::pow(2.0 * alpha / PI, 0.75) * std::sqrt(ipow(4.0 * alpha, l)) / std::sqrt(dfact(2L * l - 1));
}

double effective_coeff(double alpha, double coef, int l) {
  if (alpha == 0.0) return coef;  // src/shell.rs:182-187
  return coef * shell_norm(alpha, l);
}

// ----------------------------------------------------------------- c2s

static double fact(int n) {
  double a = 1.0;
  for (int k = 1; k <= n; ++k) a *= (double)k;
  return a;
}
static double choose(long n, long k) {
  if (k < 0 || k > n || n < 0) return 0.0;
  return fact((int)n) / (fact((int)k) * fact((int)(n - k)));
}

// Racah-normalised real solid harmonic C_l^m (m >= 0) / S_l^|m| (m < 0)
// coefficient of the monomial x^lx y^ly z^lz (Schlegel & Frisch 1995).
static double solid_harmonic_coeff(int l, int m, int lx, int ly, int lz) {
  const int M = m < 0 ? -m : m;
  if (M > l) return 0.0;
  const double norm = M == 0 ? std::sqrt(fact(l) / fact(l)) : std::sqrt(2.0 * fact(l - M) / fact(l + M));
  double acc = 0.0;
  for (int k = 0; k <= (l - M) / 2; ++k) {
    const int zpow = l - 2 * k - M;
    const double gamma = (k % 2 == 0 ? 1.0 : -1.0) * ipow(2.0, -l) * choose(l, k) * choose(2L * l - 2L * k, l) *
                         fact(l - 2 * k) / fact(l - 2 * k - M);
    if (gamma == 0.0) continue;
    for (int a = 0; a <= k; ++a)
      for (int b = 0; b <= k - a; ++b) {
        const int c = k - a - b;
        for (int p = 0; p <= M; ++p) {
          const int q = M - p;
          if (2 * a + p != lx || 2 * b + q != ly || 2 * c + zpow != lz) continue;
          const int r = q % 4;
          const double trig = m >= 0 ? (r == 0 ? 1.0 : (r == 2 ? -1.0 : 0.0)) : (r == 1 ? 1.0 : (r == 3 ? -1.0 : 0.0));
          if (trig == 0.0) continue;
          acc += gamma * (fact(k) / (fact(a) * fact(b) * fact(c))) * choose(M, p) * trig;
        }
      }
  }
  return norm * acc;
}

std::vector<std::array<int, 3>> cart_comps(int l) {
  std::vector<std::array<int, 3>> v;
  for (int lx = l; lx >= 0; --lx)
    for (int ly = l - lx; ly >= 0; --ly) v.push_back({lx, ly, l - lx - ly});
  return v;
}

static double gauss_moment(int n, double beta) {
  if (n % 2 == 1) return 0.0;
  return dfact((long)n - 1) / ipow(2.0 * beta, n / 2) * std::sqrt(PI / beta);
}

double monomial_to_raw(int l) { return l < 2 ? 1.0 : std::sqrt(4.0 * PI / (double)(2 * l + 1)); }

// Effective per-index transform M = monomial_to_raw(l) * C(l), (2l+1) x
// n_cart, rows in m order (+1,-1,0) for p, ascending m otherwise, each row
// unit-normalised against the raw Cartesian overlap (src/spherical.rs:37-48,
// src/math/solid_harmonics.rs:218-247).
std::vector<double> c2s_effective(int l) {
  auto comps = cart_comps(l);
  const int nc = (int)comps.size();
  std::vector<int> ms;
  if (l == 1)
    ms = {1, -1, 0};
  else
    for (int m = -l; m <= l; ++m) ms.push_back(m);
  const double ratio = monomial_to_raw(l);
  const double nmono = shell_norm(1.0, l);
  std::vector<double> out(ms.size() * nc, 0.0);
  for (size_t row = 0; row < ms.size(); ++row) {
    std::vector<double> co(nc);
    for (int i = 0; i < nc; ++i) co[i] = solid_harmonic_coeff(l, ms[row], comps[i][0], comps[i][1], comps[i][2]);
    double q = 0.0;
    for (int i = 0; i < nc; ++i) {
      if (co[i] == 0.0) continue;
      for (int j = 0; j < nc; ++j) {
        if (co[j] == 0.0) continue;
        const double bare = gauss_moment(comps[i][0] + comps[j][0], 2.0) * gauss_moment(comps[i][1] + comps[j][1], 2.0) *
                            gauss_moment(comps[i][2] + comps[j][2], 2.0);
        q += co[i] * co[j] * (ipow(ratio, 2) * nmono * nmono * bare);
      }
    }
    const double kappa = 1.0 / std::sqrt(q);
    for (int i = 0; i < nc; ++i) out[row * nc + i] = ratio * (kappa * co[i]);
  }
  return out;
}

// ------------------------------------------------------------ Rys tables
//
// Gauss quadrature for d mu(x) = x^{-1/2} exp(-T x) dx / 2 on [0,1] by the
// discretised Stieltjes procedure on a 128-point Gauss-Legendre rule in
// u = sqrt(x) plus Golub-Welsch, fitted per T-subinterval by degree-16
// Chebyshev series (the method of src/math/rys.rs:230-515 and
// xtask/src/gen_rys_tables.rs); above asymptotic_boundary(2n-1) the
// generalized Gauss-Laguerre(-1/2) nodes scaled by 1/T.

namespace {
const int GLN = 128;

void ql_first_row(double* d, double* e, double* z, int n) {
  if (n <= 1) return;
  const double EPS = 2.220446049250313e-16;
  for (int l = 0; l < n; ++l) {
    for (int iter = 0;; ++iter) {
      int m = l;
      for (; m < n - 1; ++m)
        if (std::fabs(e[m]) <= EPS * (std::fabs(d[m]) + std::fabs(d[m + 1]))) break;
      if (m == l || iter >= 60) break;
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = std::hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + std::copysign(r, g));
      double s = 1.0, c = 1.0, p = 0.0;
      bool under = false;
      for (int i = m - 1; i >= l; --i) {
        double f = s * e[i], b = c * e[i];
        r = std::hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {
          d[i + 1] -= p;
          e[m] = 0.0;
          under = true;
          break;
        }
        s = f / r;
        c = g / r;
        double dd = d[i + 1] - p;
        double t = (d[i] - dd) * s + 2.0 * c * b;
        p = s * t;
        d[i + 1] = dd + p;
        g = c * t - b;
        f = z[i + 1];
        z[i + 1] = s * z[i] + c * f;
        z[i] = c * z[i] - s * f;
      }
      if (under) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
}

void gauss_from_jacobi(const double* a, const double* b, int n, double* x, double* w) {
  if (n == 1) {
    x[0] = a[0];
    w[0] = b[0];
    return;
  }
  double d[MAX_ROOTS], e[MAX_ROOTS], z[MAX_ROOTS];
  for (int i = 0; i < n; ++i) {
    d[i] = a[i];
    z[i] = i == 0 ? 1.0 : 0.0;
  }
  for (int i = 1; i < n; ++i) e[i - 1] = std::sqrt(std::max(b[i], 0.0));
  e[n - 1] = 0.0;
  ql_first_row(d, e, z, n);
  int idx[MAX_ROOTS];
  for (int i = 0; i < n; ++i) idx[i] = i;
  std::stable_sort(idx, idx + n, [&](int p, int q) { return d[p] < d[q]; });
  for (int o = 0; o < n; ++o) {
    x[o] = d[idx[o]];
    w[o] = b[0] * z[idx[o]] * z[idx[o]];
  }
}

struct GL {
  double u[GLN], w[GLN];
  GL() {
    double d[GLN], e[GLN], z[GLN];
    for (int i = 0; i < GLN; ++i) {
      d[i] = 0.5;
      e[i] = 0.0;
      z[i] = i == 0 ? 1.0 : 0.0;
    }
    for (int i = 1; i < GLN; ++i) {
      const double l = (double)i;
      e[i - 1] = std::sqrt(0.25 * l * l / (4.0 * l * l - 1.0));
    }
    ql_first_row(d, e, z, GLN);
    int idx[GLN];
    for (int i = 0; i < GLN; ++i) idx[i] = i;
    std::stable_sort(idx, idx + GLN, [&](int p, int q) { return d[p] < d[q]; });
    for (int o = 0; o < GLN; ++o) {
      u[o] = d[idx[o]];
      w[o] = z[idx[o]] * z[idx[o]];
    }
  }
};

void finite_quadrature(const GL& gl, int n, double T, double* x, double* w) {
  double X[GLN], W[GLN], p0[GLN], p1[GLN], p2[GLN];
  for (int m = 0; m < GLN; ++m) {
    X[m] = gl.u[m] * gl.u[m];
    W[m] = gl.w[m] * std::exp(-T * X[m]);
    p0[m] = 0.0;
    p1[m] = 1.0;
  }
  double al[MAX_ROOTS] = {0}, be[MAX_ROOTS] = {0};
  double nrm = 0.0, xn = 0.0;
  for (int m = 0; m < GLN; ++m) {
    const double wp = W[m] * p1[m] * p1[m];
    nrm += wp;
    xn += X[m] * wp;
  }
  be[0] = nrm;
  al[0] = xn / nrm;
  for (int k = 1; k < n; ++k) {
    double nn = 0.0, xx = 0.0;
    for (int m = 0; m < GLN; ++m) {
      p2[m] = (X[m] - al[k - 1]) * p1[m] - be[k - 1] * p0[m];
      const double wp = W[m] * p2[m] * p2[m];
      nn += wp;
      xx += X[m] * wp;
    }
    al[k] = xx / nn;
    be[k] = nn / nrm;
    nrm = nn;
    for (int m = 0; m < GLN; ++m) {
      p0[m] = p1[m];
      p1[m] = p2[m];
    }
  }
  gauss_from_jacobi(al, be, n, x, w);
}

double clenshaw(const double* c, double xi) {
  double d = 0.0, dd = 0.0;
  for (int k = RYS_NC - 1; k >= 1; --k) {
    const double sv = d;
    d = 2.0 * xi * d - dd + c[k];
    dd = sv;
  }
  return xi * d - dd + 0.5 * c[0];
}

// degree-16 Chebyshev fits of the n roots and n weights on [a, b]:
// out[(i*2 + {0,1}) * 17 + k]
void fit(const GL& gl, int n, double a, double b, double* out) {
  const int NC = RYS_NC;
  double vx[RYS_NC][MAX_ROOTS], vw[RYS_NC][MAX_ROOTS];
  for (int j = 0; j < NC; ++j) {
    const double y = std::cos(PI * ((double)j + 0.5) / (double)NC);
    finite_quadrature(gl, n, y * 0.5 * (b - a) + 0.5 * (b + a), vx[j], vw[j]);
  }
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < NC; ++k) {
      double sx = 0.0, sw = 0.0;
      for (int j = 0; j < NC; ++j) {
        const double ck = std::cos(PI * (double)k * ((double)j + 0.5) / (double)NC);
        sx += vx[j][i] * ck;
        sw += vw[j][i] * ck;
      }
      out[(i * 2 + 0) * NC + k] = 2.0 / NC * sx;
      out[(i * 2 + 1) * NC + k] = 2.0 / NC * sw;
    }
}
}  // namespace

const RysTables& rys_tables() {
  static RysTables T;
  static std::once_flag once;
  std::call_once(once, [] {
    GL gl;
    T.meta.assign(MAX_ROOTS + 1, RysMeta{0, 0, 0.0, 0.0});
    std::vector<double> cell((size_t)MAX_ROOTS * 2 * RYS_NC);
    for (int n = 1; n <= MAX_ROOTS; ++n) {
      const double t_hi = 33.0 + 2.5 * (double)(2 * n - 1);
      // smallest equal-width subdivision whose fits stay within 2e-14
      int n_sub = 1;
      for (;; ++n_sub) {
        const double width = t_hi / n_sub;
        double worst = 0.0;
        for (int s = 0; s < n_sub && worst <= 2e-14; ++s) {
          const double a = s * width, b = a + width;
          fit(gl, n, a, b, cell.data());
          for (int j = 0; j < 33; ++j) {
            const double t = a + (double)j / 32.0 * (b - a);
            double rx[MAX_ROOTS], rw[MAX_ROOTS];
            finite_quadrature(gl, n, t, rx, rw);
            const double xi = (2.0 * t - (a + b)) / (b - a);
            for (int i = 0; i < n; ++i) {
              worst = std::max(worst, std::fabs(clenshaw(&cell[(i * 2) * RYS_NC], xi) - rx[i]));
              worst = std::max(worst, std::fabs(clenshaw(&cell[(i * 2 + 1) * RYS_NC], xi) - rw[i]));
            }
          }
        }
        if (worst <= 2e-14 || n_sub >= 256) break;
      }
      RysMeta m;
      m.n_sub = n_sub;
      m.off = (int)T.coef.size();
      m.width = t_hi / n_sub;
      m.t_hi = t_hi;
      T.meta[n] = m;
      for (int s = 0; s < n_sub; ++s) {
        fit(gl, n, s * m.width, s * m.width + m.width, cell.data());
        T.coef.insert(T.coef.end(), cell.begin(), cell.begin() + (size_t)n * 2 * RYS_NC);
      }
      // generalized Gauss-Laguerre(-1/2): a_k = 2k + 1/2, b_k = k(k - 1/2), b_0 = sqrt(pi)
      double a[MAX_ROOTS], b[MAX_ROOTS];
      for (int k = 0; k < n; ++k) {
        a[k] = 2.0 * k + 0.5;
        b[k] = k * (k - 0.5);
      }
      b[0] = std::sqrt(PI);
      gauss_from_jacobi(a, b, n, &T.lag_x[(n - 1) * MAX_ROOTS], &T.lag_w[(n - 1) * MAX_ROOTS]);
    }
  });
  return T;
}

}  // namespace igpu
