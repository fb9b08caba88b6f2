// ORACLE — test infrastructure only (see oracle.hpp).
// Flat C entry points so the Python tests and the CPU-baseline leg of
// bench.py can drive the restatement through ctypes.
#include <cstring>
#include <exception>
#include <string>

#include "direct.hpp"
#include "oracle.hpp"

using namespace oracle;

namespace {
thread_local std::string g_err;
std::vector<int> bra_list(const int* bras, int nbras, int npairs) {
  std::vector<int> v;
  if (nbras < 0) {
    for (int b = 0; b < npairs; ++b) v.push_back(b);
  } else {
    v.assign(bras, bras + nbras);
  }
  return v;
}
struct GradHandle {
  GradPlan plan;
  GradHandle(const Basis& b, Engine e) : plan(b, e) {}
};
}  // namespace

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

void* orc_basis_new(int nsh, const int* l, const int* spherical, const double* centers,
                    const int* nprim, const double* exps, const double* coefs) {
  try {
    std::vector<Shell> shells;
    int off = 0;
    for (int s = 0; s < nsh; ++s) {
      Shell sh;
      sh.l = l[s];
      sh.spherical = spherical[s] != 0;
      sh.center = {centers[3 * s], centers[3 * s + 1], centers[3 * s + 2]};
      sh.exps.assign(exps + off, exps + off + nprim[s]);
      sh.coefs.assign(coefs + off, coefs + off + nprim[s]);
      off += nprim[s];
      shells.push_back(sh);
    }
    return new Basis(std::move(shells));
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}
void orc_basis_free(void* b) { delete static_cast<Basis*>(b); }
int orc_nao(void* b) { return static_cast<Basis*>(b)->nao(); }
int orc_natom(void* b) { return (int)static_cast<Basis*>(b)->atoms().size(); }

void orc_set_erf_omega(double omega) { set_rys_erf_omega(omega); }

void orc_eri(void* b, int engine, double* out) {
  std::vector<double> e = static_cast<Basis*>(b)->eri((Engine)engine);
  std::memcpy(out, e.data(), e.size() * sizeof(double));
}
void orc_eri_block(void* b, int engine, int i, int j, int k, int l, double* out) {
  std::vector<double> e = static_cast<Basis*>(b)->eri_block((Engine)engine, i, j, k, l);
  std::memcpy(out, e.data(), e.size() * sizeof(double));
}
void orc_schwarz(void* b, int engine, double* q) {
  std::vector<double> e = static_cast<Basis*>(b)->schwarz((Engine)engine);
  std::memcpy(q, e.data(), e.size() * sizeof(double));
}

void* orc_direct_new(void* b, int engine) {
  return new DirectPlan(*static_cast<Basis*>(b), (Engine)engine);
}
void orc_direct_free(void* p) { delete static_cast<DirectPlan*>(p); }
void orc_direct_schwarz(void* p, double* q) {
  auto* dp = static_cast<DirectPlan*>(p);
  std::memcpy(q, dp->schwarz.data(), dp->schwarz.size() * sizeof(double));
}
void orc_density_bounds(void* p, const double* d, double* bounds) {
  std::vector<double> b = static_cast<DirectPlan*>(p)->density_bounds(d);
  std::memcpy(bounds, b.data(), b.size() * sizeof(double));
}

// J/K over the given canonical bra-pair indices (nbras < 0: all), D/J/K are
// ndens consecutive nao x nao matrices.  J/K accumulate (+=).
int orc_direct_jk(void* p, int ndens, const double* D, double thr, int want_k, const int* bras,
                  int nbras, int nthreads, double* J, double* K, uint64_t* count, uint64_t* hash,
                  int count_only) {
  try {
    auto* dp = static_cast<DirectPlan*>(p);
    size_t n2 = (size_t)dp->basis.nao() * dp->basis.nao();
    std::vector<std::vector<double>> bounds(ndens);
    JKArgs a;
    a.ndens = ndens;
    a.threshold = thr;
    a.want_k = want_k != 0;
    a.count_only = count_only != 0;
    for (int d = 0; d < ndens; ++d) {
      a.D[d] = D + d * n2;
      bounds[d] = dp->density_bounds(a.D[d]);
      a.bounds[d] = bounds[d].data();
      a.J[d] = J ? J + d * n2 : nullptr;
      a.K[d] = (K && want_k) ? K + d * n2 : nullptr;
    }
    QuartetSink sink;
    run_jk(*dp, a, bra_list(bras, nbras, (int)dp->pairs.size()), nthreads, &sink);
    if (count) *count = sink.count;
    if (hash) *hash = sink.hash;
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// Explicit screened quartet list (small systems): returns the count, writes
// up to `cap` quartets (4 ints each) and their masks.
long orc_jk_quartets(void* p, int ndens, const double* D, double thr, const int* bras, int nbras,
                     int* out4, uint64_t* masks, long cap) {
  auto* dp = static_cast<DirectPlan*>(p);
  size_t n2 = (size_t)dp->basis.nao() * dp->basis.nao();
  std::vector<std::vector<double>> bounds(ndens);
  JKArgs a;
  a.ndens = ndens;
  a.threshold = thr;
  a.count_only = true;
  for (int d = 0; d < ndens; ++d) {
    a.D[d] = D + d * n2;
    bounds[d] = dp->density_bounds(a.D[d]);
    a.bounds[d] = bounds[d].data();
  }
  std::vector<std::array<int, 4>> list;
  std::vector<uint64_t> mk;
  QuartetSink sink;
  sink.list = &list;
  sink.masks = &mk;
  run_jk(*dp, a, bra_list(bras, nbras, (int)dp->pairs.size()), 1, &sink);
  for (long q = 0; q < (long)list.size() && q < cap; ++q) {
    for (int c = 0; c < 4; ++c) out4[4 * q + c] = list[q][c];
    masks[q] = mk[q];
  }
  return (long)list.size();
}

void* orc_grad_new(void* b, int engine) {
  try {
    return new GradHandle(*static_cast<Basis*>(b), (Engine)engine);
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}
void orc_grad_free(void* g) { delete static_cast<GradHandle*>(g); }

// Gradient dE/dR over the given bra pairs; out is natom x 3 and accumulates.
int orc_direct_grad(void* g, int ncoul, const double* cf, const double* cl, const double* cr,
                    int nexch, const double* xf, const double* xl, const double* xr, double thr,
                    const int* bras, int nbras, int nthreads, double* out, uint64_t* count,
                    uint64_t* hash, int count_only) {
  try {
    auto* gh = static_cast<GradHandle*>(g);
    size_t n2 = (size_t)gh->plan.basis.nao() * gh->plan.basis.nao();
    std::vector<GradTerm> ct, xt;
    for (int t = 0; t < ncoul; ++t) ct.push_back({cf[t], cl + t * n2, cr + t * n2});
    for (int t = 0; t < nexch; ++t) xt.push_back({xf[t], xl + t * n2, xr + t * n2});
    GradDensity dens = gh->plan.density(ct, xt);
    QuartetSink sink;
    int nsh = gh->plan.basis.nsh();
    run_grad(gh->plan, dens, thr, bra_list(bras, nbras, nsh * (nsh + 1) / 2), nthreads, out,
             &sink, count_only != 0);
    if (count) *count = sink.count;
    if (hash) *hash = sink.hash;
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// Dense-gamma gradient (Basis::eri_grad_contract_with); out is natom x 3
// and accumulates.
int orc_eri_grad_contract(void* g, const double* gamma, double* out) {
  try {
    static_cast<GradHandle*>(g)->plan.dense_contract(gamma, out);
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

void orc_boys(int m, double t, double* out) { boys_array(m, t, out); }
void orc_boys_reference(int m, double t, double* out) { boys_reference(m, t, out); }
void orc_rys(int n, double t, double* r, double* w) { rys_roots_weights(n, t, r, w); }
void orc_rys_finite_reference(int n, double t, double* r, double* w) {
  rys_finite_reference(n, t, r, w);
}
int orc_rys_tables_are_reference_literals() { return rys_tables_are_reference_literals() ? 1 : 0; }
int orc_rys_table_nsub(int n, double* worst) {
  const RysTable& tb = rys_tables_regenerated()[n - 1];
  if (worst) *worst = tb.worst;
  return tb.n_sub;
}
void orc_rys_table_copy(int n, int regenerated, double* root, double* weight) {
  const RysTable& tb = (regenerated ? rys_tables_regenerated() : rys_tables())[n - 1];
  std::memcpy(root, tb.root.data(), tb.root.size() * sizeof(double));
  std::memcpy(weight, tb.weight.data(), tb.weight.size() * sizeof(double));
}
void orc_c2s(int l, double* out) {
  std::vector<double> m = c2s_matrix(l);
  std::memcpy(out, m.data(), m.size() * sizeof(double));
}
double orc_cart_norm(double a, int lx, int ly, int lz) { return cart_norm(a, lx, ly, lz); }
void orc_select_engine(int ne, int nf, int deg, int* out) { *out = (int)select_engine(ne, nf, deg); }

}  // extern "C"
