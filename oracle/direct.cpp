// ORACLE — test infrastructure only (see oracle.hpp).
// Integral-direct J/K (src/direct.rs) and the density-direct ERI gradient
// (src/direct_grad.rs), plus the screened-quartet fingerprint used to check
// that the product screens exactly the same canonical quartets.
#include "direct.hpp"

#include <algorithm>
#include <cmath>
#include <map>
#include <stdexcept>
#include <thread>
#include <tuple>

namespace oracle {

uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

uint64_t quartet_key(int i, int j, int k, int l, uint64_t mask) {
  uint64_t id = ((((uint64_t)i * 65536u + (uint64_t)j) * 65536u + (uint64_t)k) * 65536u) +
                (uint64_t)l;
  return splitmix64(id ^ splitmix64(mask + 0x5851F42D4C957F2Dull));
}

// ------------------------------------------------------------------ J/K

DirectPlan::DirectPlan(const Basis& b, Engine e) : basis(b), engine(e) {
  schwarz = b.schwarz(Engine::Auto);  // direct.rs:85: basis.schwarz_bounds()
  for (int i = 0; i < b.nsh(); ++i)
    for (int j = 0; j <= i; ++j) pairs.push_back({i, j});
}

// direct.rs:103-125
std::vector<double> DirectPlan::density_bounds(const double* d) const {
  int nsh = basis.nsh(), nao = basis.nao();
  const auto& offs = basis.offsets();
  std::vector<double> bounds((size_t)nsh * nsh, 0.0);
  for (int i = 0; i < nsh; ++i)
    for (int j = 0; j < nsh; ++j) {
      double mx = 0.0;
      for (int a = 0; a < basis.shells()[i].n_func(); ++a) {
        size_t row = (size_t)(offs[i] + a) * nao + offs[j];
        for (int bb = 0; bb < basis.shells()[j].n_func(); ++bb)
          mx = std::fmax(mx, std::fabs(d[row + bb]));
      }
      bounds[(size_t)i * nsh + j] = mx;
    }
  return bounds;
}

namespace {
// direct.rs:377-404
inline void add_contraction(double* J, double* K, const double* D, size_t n, double g, size_t a,
                            size_t b, size_t c, size_t d, bool want_k) {
  J[a * n + b] += g * D[c * n + d];
  if (want_k) K[a * n + c] += g * D[b * n + d];
}
// direct.rs:352-375
inline void scatter_unique(double* J, double* K, const double* D, size_t n, double g, size_t a,
                           size_t b, size_t c, size_t d, bool want_k) {
  add_contraction(J, K, D, n, g, a, b, c, d, want_k);
  if (a != b) add_contraction(J, K, D, n, g, b, a, c, d, want_k);
  if (c != d) {
    add_contraction(J, K, D, n, g, a, b, d, c, want_k);
    if (a != b) add_contraction(J, K, D, n, g, b, a, d, c, want_k);
  }
  if (!(a == c && b == d)) {
    add_contraction(J, K, D, n, g, c, d, a, b, want_k);
    if (c != d) add_contraction(J, K, D, n, g, d, c, a, b, want_k);
    if (a != b) {
      add_contraction(J, K, D, n, g, c, d, b, a, want_k);
      if (c != d) add_contraction(J, K, D, n, g, d, c, b, a, want_k);
    }
  }
}
}  // namespace

// direct.rs:284-326
void DirectPlan::scatter_block(const int idx[4], const double* block, uint64_t mask,
                               const JKArgs& a) const {
  const auto& sh = basis.shells();
  const auto& offs = basis.offsets();
  int si = idx[0], sj = idx[1], sk = idx[2], sl = idx[3];
  int na = sh[si].n_func(), nb = sh[sj].n_func(), nc = sh[sk].n_func(), nd = sh[sl].n_func();
  size_t n = (size_t)basis.nao();
  for (int ia = 0; ia < na; ++ia) {
    size_t mu = offs[si] + ia;
    int b_hi = si == sj ? ia + 1 : nb;
    for (int ib = 0; ib < b_hi; ++ib) {
      size_t nu = offs[sj] + ib;
      for (int ic = 0; ic < nc; ++ic) {
        size_t lam = offs[sk] + ic;
        int d_hi = sk == sl ? ic + 1 : nd;
        size_t base = (((size_t)ia * nb + ib) * nc + ic) * nd;
        for (int id = 0; id < d_hi; ++id) {
          size_t sig = offs[sl] + id;
          if (si == sk && sj == sl && std::make_pair(mu, nu) < std::make_pair(lam, sig)) continue;
          double g = block[base + id];
          for (int di = 0; di < a.ndens; ++di)
            if (mask & (1ull << di))
              scatter_unique(a.J[di], a.want_k ? a.K[di] : nullptr, a.D[di], n, g, mu, nu, lam,
                             sig, a.want_k);
        }
      }
    }
  }
}

// direct.rs:131-218, with the batch-of-4 queue order replicated (each lane
// is bit-identical to the scalar evaluation, so evaluating at flush time in
// lane order reproduces the reference's accumulation order).
void DirectPlan::accumulate_bra_pair(int i, int j, const JKArgs& a, QuartetSink* sink) const {
  int nsh = basis.nsh();
  const auto& sh = basis.shells();
  double qab = schwarz[(size_t)i * nsh + j];
  if (qab == 0.0) return;
  using Key = std::tuple<int, int, int, int>;
  std::map<Key, std::vector<std::pair<std::array<int, 4>, uint64_t>>> pending;
  auto consume = [&](const std::array<int, 4>& q, uint64_t mask) {
    std::vector<double> blk = basis.eri_block_pairs(engine, q[0], q[1], q[2], q[3]);
    scatter_block(q.data(), blk.data(), mask, a);
  };
  for (int k = 0; k <= i; ++k) {
    int l_top = k == i ? j : k;
    for (int l = 0; l <= l_top; ++l) {
      double pair_bound = qab * schwarz[(size_t)k * nsh + l];
      if (pair_bound < a.threshold) continue;
      uint64_t mask = 0;
      for (int di = 0; di < a.ndens; ++di) {
        const double* bd = a.bounds[di];
        double dbound = std::fmax(
            std::fmax(std::fmax(std::fmax(std::fmax(bd[(size_t)i * nsh + j], bd[(size_t)k * nsh + l]),
                                          bd[(size_t)i * nsh + k]),
                                bd[(size_t)i * nsh + l]),
                      bd[(size_t)j * nsh + k]),
            bd[(size_t)j * nsh + l]);
        if (pair_bound * dbound >= a.threshold) mask |= 1ull << di;
      }
      if (mask == 0) continue;
      if (sink) sink->add(i, j, k, l, mask);
      if (a.count_only) continue;
      std::array<int, 4> q = {i, j, k, l};
      // eri_batch.rs:42-61
      Engine r = engine;
      if (engine == Engine::Auto)
        r = select_engine(sh[i].l + sh[j].l, sh[k].l + sh[l].l,
                          sh[i].n_prim() * sh[j].n_prim() * sh[k].n_prim() * sh[l].n_prim());
      int ne = sh[i].l + sh[j].l, nf = sh[k].l + sh[l].l;
      if (r == Engine::OsHgp && ne <= 6 && nf <= 6) {
        Key key{ne, nf, (int)basis.pair_data(i, j).size(), (int)basis.pair_data(k, l).size()};
        auto& pend = pending[key];
        pend.push_back({q, mask});
        if (pend.size() == 4) {
          auto group = pend;
          pend.clear();
          for (auto& g : group) consume(g.first, g.second);
        }
      } else {
        consume(q, mask);
      }
    }
  }
  for (auto& kv : pending)
    for (auto& g : kv.second) consume(g.first, g.second);
}

// ------------------------------------------------------------- gradient

GradPlan::GradPlan(const Basis& b, Engine e) : basis(b), engine(e) {
  for (const Shell& s : b.shells())
    if (s.l > MAX_GRAD_L) throw std::invalid_argument("angular momentum too high for gradient");
  int nsh = b.nsh();
  for (int s = 0; s < nsh; ++s) {
    const Shell& sh = b.shells()[s];
    std::vector<double> e2;
    for (int p = 0; p < sh.n_prim(); ++p) e2.push_back(2.0 * sh.exps[p] * b.eff(s)[p]);
    eff_2a.push_back(e2);
    // transposed c2s (n_cart x n_func)
    const std::vector<double>& m = b.c2s(s);
    if (m.empty()) {
      s2c.push_back({});
    } else {
      int nf = sh.n_func(), nc = sh.n_cart();
      std::vector<double> t((size_t)nc * nf, 0.0);
      for (int f = 0; f < nf; ++f)
        for (int c = 0; c < nc; ++c) t[(size_t)c * nf + f] = m[(size_t)f * nc + c];
      s2c.push_back(t);
    }
  }
  for (int i = 0; i < nsh; ++i)
    for (int j = 0; j <= i; ++j) {
      const Shell &si = b.shells()[i], &sj = b.shells()[j];
      pair_first_2a.push_back(build_pairs(si, eff_2a[i].data(), sj, b.eff(j).data()));
      pair_second_2a.push_back(build_pairs(si, b.eff(i).data(), sj, eff_2a[j].data()));
    }
  schwarz = b.schwarz(Engine::Auto);
}

// direct_grad.rs:292-312
std::vector<double> GradPlan::shell_block_max(const double* m) const {
  int nsh = basis.nsh(), nao = basis.nao();
  const auto& offs = basis.offsets();
  std::vector<double> bounds((size_t)nsh * nsh, 0.0);
  for (int i = 0; i < nsh; ++i)
    for (int j = 0; j < nsh; ++j) {
      double mx = 0.0;
      for (int a = 0; a < basis.shells()[i].n_func(); ++a) {
        size_t row = (size_t)(offs[i] + a) * nao + offs[j];
        for (int bb = 0; bb < basis.shells()[j].n_func(); ++bb)
          mx = std::fmax(mx, std::fabs(m[row + bb]));
      }
      int lo = std::min(i, j), hi = std::max(i, j);
      double sym = std::fmax(bounds[(size_t)hi * nsh + lo], mx);
      bounds[(size_t)hi * nsh + lo] = sym;
      bounds[(size_t)lo * nsh + hi] = sym;
    }
  return bounds;
}

GradDensity GradPlan::density(const std::vector<GradTerm>& coul,
                              const std::vector<GradTerm>& exch) const {
  GradDensity d;
  for (const GradTerm& t : coul)
    d.coulomb.push_back({t, shell_block_max(t.left), shell_block_max(t.right)});
  for (const GradTerm& t : exch)
    d.exchange.push_back({t, shell_block_max(t.left), shell_block_max(t.right)});
  return d;
}

// direct_grad.rs:626-644
double GradDensity::block_bound(int nsh, int i, int j, int k, int l) const {
  auto at = [&](const std::vector<double>& m, int a, int b) { return m[(size_t)a * nsh + b]; };
  double bound = 0.0;
  for (const auto& t : coulomb)
    bound += 0.5 * std::fabs(t.term.factor) *
             (at(t.left_max, i, j) * at(t.right_max, k, l) + at(t.left_max, k, l) * at(t.right_max, i, j));
  for (const auto& t : exchange)
    bound += 0.25 * std::fabs(t.term.factor) *
             (at(t.left_max, i, k) * at(t.right_max, j, l) + at(t.left_max, j, k) * at(t.right_max, i, l) +
              at(t.left_max, i, l) * at(t.right_max, j, k) + at(t.left_max, j, l) * at(t.right_max, i, k));
  return bound;
}

// direct_grad.rs:490-547
std::vector<double> GradPlan::weight_block(const int idx[4], double degeneracy,
                                           const GradDensity& dens) const {
  size_t n = (size_t)basis.nao();
  const auto& offs = basis.offsets();
  const auto& sh = basis.shells();
  int oi = offs[idx[0]], oj = offs[idx[1]], ok = offs[idx[2]], ol = offs[idx[3]];
  int ni = sh[idx[0]].n_func(), nj = sh[idx[1]].n_func(), nk = sh[idx[2]].n_func(),
      nl = sh[idx[3]].n_func();
  std::vector<double> w((size_t)ni * nj * nk * nl, 0.0);
  for (const auto& bt : dens.coulomb) {
    const double *left = bt.term.left, *right = bt.term.right;
    double f = 0.5 * degeneracy * bt.term.factor;
    for (int a = 0; a < ni; ++a)
      for (int b = 0; b < nj; ++b) {
        size_t mn = (size_t)(oi + a) * n + oj + b;
        double l_mn = f * left[mn], r_mn = f * right[mn];
        double* row = &w[((size_t)a * nj + b) * nk * nl];
        for (int c = 0; c < nk; ++c) {
          size_t ls = (size_t)(ok + c) * n + ol;
          for (int d = 0; d < nl; ++d) row[c * nl + d] += l_mn * right[ls + d] + r_mn * left[ls + d];
        }
      }
  }
  for (const auto& bt : dens.exchange) {
    const double *left = bt.term.left, *right = bt.term.right;
    double f = 0.25 * degeneracy * bt.term.factor;
    for (int a = 0; a < ni; ++a) {
      size_t mu = (size_t)(oi + a) * n;
      for (int b = 0; b < nj; ++b) {
        size_t nu = (size_t)(oj + b) * n;
        double* row = &w[((size_t)a * nj + b) * nk * nl];
        for (int c = 0; c < nk; ++c) {
          size_t lam = ok + c;
          double l_ml = f * left[mu + lam], r_ml = f * right[mu + lam];
          double l_nl = f * left[nu + lam], r_nl = f * right[nu + lam];
          for (int d = 0; d < nl; ++d) {
            size_t sig = ol + d;
            row[c * nl + d] += l_ml * right[nu + sig] + l_nl * right[mu + sig] +
                               left[mu + sig] * r_nl + left[nu + sig] * r_ml;
          }
        }
      }
    }
  }
  const std::vector<double>* mats[4] = {&s2c[idx[0]], &s2c[idx[1]], &s2c[idx[2]], &s2c[idx[3]]};
  int dims[4] = {ni, nj, nk, nl};
  return transform_block4(std::move(w), dims, mats);
}

// direct_grad.rs:554-620
void GradPlan::shifted_block(const int idx[4], int pos, int lp, bool weighted, bool use_rys,
                             double* out) const {
  const auto& sh = basis.shells();
  int ls[4];
  for (int p = 0; p < 4; ++p) ls[p] = p == pos ? lp : sh[idx[p]].l;
  auto coeffs_at = [&](int p) -> const std::vector<double>& {
    return (p == pos && weighted) ? eff_2a[idx[p]] : basis.eff(idx[p]);
  };
  if (!use_rys) {
    size_t bra = tri_idx(idx[0], idx[1]), ket = tri_idx(idx[2], idx[3]);
    const std::vector<PrimPair>* bp = &basis.pair_data(idx[0], idx[1]);
    if (weighted && pos == 0) bp = &pair_first_2a[bra];
    if (weighted && pos == 1) bp = &pair_second_2a[bra];
    const std::vector<PrimPair>* kp = &basis.pair_data(idx[2], idx[3]);
    if (weighted && pos == 2) kp = &pair_first_2a[ket];
    os_shell_quartet(sh[idx[0]], sh[idx[1]], sh[idx[2]], sh[idx[3]], *bp, *kp, ls[0], ls[1], ls[2],
                     ls[3], out);
    return;
  }
  const std::vector<double>&c0 = coeffs_at(0), &c1 = coeffs_at(1), &c2 = coeffs_at(2),
  &c3 = coeffs_at(3);
  for (size_t pa = 0; pa < c0.size(); ++pa)
    for (size_t pb = 0; pb < c1.size(); ++pb)
      for (size_t pc = 0; pc < c2.size(); ++pc)
        for (size_t pd = 0; pd < c3.size(); ++pd) {
          double scale = c0[pa] * c1[pb] * c2[pc] * c3[pd];
          rys_prim_quartet(sh[idx[0]].exps[pa], sh[idx[0]].center, ls[0], sh[idx[1]].exps[pb],
                           sh[idx[1]].center, ls[1], sh[idx[2]].exps[pc], sh[idx[2]].center, ls[2],
                           sh[idx[3]].exps[pd], sh[idx[3]].center, ls[3], scale, out);
        }
}

// direct_grad.rs:394-485
void GradPlan::quartet(const int idx[4], double degeneracy, const GradDensity& dens,
                       double* out) const {
  contract_weights(idx, weight_block(idx, degeneracy, dens), out);
}

// The derivative of one shell quartet contracted with its Cartesian weight
// block w: raised (2-alpha weighted) and lowered blocks on positions 0..2,
// the fourth centre by translational invariance (direct_grad.rs:431-485).
void GradPlan::contract_weights(const int idx[4], const std::vector<double>& w,
                                double* out) const {
  const auto& sh = basis.shells();
  int ls[4], dims[4];
  for (int p = 0; p < 4; ++p) {
    ls[p] = sh[idx[p]].l;
    dims[p] = n_cart(ls[p]);
  }
  Engine r = engine;
  if (engine == Engine::Auto)
    r = select_engine(ls[0] + ls[1], ls[2] + ls[3],
                      sh[idx[0]].n_prim() * sh[idx[1]].n_prim() * sh[idx[2]].n_prim() *
                          sh[idx[3]].n_prim());
  bool use_rys = r == Engine::Rys;
  double fourth[3] = {0, 0, 0};
  for (int pos = 0; pos < 3; ++pos) {
    int l = ls[pos];
    int up_dims[4] = {dims[0], dims[1], dims[2], dims[3]};
    up_dims[pos] = n_cart(l + 1);
    std::vector<double> raised((size_t)up_dims[0] * up_dims[1] * up_dims[2] * up_dims[3], 0.0);
    shifted_block(idx, pos, l + 1, true, use_rys, raised.data());
    std::vector<double> lowered;
    if (l > 0) {
      int dd[4] = {dims[0], dims[1], dims[2], dims[3]};
      dd[pos] = n_cart(l - 1);
      lowered.assign((size_t)dd[0] * dd[1] * dd[2] * dd[3], 0.0);
      shifted_block(idx, pos, l - 1, false, use_rys, lowered.data());
    }
    size_t outer = 1, inner = 1;
    for (int q = 0; q < pos; ++q) outer *= dims[q];
    for (int q = pos + 1; q < 4; ++q) inner *= dims[q];
    int nn = dims[pos], n_up = up_dims[pos], n_down = l > 0 ? n_cart(l - 1) : 0;
    std::vector<Tri> comps = cart_components(l);
    double g[3] = {0, 0, 0};
    for (size_t o = 0; o < outer; ++o)
      for (int a = 0; a < nn; ++a) {
        const double* wr = &w[(o * nn + a) * inner];
        for (int axis = 0; axis < 3; ++axis) {
          Tri up = comps[a];
          up[axis] += 1;
          size_t upo = (o * n_up + cart_index(up)) * inner;
          double dot = 0.0;
          for (size_t s = 0; s < inner; ++s) dot += wr[s] * raised[upo + s];
          g[axis] += dot;
          if (comps[a][axis] != 0) {
            Tri dn = comps[a];
            dn[axis] -= 1;
            double count = (double)comps[a][axis];
            size_t dno = (o * n_down + cart_index(dn)) * inner;
            double dot2 = 0.0;
            for (size_t s = 0; s < inner; ++s) dot2 += wr[s] * lowered[dno + s];
            g[axis] -= count * dot2;
          }
        }
      }
    int atom = basis.shell_atom()[idx[pos]];
    for (int axis = 0; axis < 3; ++axis) {
      out[(size_t)atom * 3 + axis] += g[axis];
      fourth[axis] -= g[axis];
    }
  }
  int atom = basis.shell_atom()[idx[3]];
  for (int axis = 0; axis < 3; ++axis) out[(size_t)atom * 3 + axis] += fourth[axis];
}

// Basis::eri_grad_contract_with (grad.rs:427-470): the gradient of
// E = sum over all ordered quartets of gamma[mu nu la si] (mu nu|la si), the
// reference's dense oracle of the direct gradient.  gamma is nao^4, function
// space.  Each ordered quartet is evaluated in the orientation with i >= j
// and k >= l (the pair data are stored for canonical pairs), its gamma block
// permuted to match; the derivative of a permuted block is the permuted
// derivative, so the contraction is unchanged.
void GradPlan::dense_contract(const double* gamma, double* out) const {
  const auto& sh = basis.shells();
  const auto& offs = basis.offsets();
  const size_t n = (size_t)basis.nao();
  const int nsh = basis.nsh();
  for (int i = 0; i < nsh; ++i)
    for (int j = 0; j < nsh; ++j)
      for (int k = 0; k < nsh; ++k)
        for (int l = 0; l < nsh; ++l) {
          const bool sb = i < j, sk = k < l;
          const int idx[4] = {sb ? j : i, sb ? i : j, sk ? l : k, sk ? k : l};
          int dims[4];
          for (int p = 0; p < 4; ++p) dims[p] = sh[idx[p]].n_func();
          std::vector<double> w((size_t)dims[0] * dims[1] * dims[2] * dims[3]);
          const int ni = sh[i].n_func(), nj = sh[j].n_func(), nk = sh[k].n_func(), nl = sh[l].n_func();
          for (int a = 0; a < ni; ++a)
            for (int b = 0; b < nj; ++b)
              for (int c = 0; c < nk; ++c)
                for (int d = 0; d < nl; ++d) {
                  const int x0 = sb ? b : a, x1 = sb ? a : b, x2 = sk ? d : c, x3 = sk ? c : d;
                  w[(((size_t)x0 * dims[1] + x1) * dims[2] + x2) * dims[3] + x3] =
                      gamma[(((size_t)(offs[i] + a) * n + offs[j] + b) * n + offs[k] + c) * n + offs[l] + d];
                }
          const std::vector<double>* mats[4] = {&s2c[idx[0]], &s2c[idx[1]], &s2c[idx[2]], &s2c[idx[3]]};
          contract_weights(idx, transform_block4(std::move(w), dims, mats), out);
        }
}

// direct_grad.rs:328-373
void GradPlan::accumulate_bra_pair(int i, int j, const GradDensity& dens, double threshold,
                                   double* out, QuartetSink* sink, bool count_only) const {
  int nsh = basis.nsh();
  double qab = schwarz[(size_t)i * nsh + j];
  if (qab == 0.0 && threshold > 0.0) return;
  const auto& atoms = basis.shell_atom();
  for (int k = 0; k <= i; ++k) {
    int l_top = k == i ? j : k;
    for (int l = 0; l <= l_top; ++l) {
      if (atoms[i] == atoms[j] && atoms[j] == atoms[k] && atoms[k] == atoms[l]) continue;
      double pair_bound = qab * schwarz[(size_t)k * nsh + l];
      if (pair_bound < threshold) continue;
      double degeneracy = (i == j ? 1.0 : 2.0) * (k == l ? 1.0 : 2.0) * (i == k && j == l ? 1.0 : 2.0);
      if (pair_bound * degeneracy * dens.block_bound(nsh, i, j, k, l) < threshold) continue;
      if (sink) sink->add(i, j, k, l, 1);
      if (count_only) continue;
      int idx[4] = {i, j, k, l};
      quartet(idx, degeneracy, dens, out);
    }
  }
}

// ------------------------------------------------------------- drivers

void run_jk(const DirectPlan& plan, const JKArgs& a, const std::vector<int>& bras, int nthreads,
            QuartetSink* sink) {
  size_t n2 = (size_t)plan.basis.nao() * plan.basis.nao();
  if (nthreads <= 1) {
    for (int b : bras) plan.accumulate_bra_pair(plan.pairs[b][0], plan.pairs[b][1], a, sink);
    return;
  }
  // Caller-side parallelism exactly as the reference documents it: one
  // workspace and one private set of J/K buffers per worker, bra pairs as the
  // grain (static round-robin, so the summation order is reproducible), and
  // the private buffers summed at the end.
  std::vector<std::vector<double>> privJ(nthreads), privK(nthreads);
  std::vector<QuartetSink> sinks(nthreads);
  std::vector<std::thread> th;
  for (int t = 0; t < nthreads; ++t) {
    th.emplace_back([&, t] {
      privJ[t].assign(n2 * a.ndens, 0.0);
      if (a.want_k) privK[t].assign(n2 * a.ndens, 0.0);
      JKArgs mine = a;
      for (int d = 0; d < a.ndens; ++d) {
        mine.J[d] = &privJ[t][d * n2];
        mine.K[d] = a.want_k ? &privK[t][d * n2] : nullptr;
      }
      for (size_t b = t; b < bras.size(); b += nthreads)
        plan.accumulate_bra_pair(plan.pairs[bras[b]][0], plan.pairs[bras[b]][1], mine,
                                 sink ? &sinks[t] : nullptr);
    });
  }
  for (auto& x : th) x.join();
  for (int t = 0; t < nthreads; ++t) {
    for (int d = 0; d < a.ndens; ++d)
      for (size_t e = 0; e < n2; ++e) {
        a.J[d][e] += privJ[t][d * n2 + e];
        if (a.want_k) a.K[d][e] += privK[t][d * n2 + e];
      }
    if (sink) {
      sink->count += sinks[t].count;
      sink->hash += sinks[t].hash;
    }
  }
}

void run_grad(const GradPlan& plan, const GradDensity& dens, double threshold,
              const std::vector<int>& bras, int nthreads, double* out, QuartetSink* sink,
              bool count_only) {
  size_t no = (size_t)plan.basis.atoms().size() * 3;
  std::vector<std::array<int, 2>> pairs;
  for (int i = 0; i < plan.basis.nsh(); ++i)
    for (int j = 0; j <= i; ++j) pairs.push_back({i, j});
  if (nthreads <= 1) {
    for (int b : bras)
      plan.accumulate_bra_pair(pairs[b][0], pairs[b][1], dens, threshold, out, sink, count_only);
    return;
  }
  std::vector<std::vector<double>> priv(nthreads);
  std::vector<QuartetSink> sinks(nthreads);
  std::vector<std::thread> th;
  for (int t = 0; t < nthreads; ++t) {
    th.emplace_back([&, t] {
      priv[t].assign(no, 0.0);
      for (size_t b = t; b < bras.size(); b += nthreads)
        plan.accumulate_bra_pair(pairs[bras[b]][0], pairs[bras[b]][1], dens, threshold,
                                 priv[t].data(), sink ? &sinks[t] : nullptr, count_only);
    });
  }
  for (auto& x : th) x.join();
  for (int t = 0; t < nthreads; ++t) {
    for (size_t e = 0; e < no; ++e) out[e] += priv[t][e];
    if (sink) {
      sink->count += sinks[t].count;
      sink->hash += sinks[t].hash;
    }
  }
}

}  // namespace oracle
