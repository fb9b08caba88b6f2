// ORACLE — test infrastructure only (see oracle.hpp).
// L3 drivers: basis metadata, quartet glue, dense 8-fold ERI, Schwarz bounds.
#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <thread>

#include "oracle.hpp"

namespace oracle {

// shell.rs:193-276
Basis::Basis(std::vector<Shell> shells) : shells_(std::move(shells)) {
  int acc = 0;
  for (const Shell& s : shells_) {
    if (s.exps.empty()) throw std::invalid_argument("empty contraction");
    if (s.exps.size() != s.coefs.size()) throw std::invalid_argument("mismatched contraction");
    if (s.l > MAX_L || s.l < 0) throw std::invalid_argument("angular momentum too high");
    offs_.push_back(acc);
    acc += s.n_func();
  }
  nao_ = acc;
  for (const Shell& s : shells_) {
    auto it = std::find(atoms_.begin(), atoms_.end(), s.center);
    if (it == atoms_.end()) {
      shell_atom_.push_back((int)atoms_.size());
      atoms_.push_back(s.center);
    } else {
      shell_atom_.push_back((int)(it - atoms_.begin()));
    }
  }
  for (const Shell& s : shells_) {
    std::vector<double> e;
    for (int i = 0; i < s.n_prim(); ++i) e.push_back(s.primitive_coeff(i));
    eff_.push_back(e);
    if (s.spherical) {
      // spherical.rs:37-48: ratio * c2s_matrix(l)
      double ratio = monomial_to_raw_factor(s.l);
      std::vector<double> m = c2s_matrix(s.l);
      for (double& v : m) v = ratio * v;
      c2s_.push_back(m);
    } else {
      c2s_.push_back({});
    }
  }
  for (int i = 0; i < nsh(); ++i)
    for (int j = 0; j <= i; ++j)
      pair_data_.push_back(build_pairs(shells_[i], eff_[i].data(), shells_[j], eff_[j].data()));
}

const std::vector<PrimPair>& Basis::pair_data(int i, int j) const {
  return pair_data_[tri_idx((size_t)i, (size_t)j)];
}

// spherical.rs:121-179: per-axis contraction, zero matrix entries skipped.
std::vector<double> transform_block4(std::vector<double> block, const int dims_in[4],
                                     const std::vector<double>* mats[4]) {
  int dims[4] = {dims_in[0], dims_in[1], dims_in[2], dims_in[3]};
  for (int axis = 0; axis < 4; ++axis) {
    const std::vector<double>* mp = mats[axis];
    if (!mp || mp->empty()) continue;
    const std::vector<double>& mat = *mp;
    int n_in = dims[axis];
    int n_out = (int)mat.size() / dims_in[axis];
    size_t outer = 1, inner = 1;
    for (int q = 0; q < axis; ++q) outer *= dims[q];
    for (int q = axis + 1; q < 4; ++q) inner *= dims[q];
    std::vector<double> out(outer * n_out * inner, 0.0);
    for (size_t o = 0; o < outer; ++o)
      for (int q = 0; q < n_out; ++q) {
        size_t dst = (o * n_out + q) * inner;
        for (int j = 0; j < n_in; ++j) {
          double m = mat[(size_t)q * n_in + j];
          if (m == 0.0) continue;
          size_t src = (o * n_in + j) * inner;
          for (size_t s = 0; s < inner; ++s) out[dst + s] += m * block[src + s];
        }
      }
    dims[axis] = n_out;
    block.swap(out);
  }
  return block;
}

namespace {
// integrals.rs:1086-1114: Rys path over every primitive quartet.
void contract_rys(const Shell* s[4], const std::vector<double>* eff[4], const int l[4],
                  double* block) {
  for (size_t pa = 0; pa < eff[0]->size(); ++pa)
    for (size_t pb = 0; pb < eff[1]->size(); ++pb)
      for (size_t pc = 0; pc < eff[2]->size(); ++pc)
        for (size_t pd = 0; pd < eff[3]->size(); ++pd) {
          double scale = (*eff[0])[pa] * (*eff[1])[pb] * (*eff[2])[pc] * (*eff[3])[pd];
          rys_prim_quartet(s[0]->exps[pa], s[0]->center, l[0], s[1]->exps[pb], s[1]->center, l[1],
                           s[2]->exps[pc], s[2]->center, l[2], s[3]->exps[pd], s[3]->center, l[3],
                           scale, block);
        }
}
}  // namespace

std::vector<double> Basis::eri_block(Engine e, int i, int j, int k, int l) const {
  const Shell* s[4] = {&shells_[i], &shells_[j], &shells_[k], &shells_[l]};
  int ls[4] = {s[0]->l, s[1]->l, s[2]->l, s[3]->l};
  int dims[4] = {s[0]->n_cart(), s[1]->n_cart(), s[2]->n_cart(), s[3]->n_cart()};
  std::vector<double> block((size_t)dims[0] * dims[1] * dims[2] * dims[3], 0.0);
  Engine r = e;
  if (e == Engine::Auto)
    r = select_engine(ls[0] + ls[1], ls[2] + ls[3],
                      s[0]->n_prim() * s[1]->n_prim() * s[2]->n_prim() * s[3]->n_prim());
  if (r == Engine::OsHgp) {
    std::vector<PrimPair> bra = build_pairs(*s[0], eff_[i].data(), *s[1], eff_[j].data());
    std::vector<PrimPair> ket = build_pairs(*s[2], eff_[k].data(), *s[3], eff_[l].data());
    os_shell_quartet(*s[0], *s[1], *s[2], *s[3], bra, ket, ls[0], ls[1], ls[2], ls[3],
                     block.data());
  } else {
    const std::vector<double>* ef[4] = {&eff_[i], &eff_[j], &eff_[k], &eff_[l]};
    contract_rys(s, ef, ls, block.data());
  }
  const std::vector<double>* mats[4] = {&c2s_[i], &c2s_[j], &c2s_[k], &c2s_[l]};
  return transform_block4(std::move(block), dims, mats);
}

std::vector<double> Basis::eri_block_pairs(Engine e, int i, int j, int k, int l) const {
  const Shell* s[4] = {&shells_[i], &shells_[j], &shells_[k], &shells_[l]};
  int ls[4] = {s[0]->l, s[1]->l, s[2]->l, s[3]->l};
  int dims[4] = {s[0]->n_cart(), s[1]->n_cart(), s[2]->n_cart(), s[3]->n_cart()};
  std::vector<double> block((size_t)dims[0] * dims[1] * dims[2] * dims[3], 0.0);
  Engine r = e;
  if (e == Engine::Auto)
    r = select_engine(ls[0] + ls[1], ls[2] + ls[3],
                      s[0]->n_prim() * s[1]->n_prim() * s[2]->n_prim() * s[3]->n_prim());
  if (r == Engine::OsHgp) {
    os_shell_quartet(*s[0], *s[1], *s[2], *s[3], pair_data(i, j), pair_data(k, l), ls[0], ls[1],
                     ls[2], ls[3], block.data());
  } else {
    const std::vector<double>* ef[4] = {&eff_[i], &eff_[j], &eff_[k], &eff_[l]};
    contract_rys(s, ef, ls, block.data());
  }
  const std::vector<double>* mats[4] = {&c2s_[i], &c2s_[j], &c2s_[k], &c2s_[l]};
  return transform_block4(std::move(block), dims, mats);
}

namespace {
// integrals.rs:1235-1244
const int PERMS8[8][4] = {{0, 1, 2, 3}, {1, 0, 2, 3}, {0, 1, 3, 2}, {1, 0, 3, 2},
                          {2, 3, 0, 1}, {2, 3, 1, 0}, {3, 2, 0, 1}, {3, 2, 1, 0}};

// integrals.rs:1271-1312
void scatter_s8(double* out, size_t nao, const int sidx[4], const std::vector<int>& offs,
                const int n[4], const double* block) {
  int seen[8][4];
  int n_seen = 0;
  for (const auto& perm : PERMS8) {
    int tup[4] = {sidx[perm[0]], sidx[perm[1]], sidx[perm[2]], sidx[perm[3]]};
    bool dup = false;
    for (int s = 0; s < n_seen; ++s)
      if (std::equal(tup, tup + 4, seen[s])) dup = true;
    if (dup) continue;
    std::copy(tup, tup + 4, seen[n_seen++]);
    size_t stride[4] = {0, 0, 0, 0};
    size_t base = 0;
    for (int q = 0; q < 4; ++q) {
      int src_axis = perm[q];
      size_t st = 1;
      for (int e = 0; e < 3 - q; ++e) st *= nao;
      stride[src_axis] = st;
      base += (size_t)offs[sidx[src_axis]] * st;
    }
    size_t src = 0;
    for (int a = 0; a < n[0]; ++a)
      for (int b = 0; b < n[1]; ++b)
        for (int c = 0; c < n[2]; ++c)
          for (int d = 0; d < n[3]; ++d)
            out[base + a * stride[0] + b * stride[1] + c * stride[2] + d * stride[3]] =
                block[src++];
  }
}
}  // namespace

// integrals.rs:671-754 (the batch-of-4 path is bit-identical per lane and
// every output slot is written exactly once, so evaluation order is moot).
std::vector<double> Basis::eri(Engine e) const {
  size_t n = (size_t)nao_;
  std::vector<double> out(n * n * n * n, 0.0);
  for (int si = 0; si < nsh(); ++si)
    for (int sj = 0; sj <= si; ++sj)
      for (int sk = 0; sk <= si; ++sk) {
        int l_top = sk == si ? sj : sk;
        for (int sl = 0; sl <= l_top; ++sl) {
          std::vector<double> blk = eri_block_pairs(e, si, sj, sk, sl);
          int sidx[4] = {si, sj, sk, sl};
          int nf[4] = {shells_[si].n_func(), shells_[sj].n_func(), shells_[sk].n_func(),
                       shells_[sl].n_func()};
          scatter_s8(out.data(), n, sidx, offs_, nf, blk.data());
        }
      }
  return out;
}

// integrals.rs:842-862
// Every entry is an independent evaluation, so rows are spread over host
// threads (each entry's arithmetic is unchanged).
std::vector<double> Basis::schwarz(Engine e) const {
  int n = nsh();
  std::vector<double> q((size_t)n * n, 0.0);
  auto row = [&](int i) {
    for (int j = 0; j < n; ++j) {
      int ni = shells_[i].n_func(), nj = shells_[j].n_func();
      std::vector<double> blk = eri_block(e, i, j, i, j);
      double mx = 0.0;
      for (int mu = 0; mu < ni; ++mu)
        for (int nu = 0; nu < nj; ++nu) {
          size_t idx = (((size_t)mu * nj + nu) * ni + mu) * nj + nu;
          mx = std::fmax(mx, std::fabs(blk[idx]));
        }
      q[(size_t)i * n + j] = std::sqrt(mx);
    }
  };
  int nt = (int)std::thread::hardware_concurrency();
  if (nt < 1) nt = 1;
  if (nt > 64) nt = 64;
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t)
    th.emplace_back([&, t] {
      for (int i = t; i < n; i += nt) row(i);
    });
  for (auto& x : th) x.join();
  return q;
}

}  // namespace oracle
