// Task decoding, screening, and the per-quartet post phase (horizontal
// recurrences on the contracted table, Cartesian -> spherical transform, and
// the consumers: J/K contraction, dense 8-fold scatter, EriBuilder 4-fold
// scatter, Schwarz diagonal maximum).  Runs on a team of T lanes over a
// per-team scratch slot in global memory.
#pragma once
#include "device_common.cuh"

namespace igpu {

struct ClassDims {
  int la, lb, lc, ld;
};

// Scratch-slot layout of one quartet (in doubles): three level buffers of S
// doubles (the first holds G on entry), then the Cartesian block and its
// transform partner.
struct SlotLayout {
  size_t S, blk, total;
};
__host__ __device__ inline SlotLayout slot_layout(int la, int lb, int lc, int ld) {
  int ne = la + lb, nf = lc + ld;
  int nep = nrange(la, ne), nfp = nrange(lc, nf);
  size_t S = (size_t)nep * nfp;
  for (int kb = 1; kb <= lb; ++kb) {
    size_t s = (size_t)ncart(kb) * nrange(la, ne - kb) * nfp;
    S = s > S ? s : S;
  }
  size_t nab = (size_t)ncart(la) * ncart(lb);
  for (int kd = 1; kd <= ld; ++kd) {
    size_t s = nab * ncart(kd) * nrange(lc, nf - kd);
    S = s > S ? s : S;
  }
  size_t blk = nab * ncart(lc) * ncart(ld);
  SlotLayout L;
  L.S = S;
  L.blk = blk;
  L.total = 3 * S + 2 * blk;
  return L;
}

// Position in a task list: segment `seg` (one bra pair and a run of its
// kets) covers tasks [lo, hi) with lo = prefix[seg].  A team seeks once per
// claimed chunk (binary search) and then walks forward, its tasks being
// increasing.  Task g is ket ket_start[seg] + (g - lo) of bra bra_pair[seg].
struct TaskCursor {
  int seg;
  unsigned long long lo, hi;
};
__device__ __forceinline__ void cursor_seek(const TaskList& t, unsigned long long g, TaskCursor& c) {
  int lo = 0, hi = t.nbra;  // prefix[lo] <= g < prefix[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (t.prefix[mid] <= g)
      lo = mid;
    else
      hi = mid;
  }
  c.seg = lo;
  c.lo = t.prefix[lo];
  c.hi = t.prefix[lo + 1];
}
__device__ __forceinline__ void cursor_decode(const TaskList& t, unsigned long long g, TaskCursor& c, int& pbi,
                                              int& pki) {
  while (g >= c.hi) {  // g < prefix[nbra] = total, so seg stays below nbra
    ++c.seg;
    c.lo = c.hi;
    c.hi = t.prefix[c.seg + 1];
  }
  const int kpos = (int)(g - c.lo) + (t.ket_start ? t.ket_start[c.seg] : 0);
  pbi = t.bra_pair[c.seg];
  pki = t.ket_pairs[kpos];
}

struct Screen {
  bool keep;
  bool swapped;       // reference bra is the evaluation ket pair
  uint64_t mask;      // densities this quartet contributes to
  int i, j, k, l;     // reference canonical shells
  double degeneracy;  // gradient: images of the canonical quartet
};

// Bound on the permutation-averaged two-particle density over the function
// block of canonical quartet (i,j,k,l) (src/direct_grad.rs:626-644).  The
// rounding of every product and sum is the reference's (no contraction into
// fused multiply-adds), so the screened list is bit-identical.
__device__ __forceinline__ double grad_block_bound(const GradDev& g, int nsh, int i, int j, int k, int l) {
  auto at = [nsh](const double* m, int a, int b) { return __ldg(m + (size_t)a * nsh + b); };
  double bound = 0.0;
  for (int t = 0; t < g.ncoul; ++t) {
    const double* L = g.cl_max[t];
    const double* R = g.cr_max[t];
    const double s = __dadd_rn(__dmul_rn(at(L, i, j), at(R, k, l)), __dmul_rn(at(L, k, l), at(R, i, j)));
    bound = __dadd_rn(bound, __dmul_rn(__dmul_rn(0.5, fabs(g.cf[t])), s));
  }
  for (int t = 0; t < g.nexch; ++t) {
    const double* L = g.xl_max[t];
    const double* R = g.xr_max[t];
    double s = __dadd_rn(__dmul_rn(at(L, i, k), at(R, j, l)), __dmul_rn(at(L, j, k), at(R, i, l)));
    s = __dadd_rn(s, __dmul_rn(at(L, i, l), at(R, j, k)));
    s = __dadd_rn(s, __dmul_rn(at(L, j, l), at(R, i, k)));
    bound = __dadd_rn(bound, __dmul_rn(__dmul_rn(0.25, fabs(g.xf[t])), s));
  }
  return bound;
}

// Reference screening of one canonical quartet.  The reference bra is the
// pair with the larger canonical index (its loops run k <= i, l <= l_top,
// src/direct.rs:169-190); the Schwarz product Q_ij*Q_kl and the density
// mask max(|D| over the six blocks) are evaluated in that orientation so the
// accepted list is the reference's, bit for bit.
__device__ __forceinline__ Screen screen_quartet(const KernelArgs& A, const PairD& pb, const PairD& pk) {
  Screen s;
  s.swapped = pk.tri > pb.tri;
  const PairD& rb = s.swapped ? pk : pb;
  const PairD& rk = s.swapped ? pb : pk;
  s.i = rb.i;
  s.j = rb.j;
  s.k = rk.i;
  s.l = rk.j;
  s.mask = 1;
  s.keep = true;
  s.degeneracy = 1.0;
  if (A.bra_bitmap && !((__ldg(A.bra_bitmap + (rb.tri >> 5)) >> (rb.tri & 31)) & 1u)) {
    s.keep = false;
    return s;
  }
  if (A.mode == MODE_JK) {
    const double qab = rb.q;
    if (qab == 0.0) {  // direct.rs:166, unconditional
      s.keep = false;
      return s;
    }
    const double pair_bound = qab * rk.q;
    if (pair_bound < A.jk.threshold) {
      s.keep = false;
      return s;
    }
    const int n = A.nsh;
    uint64_t mask = 0;
    for (int d = 0; d < A.jk.ndens; ++d) {
      const double* bd = A.jk.bounds + (size_t)d * n * n;
      double db = fmax(fmax(fmax(fmax(fmax(__ldg(bd + (size_t)s.i * n + s.j), __ldg(bd + (size_t)s.k * n + s.l)),
                                      __ldg(bd + (size_t)s.i * n + s.k)),
                                 __ldg(bd + (size_t)s.i * n + s.l)),
                            __ldg(bd + (size_t)s.j * n + s.k)),
                       __ldg(bd + (size_t)s.j * n + s.l));
      if (pair_bound * db >= A.jk.threshold) mask |= 1ull << d;
    }
    s.mask = mask;
    s.keep = mask != 0;
  } else if (A.mode == MODE_GRAD) {
    // src/direct_grad.rs:347-370
    const double thr = A.grad.threshold;
    const double qab = rb.q;
    if (qab == 0.0 && thr > 0.0) {
      s.keep = false;
      return s;
    }
    const int ai = A.shells[s.i].atom, aj = A.shells[s.j].atom, ak = A.shells[s.k].atom, al = A.shells[s.l].atom;
    if (ai == aj && aj == ak && ak == al) {
      s.keep = false;
      return s;
    }
    const double pair_bound = qab * rk.q;
    if (pair_bound < thr) {
      s.keep = false;
      return s;
    }
    const double deg = (s.i == s.j ? 1.0 : 2.0) * (s.k == s.l ? 1.0 : 2.0) * (s.i == s.k && s.j == s.l ? 1.0 : 2.0);
    s.degeneracy = deg;
    if (__dmul_rn(__dmul_rn(pair_bound, deg), grad_block_bound(A.grad, A.nsh, s.i, s.j, s.k, s.l)) < thr)
      s.keep = false;
  }
  return s;
}

struct QuartetCounters {
  unsigned long long quartets = 0, hash = 0, fp32 = 0, prims = 0;
  __device__ __forceinline__ void add(const Screen& s, const PairD& pb, const PairD& pk, int fp32flag) {
    quartets += 1;
    hash += quartet_key(s.i, s.j, s.k, s.l, s.mask);
    if (fp32flag) fp32 += 1;
    prims += (unsigned long long)pb.nprim * (unsigned long long)pk.nprim;
  }
  __device__ __forceinline__ void flush(Counters* c) {
    unsigned long long q = warp_sum_u64(quartets), h = warp_sum_u64(hash), f = warp_sum_u64(fp32),
                       p = warp_sum_u64(prims);
    if ((threadIdx.x & 31) == 0 && c) {
      if (q) atomicAdd(&c->quartets, q);
      if (h) atomicAdd(&c->hash, h);
      if (f) atomicAdd(&c->fp32_quartets, f);
      if (p) atomicAdd(&c->prim_quartets, p);
    }
  }
};

// ------------------------------------------------------- horizontal recurrences

// Bra HRR (a, b+1_i | f) = (a+1_i, b | f) + AB_i (a, b | f), i = first
// nonzero axis of b (src/engine/os_eri.rs:3083-3116), level by level over the
// whole table; returns the buffer that holds [b][a][f] with a of degree la.
template <typename V>
__device__ __forceinline__ V* hrr_bra(V* buf[3], int& cur, int la, int lb, int nfp, const double ab[3], int lane,
                                      int T, unsigned tmask) {
  const int ne = la + lb;
  const int base_a = tri_below(la);
  for (int kb = 1; kb <= lb; ++kb) {
    const V* src = buf[cur];
    V* dst = buf[(cur + 1) % 3];
    const int nb_k = ncart(kb);
    const int na_k = nrange(la, ne - kb);
    const int na_p = nrange(la, ne - kb + 1);
    const int total = nb_k * na_k * nfp;
    for (int q = lane; q < total; q += T) {
      const int f = q % nfp;
      const int r = q / nfp;
      const int ia = r % na_k;
      const int ib = r / na_k;
      // b: component ib of degree kb
      const int baddr = tri_below(kb) + ib;
      const int bx = addr_lx(baddr), by = addr_ly(baddr), bz = addr_lz(baddr);
      const int ax_ = bx > 0 ? 0 : (by > 0 ? 1 : 2);
      const int b1x = bx - (ax_ == 0), b1y = by - (ax_ == 1), b1z = bz - (ax_ == 2);
      const int ib1 = cart_index3(b1x, b1y, b1z);
      const int aaddr = base_a + ia;
      const int ax = addr_lx(aaddr), ay = addr_ly(aaddr), az = addr_lz(aaddr);
      const int ia1 = addr3(ax + (ax_ == 0), ay + (ax_ == 1), az + (ax_ == 2)) - base_a;
      const V v1 = src[((size_t)ib1 * na_p + ia1) * nfp + f];
      const V v0 = src[((size_t)ib1 * na_p + ia) * nfp + f];
      dst[q] = v1 + (V)ab[ax_] * v0;
    }
    __syncwarp(tmask);
    cur = (cur + 1) % 3;
  }
  return buf[cur];
}

// Ket HRR per (a,b) row, then the Cartesian block [a][b][c][d].
template <typename V>
__device__ __forceinline__ void hrr_ket(V* buf[3], int hcur, V* blk, int la, int lb, int lc, int ld, int nfp,
                                        const double cd[3], int lane, int T, unsigned tmask) {
  const int na = ncart(la), nb = ncart(lb), nc = ncart(lc), nd = ncart(ld);
  const int nab = na * nb;
  const int nf = lc + ld;
  const int base_c = tri_below(lc);
  const V* H = buf[hcur];  // [ib][ia][f]
  if (ld == 0) {
    const int total = nab * nc;
    for (int q = lane; q < total; q += T) {
      const int ic = q % nc, ab = q / nc;
      const int ia = ab / nb, ib = ab % nb;
      blk[q] = H[((size_t)ib * na + ia) * nfp + ic];
    }
    __syncwarp(tmask);
    return;
  }
  int cur = -1;  // level 0 read from H
  int w0 = (hcur + 1) % 3, w1 = (hcur + 2) % 3;
  const V* src = H;
  for (int kd = 1; kd <= ld; ++kd) {
    V* dst = (kd & 1) ? buf[w0] : buf[w1];
    const int nd_k = ncart(kd);
    const int nc_k = nrange(lc, nf - kd);
    const int nc_p = nrange(lc, nf - kd + 1);
    const int total = nab * nd_k * nc_k;
    for (int q = lane; q < total; q += T) {
      const int ic = q % nc_k;
      const int r = q / nc_k;
      const int id = r % nd_k;
      const int ab = r / nd_k;
      const int daddr = tri_below(kd) + id;
      const int dx = addr_lx(daddr), dy = addr_ly(daddr), dz = addr_lz(daddr);
      const int jx = dx > 0 ? 0 : (dy > 0 ? 1 : 2);
      const int id1 = cart_index3(dx - (jx == 0), dy - (jx == 1), dz - (jx == 2));
      const int caddr = base_c + ic;
      const int cx = addr_lx(caddr), cy = addr_ly(caddr), cz = addr_lz(caddr);
      const int ic1 = addr3(cx + (jx == 0), cy + (jx == 1), cz + (jx == 2)) - base_c;
      V v1, v0;
      if (kd == 1) {
        const int ia = ab / nb, ib = ab % nb;
        const size_t row = ((size_t)ib * na + ia) * nfp;
        v1 = src[row + ic1];
        v0 = src[row + ic];
      } else {
        v1 = src[((size_t)ab * ncart(kd - 1) + id1) * nc_p + ic1];
        v0 = src[((size_t)ab * ncart(kd - 1) + id1) * nc_p + ic];
      }
      dst[q] = v1 + (V)cd[jx] * v0;
    }
    __syncwarp(tmask);
    src = dst;
    (void)cur;
  }
  // final level [ab][d][c] (c of degree lc) -> block [ab][c][d]
  const int total = nab * nc * nd;
  for (int q = lane; q < total; q += T) {
    const int id = q % nd;
    const int r = q / nd;
    const int ic = r % nc;
    const int ab = r / nc;
    blk[q] = src[((size_t)ab * nd + id) * nc + ic];
  }
  __syncwarp(tmask);
}

// Apply the per-axis c2s matrix (nfunc x ncart) of every spherical shell
// (src/spherical.rs:121-179); dims updated in place.  Returns the buffer that
// holds the function-space block.
__device__ __forceinline__ double* c2s_block(const KernelArgs& A, double* blk, double* tmp, int dims[4],
                                             const int ls[4], const int sph[4], int lane, int T,
                                             unsigned tmask) {
  double* cur = blk;
  double* oth = tmp;
  for (int axis = 0; axis < 4; ++axis) {
    if (!sph[axis]) continue;
    const int l = ls[axis];
    const int n_in = dims[axis], n_out = 2 * l + 1;
    const double* M = A.c2s + A.c2s_off[l];
    int outer = 1, inner = 1;
    for (int q = 0; q < axis; ++q) outer *= dims[q];
    for (int q = axis + 1; q < 4; ++q) inner *= dims[q];
    const int total = outer * n_out * inner;
    for (int q = lane; q < total; q += T) {
      const int s = q % inner;
      const int r = q / inner;
      const int o = r / n_out, m = r % n_out;
      double acc = 0.0;
      for (int j = 0; j < n_in; ++j) {
        const double c = __ldg(M + m * n_in + j);
        if (c != 0.0) acc += c * cur[((size_t)o * n_in + j) * inner + s];
      }
      oth[q] = acc;
    }
    __syncwarp(tmask);
    dims[axis] = n_out;
    double* t = cur;
    cur = oth;
    oth = t;
  }
  return cur;
}

// ----------------------------------------------------------------- consumers

// Shell tuples of the 8 permutations (src/integrals.rs:1235-1244) and which
// of them are distinct (the reference's dedup by permuted shell tuple).
// The densities in value type V: the FP64 matrices, or their FP32 copy for
// the FP32 launches of the mixed path.
template <typename V>
__device__ __forceinline__ const V* dens_of(const JKDev& jk) {
  if constexpr (sizeof(V) == 4)
    return jk.Df;
  else
    return jk.D;
}

__device__ __forceinline__ unsigned distinct_perms(const int s[4]) {
  const int P[8][4] = {{0, 1, 2, 3}, {1, 0, 2, 3}, {0, 1, 3, 2}, {1, 0, 3, 2},
                       {2, 3, 0, 1}, {2, 3, 1, 0}, {3, 2, 0, 1}, {3, 2, 1, 0}};
  unsigned w = 0;
  for (int p = 0; p < 8; ++p) {
    bool dup = false;
    for (int q = 0; q < p; ++q)
      if ((w >> q) & 1u)
        if (s[P[p][0]] == s[P[q][0]] && s[P[p][1]] == s[P[q][1]] && s[P[p][2]] == s[P[q][2]] &&
            s[P[p][3]] == s[P[q][3]])
          dup = true;
    if (!dup) w |= 1u << p;
  }
  return w;
}

// One contraction term: for every (iu, iv) on axes (u, v) of the block,
// val = sum over axes (s, t) of B * Dm[row axis ds][col axis dt]; then
// T1[u-row][v-col] += w1*val and T2[v-row][u-col] += w2*val.
__device__ __forceinline__ void jk_term(const double* B, const int dims[4], const int offs[4], int nao, int u, int v,
                                        int s, int t, const double* Dm, int ds, int dt, double* T1, double w1,
                                        double* T2, double w2, int lane, int T) {
  const int st[4] = {dims[1] * dims[2] * dims[3], dims[2] * dims[3], dims[3], 1};
  const int nu = dims[u], nv = dims[v], ns = dims[s], nt = dims[t];
  for (int q = lane; q < nu * nv; q += T) {
    const int iu = q / nv, iv = q % nv;
    const size_t bb = (size_t)iu * st[u] + (size_t)iv * st[v];
    double acc = 0.0;
    for (int is = 0; is < ns; ++is) {
      for (int it = 0; it < nt; ++it) {
        const int ids = ds == s ? is : it;
        const int idt = dt == s ? is : it;
        const double dv = __ldg(Dm + (size_t)(offs[ds] + ids) * nao + offs[dt] + idt);
        acc += B[bb + (size_t)is * st[s] + (size_t)it * st[t]] * dv;
      }
    }
    if (w1 != 0.0) atomicAdd(T1 + (size_t)(offs[u] + iu) * nao + offs[v] + iv, w1 * acc);
    if (w2 != 0.0) atomicAdd(T2 + (size_t)(offs[v] + iv) * nao + offs[u] + iu, w2 * acc);
  }
}

// Atomically add a team's running bra-block accumulators to J' and clear
// them.  acc layout: [0] = evaluation bra pair index (or -1), then
// ndens blocks of n_func(A) x n_func(B).
__device__ __forceinline__ void flush_bra_acc(const KernelArgs& A, double* acc, int lane, int T, unsigned tmask) {
  const int bra = (int)acc[0];
  if (bra >= 0) {
    const PairD pb = A.pairs[bra];
    const DevShell sa = A.shells[pb.a], sb = A.shells[pb.b];
    const int nab = sa.nfunc * sb.nfunc;
    const size_t n2 = (size_t)A.nao * A.nao;
    for (int d = 0; d < A.jk.ndens; ++d) {
      double* a = acc + 1 + (size_t)d * nab;
      for (int q = lane; q < nab; q += T) {
        const double v = a[q];
        if (v != 0.0) {
          const int ia = q / sb.nfunc, ib = q % sb.nfunc;
          atomicAdd(A.jk.J + d * n2 + (size_t)(sa.off + ia) * A.nao + sb.off + ib, v);
          a[q] = 0.0;
        }
      }
    }
  }
  __syncwarp(tmask);
  if (lane == 0) acc[0] = -1.0;
  __syncwarp(tmask);
}

// Symmetric densities: one orientation of every image, the six
// contractions
//   t0 J'[A a][B b] += w0 sum_cd B D[C c][D d]   (running bra accumulator)
//   t1 J'[C c][D d] += w1 sum_ab B D[A a][B b]
//   t2 K'[A a][C c] += w2 sum_bd B D[B b][D d]   t3 K'[B b][C c] += w3 sum_ad B D[A a][D d]
//   t4 K'[A a][D d] += w4 sum_bc B D[B b][C c]   t5 K'[B b][D d] += w5 sum_ac B D[A a][C c]
// with the summed weights of the permutation images landing on each block
// or its transpose.  All output elements of all six terms form one list
// spread over the team's lanes; each lane sums its elements for up to DCH
// densities at once (densities d0 + k with bit k of m set), so every block
// element read feeds up to DCH products.
constexpr int JK_DCH = 4;

template <int DCH>
__device__ __forceinline__ void jk_sym_chunk(const KernelArgs& A, const double* B, const int dims[4],
                                             const int offs[4], const double wt[6], int nterm, int d0, unsigned m,
                                             double* acc, int lane, int T) {
  // (u, v) output axes and (s, t) summed axes of term t, one nibble per term
  // (no dynamically indexed local arrays); D block rows on s, columns on t
  constexpr unsigned PU = 0x101020u, PV = 0x332231u, PS = 0x010102u, PT = 0x223313u;
  const int st0 = dims[1] * dims[2] * dims[3], st1 = dims[2] * dims[3], st2 = dims[3];
  auto stride = [&](int ax) { return ax == 0 ? st0 : (ax == 1 ? st1 : (ax == 2 ? st2 : 1)); };
  auto dim = [&](int ax) { return ax == 0 ? dims[0] : (ax == 1 ? dims[1] : (ax == 2 ? dims[2] : dims[3])); };
  auto off = [&](int ax) { return ax == 0 ? offs[0] : (ax == 1 ? offs[1] : (ax == 2 ? offs[2] : offs[3])); };
  auto nib = [](unsigned p, int t) { return (int)((p >> (4 * t)) & 0xFu); };
  const int nab = dims[0] * dims[1];
  const int nao = A.nao;
  const size_t n2 = (size_t)nao * nao;
  auto len = [&](int t) { return (t < nterm && wt[t] != 0.0) ? dim(nib(PU, t)) * dim(nib(PV, t)) : 0; };
  const int e1 = len(0), e2 = e1 + len(1), e3 = e2 + len(2), e4 = e3 + len(3), e5 = e4 + len(4), e6 = e5 + len(5);
  for (int q = lane; q < e6; q += T) {
    const int t = q < e1 ? 0 : (q < e2 ? 1 : (q < e3 ? 2 : (q < e4 ? 3 : (q < e5 ? 4 : 5))));
    const int base = t == 0 ? 0 : (t == 1 ? e1 : (t == 2 ? e2 : (t == 3 ? e3 : (t == 4 ? e4 : e5))));
    const double w = t == 0 ? wt[0] : (t == 1 ? wt[1] : (t == 2 ? wt[2] : (t == 3 ? wt[3] : (t == 4 ? wt[4] : wt[5]))));
    const int u = nib(PU, t), v = nib(PV, t), s = nib(PS, t), tt = nib(PT, t);
    const int r = q - base;
    const int nv = dim(v);
    const int iu = r / nv, iv = r - iu * nv;
    const int ns = dim(s), nt = dim(tt);
    const double* Bp = B + (size_t)iu * stride(u) + (size_t)iv * stride(v);
    const int ss = stride(s), stt = stride(tt);
    const double* Dp = A.jk.D + (size_t)d0 * n2 + (size_t)off(s) * nao + off(tt);
    double sum[DCH];
#pragma unroll
    for (int k = 0; k < DCH; ++k) sum[k] = 0.0;
    for (int is = 0; is < ns; ++is) {
      const double* br = Bp + (size_t)is * ss;
      const double* dr = Dp + (size_t)is * nao;
      for (int it = 0; it < nt; ++it) {
        const double b = br[(size_t)it * stt];
#pragma unroll
        for (int k = 0; k < DCH; ++k)
          if ((m >> k) & 1u) sum[k] += b * __ldg(dr + (size_t)k * n2 + it);
      }
    }
    if (t == 0) {
#pragma unroll
      for (int k = 0; k < DCH; ++k)
        if ((m >> k) & 1u) acc[1 + (size_t)(d0 + k) * nab + r] += w * sum[k];
    } else {
      double* out = t == 1 ? A.jk.J : A.jk.K;
      const size_t o = (size_t)(off(u) + iu) * nao + off(v) + iv;
#pragma unroll
      for (int k = 0; k < DCH; ++k)
        if ((m >> k) & 1u) atomicAdd(out + (size_t)(d0 + k) * n2 + o, w * sum[k]);
    }
  }
}

// Shared memory a team needs for its copy of the Cartesian block la..ld.
__host__ __device__ constexpr int jk_stage_doubles(int la, int lb, int lc, int ld) {
  return ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
}

__device__ __forceinline__ void consume_jk(const KernelArgs& A, const double* B, const int dims[4],
                                           const int offs[4], const int sh[4], uint64_t mask, int lane, int T,
                                           double* acc, int pbi, unsigned tmask, double* stage) {
  const unsigned w = distinct_perms(sh);
  auto W = [&](int p) { return (double)((w >> p) & 1u); };
  const int nao = A.nao;
  const size_t n2 = (size_t)nao * nao;
  if (A.jk.symmetric) {
    if ((int)acc[0] != pbi) {
      flush_bra_acc(A, acc, lane, T, tmask);
      if (lane == 0) acc[0] = (double)pbi;
      __syncwarp(tmask);
    }
    const double wt[6] = {W(0) + W(1) + W(2) + W(3), W(4) + W(5) + W(6) + W(7), W(0) + W(4),
                          W(1) + W(5),               W(2) + W(6),               W(3) + W(7)};
    const int nterm = A.jk.want_k ? 6 : 2;
    // the sums read the block with lane-dependent strides: work from a
    // shared-memory copy (one coalesced pass) when the team has one
    const double* Bs = B;
    if (stage) {
      const int nblk = dims[0] * dims[1] * dims[2] * dims[3];
      for (int q = lane; q < nblk; q += T) stage[q] = B[q];
      __syncwarp(tmask);
      Bs = stage;
    }
    const unsigned long long live = A.jk.ndens >= 64 ? ~0ull : ((1ull << A.jk.ndens) - 1ull);
    for (int d0 = 0; d0 < A.jk.ndens; d0 += JK_DCH) {
      const unsigned m = (unsigned)(((mask & live) >> d0) & ((1u << JK_DCH) - 1u));
      if (m) jk_sym_chunk<JK_DCH>(A, Bs, dims, offs, wt, nterm, d0, m, acc, lane, T);
    }
    __syncwarp(tmask);
    return;
  }
  for (int d = 0; d < A.jk.ndens; ++d) {
    if (!((mask >> d) & 1ull)) continue;
    const double* Dm = A.jk.D + d * n2;
    double* J = A.jk.J + d * n2;
    double* K = A.jk.want_k ? A.jk.K + d * n2 : nullptr;
    {
      // P0..P3 J on (A,B); P4..P7 J on (C,D)
      jk_term(B, dims, offs, nao, 0, 1, 2, 3, Dm, 2, 3, J, W(0), J, W(1), lane, T);
      jk_term(B, dims, offs, nao, 0, 1, 2, 3, Dm, 3, 2, J, W(2), J, W(3), lane, T);
      jk_term(B, dims, offs, nao, 2, 3, 0, 1, Dm, 0, 1, J, W(4), J, W(6), lane, T);
      jk_term(B, dims, offs, nao, 2, 3, 0, 1, Dm, 1, 0, J, W(5), J, W(7), lane, T);
      if (K) {
        jk_term(B, dims, offs, nao, 0, 2, 1, 3, Dm, 1, 3, K, W(0), K, 0.0, lane, T);
        jk_term(B, dims, offs, nao, 0, 2, 1, 3, Dm, 3, 1, K, 0.0, K, W(4), lane, T);
        jk_term(B, dims, offs, nao, 1, 2, 0, 3, Dm, 0, 3, K, W(1), K, 0.0, lane, T);
        jk_term(B, dims, offs, nao, 1, 2, 0, 3, Dm, 3, 0, K, 0.0, K, W(5), lane, T);
        jk_term(B, dims, offs, nao, 0, 3, 1, 2, Dm, 1, 2, K, W(2), K, 0.0, lane, T);
        jk_term(B, dims, offs, nao, 0, 3, 1, 2, Dm, 2, 1, K, 0.0, K, W(6), lane, T);
        jk_term(B, dims, offs, nao, 1, 3, 0, 2, Dm, 0, 2, K, W(3), K, 0.0, lane, T);
        jk_term(B, dims, offs, nao, 1, 3, 0, 2, Dm, 2, 0, K, 0.0, K, W(7), lane, T);
      }
    }
  }
}

// Dense tensor: every distinct permutation slot of the block, written once
// (src/integrals.rs:1271-1312).
__device__ __forceinline__ void consume_dense(const KernelArgs& A, const double* B, const int dims[4],
                                              const int offs[4], const int sh[4], int lane, int T) {
  const int P[8][4] = {{0, 1, 2, 3}, {1, 0, 2, 3}, {0, 1, 3, 2}, {1, 0, 3, 2},
                       {2, 3, 0, 1}, {2, 3, 1, 0}, {3, 2, 0, 1}, {3, 2, 1, 0}};
  const unsigned w = distinct_perms(sh);
  const size_t n = (size_t)A.nao;
  const int total = dims[0] * dims[1] * dims[2] * dims[3];
  for (int q = lane; q < total; q += T) {
    int idx[4];
    idx[3] = q % dims[3];
    int r = q / dims[3];
    idx[2] = r % dims[2];
    r /= dims[2];
    idx[1] = r % dims[1];
    idx[0] = r / dims[1];
    size_t X[4];
    for (int a = 0; a < 4; ++a) X[a] = (size_t)(offs[a] + idx[a]);
    const double v = B[q];
    for (int p = 0; p < 8; ++p) {
      if (!((w >> p) & 1u)) continue;
      A.dense[((X[P[p][0]] * n + X[P[p][1]]) * n + X[P[p][2]]) * n + X[P[p][3]]] = v;
    }
  }
}

// EriBuilder fill: the four bra/ket-internal slots of the requested bra pair
// (src/eri_builder.rs:650-690).  `bra_is_eval_ket` tells which evaluation
// pair is the requested bra.
__device__ __forceinline__ void consume_builder(const KernelArgs& A, const double* B, const int dims[4],
                                                const int offs[4], const int sh[4], bool bra_is_eval_ket,
                                                int lane, int T) {
  const size_t n = (size_t)A.nao;
  const int total = dims[0] * dims[1] * dims[2] * dims[3];
  const int r0 = bra_is_eval_ket ? 2 : 0, r1 = bra_is_eval_ket ? 3 : 1;
  const int c0 = bra_is_eval_ket ? 0 : 2, c1 = bra_is_eval_ket ? 1 : 3;
  const bool bra_same = sh[r0] == sh[r1];
  const bool ket_same = sh[c0] == sh[c1];
  for (int q = lane; q < total; q += T) {
    int idx[4];
    idx[3] = q % dims[3];
    int r = q / dims[3];
    idx[2] = r % dims[2];
    r /= dims[2];
    idx[1] = r % dims[1];
    idx[0] = r / dims[1];
    size_t X[4];
    for (int a = 0; a < 4; ++a) X[a] = (size_t)(offs[a] + idx[a]);
    const double v = B[q];
    const size_t mu = X[r0], nu = X[r1], la = X[c0], sg = X[c1];
    A.dense[((mu * n + nu) * n + la) * n + sg] = v;
    if (!bra_same) A.dense[((nu * n + mu) * n + la) * n + sg] = v;
    if (!ket_same) A.dense[((mu * n + nu) * n + sg) * n + la] = v;
    if (!bra_same && !ket_same) A.dense[((nu * n + mu) * n + sg) * n + la] = v;
  }
}

// Packed symmetry-unique tensor (src/packed_eri.rs:10-21, 297-327): AO pairs
// numbered shell-pair blocked (canonical shell pair, then (a, b) row-major
// with b <= a when i == j), element (t|u), u <= t, at t(t+1)/2 + u.  The block
// is taken in the reference orientation (i,j|k,l) of the canonical quartet,
// bra = the pair with the larger canonical index; every unique element is
// written once.
__device__ __forceinline__ void consume_packed(const KernelArgs& A, const double* B, const int dims[4],
                                               const PairD& pb, const PairD& pk, const Screen& sc, int lane, int T) {
  const PairD& rb = sc.swapped ? pk : pb;
  const PairD& rk = sc.swapped ? pb : pk;
  // evaluation slot of reference positions i, j, k, l
  const bool bflip = pb.a != pb.i, kflip = pk.a != pk.i;
  const int e0 = !sc.swapped ? (bflip ? 1 : 0) : (kflip ? 3 : 2);
  const int e1 = !sc.swapped ? (bflip ? 0 : 1) : (kflip ? 2 : 3);
  const int e2 = !sc.swapped ? (kflip ? 3 : 2) : (bflip ? 1 : 0);
  const int e3 = !sc.swapped ? (kflip ? 2 : 3) : (bflip ? 0 : 1);
  auto pick = [](int e, int x0, int x1, int x2, int x3) { return e == 0 ? x0 : (e == 1 ? x1 : (e == 2 ? x2 : x3)); };
  const int nj = pick(e1, dims[0], dims[1], dims[2], dims[3]);
  const int nl = pick(e3, dims[0], dims[1], dims[2], dims[3]);
  const bool bra_diag = rb.i == rb.j, ket_diag = rk.i == rk.j, same = rb.tri == rk.tri;
  const long long t0 = A.packed_start[rb.tri], u0 = A.packed_start[rk.tri];
  const int total = dims[0] * dims[1] * dims[2] * dims[3];
  for (int q = lane; q < total; q += T) {
    const int f3 = q % dims[3], f2 = (q / dims[3]) % dims[2], f1 = (q / (dims[3] * dims[2])) % dims[1],
              f0 = q / (dims[3] * dims[2] * dims[1]);
    const int a = pick(e0, f0, f1, f2, f3), b = pick(e1, f0, f1, f2, f3);
    const int c = pick(e2, f0, f1, f2, f3), d = pick(e3, f0, f1, f2, f3);
    if (bra_diag && b > a) continue;
    if (ket_diag && d > c) continue;
    const long long t = t0 + (bra_diag ? (long long)a * (a + 1) / 2 + b : (long long)a * nj + b);
    const long long u = u0 + (ket_diag ? (long long)c * (c + 1) / 2 + d : (long long)c * nl + d);
    if (same && u > t) continue;
    A.dense[(size_t)t * (size_t)(t + 1) / 2 + (size_t)u] = B[q];
  }
}

// Store of the density-fitting and block writers: an index outside the
// output raises the launch's fault flag instead of writing.
__device__ __forceinline__ void df_store(const KernelArgs& A, size_t at, double v) {
  if (at < A.dense_len)
    A.dense[at] = v;
  else
    atomicOr(A.store_fault, 1u);
}

// Unpacks block position q of a row-major [dims0][dims1][dims2][dims3] block.
__device__ __forceinline__ void block_index(int q, const int dims[4], int idx[4]) {
  idx[3] = q % dims[3];
  int r = q / dims[3];
  idx[2] = r % dims[2];
  r /= dims[2];
  idx[1] = r % dims[1];
  idx[0] = r / dims[1];
}

// Three-centre tensor (Eri3cBuilder::fill, src/df.rs:463-513): the block is
// (main pair | aux shell, unit s), or (aux shell, unit s | main pair) when
// the aux class is the larger one.  Element (mu nu|P) goes to
// out[(mu*nao + nu)*naux + P] and, for two distinct main shells, to
// (nu mu|P) as well: the (i, j) and (j, i) bands of the reference.
__device__ __forceinline__ void consume_df3(const KernelArgs& A, const double* B, const int dims[4],
                                            const int offs[4], const int sh[4], bool aux_is_bra, int lane,
                                            int T) {
  const int m0 = aux_is_bra ? 2 : 0, m1 = aux_is_bra ? 3 : 1, pp = aux_is_bra ? 0 : 2;
  const bool same = sh[m0] == sh[m1];
  const size_t n = (size_t)A.nao, na = (size_t)A.naux;
  const int total = dims[0] * dims[1] * dims[2] * dims[3];
  for (int q = lane; q < total; q += T) {
    int idx[4];
    block_index(q, dims, idx);
    const size_t mu = (size_t)(offs[m0] + idx[m0]), nu = (size_t)(offs[m1] + idx[m1]);
    const size_t P = (size_t)(offs[pp] + idx[pp]);
    const double v = B[q];
    df_store(A, (mu * n + nu) * na + P, v);
    if (!same) df_store(A, (nu * n + mu) * na + P, v);
  }
}

// Two-centre metric (Basis::eri_2c, src/df.rs:56-93): the block is
// (aux shell P, unit s | aux shell Q, unit s); (P|Q) and (Q|P) receive the
// same value.  On a diagonal shell block only the elements with bra index
// >= ket index are taken, the values the reference's mirrored writes leave,
// so the matrix is exactly symmetric.
__device__ __forceinline__ void consume_df2(const KernelArgs& A, const double* B, const int dims[4],
                                            const int offs[4], const int sh[4], int lane, int T) {
  const bool same = sh[0] == sh[2];
  const size_t na = (size_t)A.naux;
  const int total = dims[0] * dims[1] * dims[2] * dims[3];
  for (int q = lane; q < total; q += T) {
    int idx[4];
    block_index(q, dims, idx);
    if (same && idx[2] > idx[0]) continue;
    const size_t P = (size_t)(offs[0] + idx[0]), Q = (size_t)(offs[2] + idx[2]);
    const double v = B[q];
    df_store(A, P * na + Q, v);
    df_store(A, Q * na + P, v);
  }
}

// One shell-quartet block (Basis::eri_block, src/integrals.rs:600-640): the
// evaluated quartet is one of the 8 permutations of the requested
// (i, j, k, l).  The first permutation whose shells match maps every
// evaluated element to the requested row-major [n_i][n_j][n_k][n_l] block.
__device__ __forceinline__ void consume_block(const KernelArgs& A, const double* B, const int dims[4],
                                              const int sh[4], int lane, int T) {
  // P8[p][r]: evaluation slot of requested position r under permutation p
  const int P8[8][4] = {{0, 1, 2, 3}, {1, 0, 2, 3}, {0, 1, 3, 2}, {1, 0, 3, 2},
                        {2, 3, 0, 1}, {3, 2, 0, 1}, {2, 3, 1, 0}, {3, 2, 1, 0}};
  int pick = -1;
  for (int p = 0; p < 8 && pick < 0; ++p)
    if (sh[P8[p][0]] == A.blk_shells[0] && sh[P8[p][1]] == A.blk_shells[1] && sh[P8[p][2]] == A.blk_shells[2] &&
        sh[P8[p][3]] == A.blk_shells[3])
      pick = p;
  if (pick < 0) {
    if (lane == 0) atomicOr(A.store_fault, 2u);
    return;
  }
  const int* m = P8[pick];
  const int total = dims[0] * dims[1] * dims[2] * dims[3];
  for (int q = lane; q < total; q += T) {
    int idx[4];
    block_index(q, dims, idx);
    const size_t at =
        (((size_t)idx[m[0]] * A.blk_dims[1] + idx[m[1]]) * A.blk_dims[2] + idx[m[2]]) * A.blk_dims[3] + idx[m[3]];
    df_store(A, at, B[q]);
  }
}

// Schwarz: sqrt(max |(mu nu|mu nu)|) over the function-space diagonal of the
// (ij|ij) block (src/integrals.rs:850-860).
__device__ __forceinline__ void consume_schwarz(const KernelArgs& A, const double* B, const int dims[4],
                                                int pair_index, int lane, int T, unsigned tmask) {
  const int ni = dims[0], nj = dims[1];
  double mx = 0.0;
  for (int q = lane; q < ni * nj; q += T) {
    const int mu = q / nj, nu = q % nj;
    mx = fmax(mx, fabs(B[(((size_t)mu * nj + nu) * ni + mu) * nj + nu]));
  }
  for (int o = T / 2; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(tmask, mx, o, T));
  if (lane == 0) A.schwarz_out[pair_index] = sqrt(mx);
}

// Post phase of one quartet: G (in slot) -> Cartesian block -> function
// block -> consumer.
__device__ __forceinline__ void post_quartet(const KernelArgs& A, const ClassDims& cd_, const PairD& pb,
                                             const PairD& pk, const Screen& sc, double* slot, int lane, int T,
                                             unsigned tmask, int pb_index, double* stage) {
  const int la = cd_.la, lb = cd_.lb, lc = cd_.lc, ld = cd_.ld;
  const SlotLayout L = slot_layout(la, lb, lc, ld);
  double* buf[3] = {slot, slot + L.S, slot + 2 * L.S};
  double* blk = slot + 3 * L.S;
  double* tmp = blk + L.blk;
  const int nfp = nrange(lc, lc + ld);
  const double ab[3] = {pb.abx, pb.aby, pb.abz};
  const double cdv[3] = {pk.abx, pk.aby, pk.abz};
  int cur = 0;
  hrr_bra(buf, cur, la, lb, nfp, ab, lane, T, tmask);
  hrr_ket(buf, cur, blk, la, lb, lc, ld, nfp, cdv, lane, T, tmask);
  const int shl[4] = {pb.a, pb.b, pk.a, pk.b};
  const DevShell s0 = A.shells[shl[0]], s1 = A.shells[shl[1]], s2 = A.shells[shl[2]], s3 = A.shells[shl[3]];
  int dims[4] = {ncart(la), ncart(lb), ncart(lc), ncart(ld)};
  const int ls[4] = {la, lb, lc, ld};
  const int sph[4] = {s0.spherical, s1.spherical, s2.spherical, s3.spherical};
  const double* B = c2s_block(A, blk, tmp, dims, ls, sph, lane, T, tmask);
  const int offs[4] = {s0.off, s1.off, s2.off, s3.off};
  switch (A.mode) {
    case MODE_JK:
      consume_jk(A, B, dims, offs, shl, sc.mask, lane, T, slot + A.acc_offset, pb_index, tmask, stage);
      break;
    case MODE_DENSE:
      consume_dense(A, B, dims, offs, shl, lane, T);
      break;
    case MODE_BUILDER:
      consume_builder(A, B, dims, offs, shl, A.builder_swap != 0, lane, T);
      break;
    case MODE_PACKED:
      consume_packed(A, B, dims, pb, pk, sc, lane, T);
      break;
    case MODE_SCHWARZ:
      consume_schwarz(A, B, dims, pb_index, lane, T, tmask);
      break;
    case MODE_DF3:
      consume_df3(A, B, dims, offs, shl, pb.j < 0, lane, T);
      break;
    case MODE_DF2:
      consume_df2(A, B, dims, offs, shl, lane, T);
      break;
    case MODE_BLOCK:
      consume_block(A, B, dims, shl, lane, T);
      break;
    default:
      break;
  }
}

// ----------------------------------------- J/K post phase, Cartesian classes

// One contraction term of the symmetric J/K images with the block shape
// known at compile time: output (u, v), summed (s, t), D block rows on s and
// columns on t.  Every sum is fully unrolled, so its block and density loads
// are independent and in flight together.
template <int U, int V, int S, int TT, int N0, int N1, int N2, int N3, int T, bool ACC, typename X>
__device__ __forceinline__ void jk_term_ct(const KernelArgs& A, const X* B, const int offs[4], X w, int d0, unsigned m,
                                           double* out, int lane) {
  constexpr int N[4] = {N0, N1, N2, N3};
  constexpr int ST[4] = {N1 * N2 * N3, N2 * N3, N3, 1};
  constexpr int NU = N[U], NV = N[V], NS = N[S], NT = N[TT];
  constexpr int DCH = JK_DCH;
  const int nao = A.nao;
  const size_t n2 = (size_t)nao * nao;
  const X* Dp = dens_of<X>(A.jk) + (size_t)d0 * n2 + (size_t)offs[S] * nao + offs[TT];
  for (int r = lane; r < NU * NV; r += T) {
    const int iu = r / NV, iv = r - (r / NV) * NV;
    const X* Bp = B + iu * ST[U] + iv * ST[V];
    X sum[DCH];
#pragma unroll
    for (int k = 0; k < DCH; ++k) sum[k] = X(0);
#pragma unroll
    for (int is = 0; is < NS; ++is)
#pragma unroll
      for (int it = 0; it < NT; ++it) {
        const X b = Bp[is * ST[S] + it * ST[TT]];
#pragma unroll
        for (int k = 0; k < DCH; ++k)
          if ((m >> k) & 1u) sum[k] += b * __ldg(Dp + k * n2 + (size_t)is * nao + it);
      }
    if (ACC) {
#pragma unroll
      for (int k = 0; k < DCH; ++k)
        if ((m >> k) & 1u) out[1 + (size_t)(d0 + k) * (N0 * N1) + r] += (double)(w * sum[k]);
    } else {
      const size_t o = (size_t)(offs[U] + iu) * nao + offs[V] + iv;
#pragma unroll
      for (int k = 0; k < DCH; ++k)
        if ((m >> k) & 1u) atomicAdd(out + (size_t)(d0 + k) * n2 + o, (double)(w * sum[k]));
    }
  }
}

// Index tables of the team horizontal recurrences of one class, built once
// per block in shared memory: one entry per element of a bra level (b, a) or
// a ket level (d, c), packing the two source rows of the recurrence (bits
// 0-10 and 11-21, within the previous level), its axis (22-23) and, on the
// last ket level, the element's place in the [c][d] block row (24-31).  The
// loops then spend a shared-memory load per element instead of the
// component arithmetic.
template <int LA, int LB, int LC, int LD>
struct HrrTab {
  static constexpr int NE = LA + LB, NF = LC + LD;
  static __host__ __device__ constexpr int bra_off(int kb) {
    int o = 0;
    for (int k = 1; k < kb; ++k) o += ncart(k) * nrange(LA, NE - k);
    return o;
  }
  static __host__ __device__ constexpr int ket_off(int kd) {
    int o = bra_off(LB + 1);
    for (int k = 1; k < kd; ++k) o += ncart(k) * nrange(LC, NF - k);
    return o;
  }
  static constexpr int TOTAL = ket_off(LD + 1) > 0 ? ket_off(LD + 1) : 1;
};

template <int LA, int LB, int LC, int LD>
__device__ __forceinline__ void build_hrr_tab(int* tab) {
  using H = HrrTab<LA, LB, LC, LD>;
  constexpr int NE = H::NE, NF = H::NF;
  for (int t = threadIdx.x; t < H::TOTAL; t += blockDim.x) {
    if (t >= H::ket_off(LD + 1)) break;
    int v = 0;
    if (t < H::bra_off(LB + 1)) {
      int kb = 1;
      while (t >= H::bra_off(kb + 1)) ++kb;
      const int el = t - H::bra_off(kb);
      const int nak = nrange(LA, NE - kb), nap = nrange(LA, NE - kb + 1);
      const int ib = el / nak, ia = el % nak;
      const int baddr = tri_below(kb) + ib;
      const int bx = addr_lx(baddr), by = addr_ly(baddr), bz = addr_lz(baddr);
      const int ax = bx > 0 ? 0 : (by > 0 ? 1 : 2);
      const int ib1 = cart_index3(bx - (ax == 0), by - (ax == 1), bz - (ax == 2));
      const int aaddr = tri_below(LA) + ia;
      const int px = addr_lx(aaddr), py = addr_ly(aaddr), pz = addr_lz(aaddr);
      const int ia1 = addr3(px + (ax == 0), py + (ax == 1), pz + (ax == 2)) - tri_below(LA);
      v = (ib1 * nap + ia1) | ((ib1 * nap + ia) << 11) | (ax << 22);
    } else {
      int kd = 1;
      while (t >= H::ket_off(kd + 1)) ++kd;
      const int el = t - H::ket_off(kd);
      const int nck = nrange(LC, NF - kd), ncp = nrange(LC, NF - kd + 1);
      const int id = el / nck, ic = el % nck;
      const int daddr = tri_below(kd) + id;
      const int dx = addr_lx(daddr), dy = addr_ly(daddr), dz = addr_lz(daddr);
      const int jx = dx > 0 ? 0 : (dy > 0 ? 1 : 2);
      const int id1 = cart_index3(dx - (jx == 0), dy - (jx == 1), dz - (jx == 2));
      const int caddr = tri_below(LC) + ic;
      const int cx = addr_lx(caddr), cy = addr_ly(caddr), cz = addr_lz(caddr);
      const int ic1 = addr3(cx + (jx == 0), cy + (jx == 1), cz + (jx == 2)) - tri_below(LC);
      const int dpos = ic * ncart(LD) + id;  // place in the block row (last level)
      v = (id1 * ncp + ic1) | ((id1 * ncp + ic) << 11) | (jx << 22) | (dpos << 24);
    }
    tab[t] = v;
  }
}

template <typename X>
__device__ __forceinline__ X pick_axis(int ax, const X v[3]) {
  return ax == 0 ? v[0] : (ax == 1 ? v[1] : v[2]);
}

// The horizontal recurrences of one quartet on a team, table driven (same
// recurrences and order as hrr_bra / hrr_ket): the [e0|f0] table in buf[0]
// ([e][f]) becomes the Cartesian block [a][b][c][d] in `out`.
template <int LA, int LB, int LC, int LD, int T, typename X>
__device__ __forceinline__ void team_hrr(X* buf[3], const int* tab, X* out, const double ab[3], const double cd[3],
                                         int lane, unsigned tmask) {
  using H = HrrTab<LA, LB, LC, LD>;
  constexpr int NE = H::NE, NF = H::NF;
  constexpr int NFP = nrange(LC, NF);
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  constexpr int NAB = NA * NB;
  const X abv[3] = {(X)ab[0], (X)ab[1], (X)ab[2]};
  const X cdv[3] = {(X)cd[0], (X)cd[1], (X)cd[2]};
  int cur = 0;
  static_for<LB>([&](auto k_) {
    constexpr int KB = decltype(k_)::value + 1;
    constexpr int N = ncart(KB) * nrange(LA, NE - KB) * NFP;
    constexpr int OFF = H::bra_off(KB);
    const X* src = buf[cur];
    X* dst = buf[(cur + 1) % 3];
    for (int q = lane; q < N; q += T) {
      const int row = q / NFP, f = q - row * NFP;
      const int e = tab[OFF + row];
      dst[q] = src[(e & 0x7ff) * NFP + f] + pick_axis(e >> 22 & 3, abv) * src[((e >> 11) & 0x7ff) * NFP + f];
    }
    __syncwarp(tmask);
    cur = (cur + 1) % 3;
  });
  const X* Hb = buf[cur];  // [b][a][f]
  if constexpr (LD == 0) {
    for (int q = lane; q < NAB * NC; q += T) {
      const int abr = q / NC, ic = q - abr * NC;
      const int ia = abr / NB, ib = abr - ia * NB;
      out[q] = Hb[(ib * NA + ia) * NFP + ic];
    }
  } else {
    const int w0 = (cur + 1) % 3, w1 = (cur + 2) % 3;
    static_for<LD>([&](auto k_) {
      constexpr int KD = decltype(k_)::value + 1;
      constexpr int NEL = ncart(KD) * nrange(LC, NF - KD);
      constexpr int NELP = ncart(KD - 1) * nrange(LC, NF - KD + 1);
      constexpr int OFF = H::ket_off(KD);
      const X* src = KD == 1 ? Hb : ((KD & 1) ? buf[w1] : buf[w0]);
      X* dst = (KD & 1) ? buf[w0] : buf[w1];
      for (int q = lane; q < NAB * NEL; q += T) {
        const int abr = q / NEL, el = q - abr * NEL;
        const int e = tab[OFF + el];
        int base;
        if constexpr (KD == 1) {
          const int ia = abr / NB, ib = abr - ia * NB;
          base = (ib * NA + ia) * NFP;
        } else {
          base = abr * NELP;
        }
        const X v = src[base + (e & 0x7ff)] + pick_axis(e >> 22 & 3, cdv) * src[base + ((e >> 11) & 0x7ff)];
        if constexpr (KD == LD)
          out[abr * (NC * ND) + ((e >> 24) & 0xff)] = v;
        else
          dst[q] = v;
      }
      __syncwarp(tmask);
    });
  }
  __syncwarp(tmask);
}

// One axis of the Cartesian -> spherical transform of a [D0][D1][D2][D3]
// block on a team (same sums as c2s_axis): M is the (2l+1) x n_cart matrix
// in shared memory.
template <int AXIS, int D0, int D1, int D2, int D3, int NOUT, int T, typename X>
__device__ __forceinline__ void team_c2s_axis(const X* in, X* out, const X* M, int lane) {
  constexpr int dims[4] = {D0, D1, D2, D3};
  constexpr int NIN = dims[AXIS];
  constexpr int outer = AXIS == 0 ? 1 : (AXIS == 1 ? D0 : (AXIS == 2 ? D0 * D1 : D0 * D1 * D2));
  constexpr int inner = AXIS == 0 ? D1 * D2 * D3 : (AXIS == 1 ? D2 * D3 : (AXIS == 2 ? D3 : 1));
  for (int q = lane; q < outer * NOUT * inner; q += T) {
    const int sidx = q % inner, t = q / inner;
    const int qo = t % NOUT, o = t / NOUT;
    const X* src = in + (o * NIN) * inner + sidx;
    const X* m = M + qo * NIN;
    X acc = X(0);
#pragma unroll
    for (int j = 0; j < NIN; ++j) acc += m[j] * src[j * inner];
    out[q] = acc;
  }
}

// Shared-memory copies of the four c2s matrices of a class (l_a, l_b, l_c,
// l_d), each (2l+1) x n_cart, at most 9 x 15 (g shells).
constexpr int C2S_TILE = 9 * 15;
template <int LA, int LB, int LC, int LD, typename X>
__device__ __forceinline__ void stage_c2s(const KernelArgs& A, X* s_m) {
  static_assert((2 * LA + 1) * ncart(LA) <= C2S_TILE && (2 * LB + 1) * ncart(LB) <= C2S_TILE &&
                    (2 * LC + 1) * ncart(LC) <= C2S_TILE && (2 * LD + 1) * ncart(LD) <= C2S_TILE,
                "c2s matrix larger than its shared-memory tile");
  const int ls[4] = {LA, LB, LC, LD};
  for (int t = threadIdx.x; t < 4 * C2S_TILE; t += blockDim.x) {
    const int ax = t / C2S_TILE, i = t - ax * C2S_TILE;
    const int l = ls[ax];
    s_m[t] = i < (2 * l + 1) * ncart(l) ? (X)A.c2s[A.c2s_off[l] + i] : X(0);
  }
}

// Post phase of a symmetric J/K quartet whose four shells are Cartesian:
// horizontal recurrences into the slot, the block copied to the team's
// shared memory (when it has room), then the six image contractions of
// consume_jk with the shape fixed at compile time.
template <int LA, int LB, int LC, int LD, int T, typename X>
__device__ __forceinline__ void post_quartet_jk_cart(const KernelArgs& A, const PairD& pb, const PairD& pk,
                                                     const Screen& sc, double* slot, int lane, unsigned tmask, int pbi,
                                                     X* stage, const int* hrr_tab) {
  constexpr int N0 = ncart(LA), N1 = ncart(LB), N2 = ncart(LC), N3 = ncart(LD);
  const SlotLayout L = slot_layout(LA, LB, LC, LD);
  X* xs = reinterpret_cast<X*>(slot);
  X* buf[3] = {xs, xs + L.S, xs + 2 * L.S};
  const double ab[3] = {pb.abx, pb.aby, pb.abz};
  const double cdv[3] = {pk.abx, pk.aby, pk.abz};
  // the block goes straight to the team's shared memory when it has room
  X* B = stage ? stage : xs + 3 * L.S;
  team_hrr<LA, LB, LC, LD, T, X>(buf, hrr_tab, B, ab, cdv, lane, tmask);
  const int shl[4] = {pb.a, pb.b, pk.a, pk.b};
  const int offs[4] = {A.shells[shl[0]].off, A.shells[shl[1]].off, A.shells[shl[2]].off, A.shells[shl[3]].off};
  double* acc = slot + A.acc_offset;
  if ((int)acc[0] != pbi) {
    flush_bra_acc(A, acc, lane, T, tmask);
    if (lane == 0) acc[0] = (double)pbi;
    __syncwarp(tmask);
  }
  const unsigned wp = distinct_perms(shl);
  auto W = [&](int p) { return (X)((wp >> p) & 1u); };
  const X w0 = W(0) + W(1) + W(2) + W(3), w1 = W(4) + W(5) + W(6) + W(7);
  const X w2 = W(0) + W(4), w3 = W(1) + W(5), w4 = W(2) + W(6), w5 = W(3) + W(7);
  const unsigned long long live = A.jk.ndens >= 64 ? ~0ull : ((1ull << A.jk.ndens) - 1ull);
  const uint64_t mask = sc.mask & live;
  for (int d0 = 0; d0 < A.jk.ndens; d0 += JK_DCH) {
    const unsigned m = (unsigned)((mask >> d0) & ((1u << JK_DCH) - 1u));
    if (!m) continue;
    jk_term_ct<0, 1, 2, 3, N0, N1, N2, N3, T, true, X>(A, B, offs, w0, d0, m, acc, lane);
    if (w1 != X(0)) jk_term_ct<2, 3, 0, 1, N0, N1, N2, N3, T, false, X>(A, B, offs, w1, d0, m, A.jk.J, lane);
    if (A.jk.want_k) {
      if (w2 != X(0)) jk_term_ct<0, 2, 1, 3, N0, N1, N2, N3, T, false, X>(A, B, offs, w2, d0, m, A.jk.K, lane);
      if (w3 != X(0)) jk_term_ct<1, 2, 0, 3, N0, N1, N2, N3, T, false, X>(A, B, offs, w3, d0, m, A.jk.K, lane);
      if (w4 != X(0)) jk_term_ct<0, 3, 1, 2, N0, N1, N2, N3, T, false, X>(A, B, offs, w4, d0, m, A.jk.K, lane);
      if (w5 != X(0)) jk_term_ct<1, 3, 0, 2, N0, N1, N2, N3, T, false, X>(A, B, offs, w5, d0, m, A.jk.K, lane);
    }
  }
  __syncwarp(tmask);
}

// Post phase of a symmetric J/K quartet whose four shells are spherical:
// table-driven horizontal recurrences into the slot, the four transform
// axes on the team, the spherical block in the team's shared memory when it
// has room, then the six image contractions with the spherical shape.
template <int LA, int LB, int LC, int LD, int T, typename X>
__device__ __forceinline__ void post_quartet_jk_sph(const KernelArgs& A, const PairD& pb, const PairD& pk,
                                                    const Screen& sc, double* slot, int lane, unsigned tmask, int pbi,
                                                    X* stage, const int* hrr_tab, const X* s_m) {
  constexpr int N0 = ncart(LA), N1 = ncart(LB), N2 = ncart(LC), N3 = ncart(LD);
  constexpr int F0 = 2 * LA + 1, F1 = 2 * LB + 1, F2 = 2 * LC + 1, F3 = 2 * LD + 1;
  const SlotLayout L = slot_layout(LA, LB, LC, LD);
  X* xs = reinterpret_cast<X*>(slot);
  X* buf[3] = {xs, xs + L.S, xs + 2 * L.S};
  X* blk = xs + 3 * L.S;
  X* tmp = blk + L.blk;
  const double ab[3] = {pb.abx, pb.aby, pb.abz};
  const double cdv[3] = {pk.abx, pk.aby, pk.abz};
  team_hrr<LA, LB, LC, LD, T, X>(buf, hrr_tab, blk, ab, cdv, lane, tmask);
  team_c2s_axis<0, N0, N1, N2, N3, F0, T, X>(blk, tmp, s_m + 0 * C2S_TILE, lane);
  __syncwarp(tmask);
  team_c2s_axis<1, F0, N1, N2, N3, F1, T, X>(tmp, blk, s_m + 1 * C2S_TILE, lane);
  __syncwarp(tmask);
  team_c2s_axis<2, F0, F1, N2, N3, F2, T, X>(blk, tmp, s_m + 2 * C2S_TILE, lane);
  __syncwarp(tmask);
  X* B = stage ? stage : blk;
  team_c2s_axis<3, F0, F1, F2, N3, F3, T, X>(tmp, B, s_m + 3 * C2S_TILE, lane);
  __syncwarp(tmask);
  const int shl[4] = {pb.a, pb.b, pk.a, pk.b};
  const int offs[4] = {A.shells[shl[0]].off, A.shells[shl[1]].off, A.shells[shl[2]].off, A.shells[shl[3]].off};
  double* acc = slot + A.acc_offset;
  if ((int)acc[0] != pbi) {
    flush_bra_acc(A, acc, lane, T, tmask);
    if (lane == 0) acc[0] = (double)pbi;
    __syncwarp(tmask);
  }
  const unsigned wp = distinct_perms(shl);
  auto W = [&](int p) { return (X)((wp >> p) & 1u); };
  const X w0 = W(0) + W(1) + W(2) + W(3), w1 = W(4) + W(5) + W(6) + W(7);
  const X w2 = W(0) + W(4), w3 = W(1) + W(5), w4 = W(2) + W(6), w5 = W(3) + W(7);
  const unsigned long long live = A.jk.ndens >= 64 ? ~0ull : ((1ull << A.jk.ndens) - 1ull);
  const uint64_t mask = sc.mask & live;
  for (int d0 = 0; d0 < A.jk.ndens; d0 += JK_DCH) {
    const unsigned m = (unsigned)((mask >> d0) & ((1u << JK_DCH) - 1u));
    if (!m) continue;
    jk_term_ct<0, 1, 2, 3, F0, F1, F2, F3, T, true, X>(A, B, offs, w0, d0, m, acc, lane);
    if (w1 != X(0)) jk_term_ct<2, 3, 0, 1, F0, F1, F2, F3, T, false, X>(A, B, offs, w1, d0, m, A.jk.J, lane);
    if (A.jk.want_k) {
      if (w2 != X(0)) jk_term_ct<0, 2, 1, 3, F0, F1, F2, F3, T, false, X>(A, B, offs, w2, d0, m, A.jk.K, lane);
      if (w3 != X(0)) jk_term_ct<1, 2, 0, 3, F0, F1, F2, F3, T, false, X>(A, B, offs, w3, d0, m, A.jk.K, lane);
      if (w4 != X(0)) jk_term_ct<0, 3, 1, 2, F0, F1, F2, F3, T, false, X>(A, B, offs, w4, d0, m, A.jk.K, lane);
      if (w5 != X(0)) jk_term_ct<1, 3, 0, 2, F0, F1, F2, F3, T, false, X>(A, B, offs, w5, d0, m, A.jk.K, lane);
    }
  }
  __syncwarp(tmask);
}

}  // namespace igpu
