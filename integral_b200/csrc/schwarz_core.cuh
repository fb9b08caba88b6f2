// The diagonal Schwarz quartet (ij|ij) of the reference's OS/HGP engine for
// the device: the same arithmetic, in the same order, as the host evaluation
// (host_schwarz.cpp) and the reference (src/engine/os_eri.rs:455-697,
// 2860-3143, src/math/boys.rs:63-431, src/spherical.rs:121-179), so that the
// device produces the reference's Schwarz bounds bit for bit.  One thread,
// or one warp for the larger classes, evaluates one shell pair; its work
// arrays live in a slice of a global scratch buffer, element k at
// base[k * stride] (one thread per pair: stride = threads of the launch, so
// that the threads of a warp touch consecutive words; one warp per pair:
// stride 1, the lanes splitting each level).  The vertical recurrence keeps the reference's
// rolling window of three ket levels, each packed by Boys order.  Compile
// with -fmad=false: every product and sum rounds on its own, as in Rust.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <cstdint>

// host and device: the host copy serves the CPU check of this code
#define SC_HD __host__ __device__ __forceinline__

namespace igpu {
namespace sc {

constexpr double kPi = 3.14159265358979323846;
constexpr int kBoysMaxM = 24, kBoysTaylor = 8, kBoysOrders = 33, kBoysRow = 34;

// The Boys interpolation table of the host (T0 = 0.1 i, orders 0..32 and
// e^{-T0}) and its constants.
struct BoysDev {
  const double* tab;
  double tmax, h;
  double inv_fact[kBoysTaylor + 1];
  double inv_odd[kBoysMaxM + 1];
};

// Strided view of one thread's slice of the scratch buffer.
struct Slice {
  double* base;
  size_t stride;
  SC_HD double& operator[](size_t k) const { return base[k * stride]; }
};

// Degree-indexed Cartesian triple helpers (src/math/am.rs order: lx
// descending, then ly descending).
SC_HD int sc_deg_below(int d) { return d * (d + 1) * (d + 2) / 6; }
SC_HD int sc_ncart(int l) { return (l + 1) * (l + 2) / 2; }
SC_HD void sc_triple(int d, int idx, int& x, int& y, int& z) {
  int r = 0;
  while ((r + 1) * (r + 2) / 2 <= idx) ++r;
  z = idx - r * (r + 1) / 2;
  y = r - z;
  x = d - r;
}
SC_HD int sc_within(int x, int y, int z) {
  const int r = y + z;
  return r * (r + 1) / 2 + z;
}
SC_HD int sc_addr(int x, int y, int z) { return sc_deg_below(x + y + z) + sc_within(x, y, z); }
SC_HD int sc_low_axis(int x, int y, int) { return x > 0 ? 0 : (y > 0 ? 1 : 2); }
SC_HD int sc_get(int x, int y, int z, int a) { return a == 0 ? x : (a == 1 ? y : z); }

// F_0..F_mmax(t) into f (src/math/boys.rs: boys_array).  Above the table
// (t >= 93) the top order is the asymptotic closed form and the downward
// recurrence adds e^{-t} < 4e-41 to terms of at least 1e-24 (m <= 24), far
// below half an ulp, so the device exp gives the same bits as libm's.
SC_HD void sc_boys(const BoysDev& B, int mmax, double t, double* f) {
  if (t < B.tmax && mmax + kBoysTaylor < kBoysOrders) {
    const size_t i = (size_t)::round(t * (1.0 / B.h));
    const double nd = (double)i * B.h - t;
    const double* row = B.tab + i * kBoysRow;
    double top = row[mmax + kBoysTaylor] * B.inv_fact[kBoysTaylor];
    for (int k = kBoysTaylor - 1; k >= 0; --k) top = top * nd + row[mmax + k] * B.inv_fact[k];
    f[mmax] = top;
    if (mmax > 0) {
      double ep = B.inv_fact[kBoysTaylor];
      for (int k = kBoysTaylor - 1; k >= 0; --k) ep = ep * nd + B.inv_fact[k];
      const double et = row[kBoysOrders] * ep;
      const double two_t = 2.0 * t;
      for (int m = mmax; m > 0; --m) f[m - 1] = (two_t * f[m] + et) * B.inv_odd[m];
    }
    return;
  }
  const double et = ::exp(-t);
  double v = 0.5 * ::sqrt(kPi / t);
  const double two_t = 2.0 * t;
  for (int k = 1; k <= mmax; ++k) v *= (double)(2 * k - 1) / two_t;
  f[mmax] = v;
  for (int m = mmax; m > 0; --m) f[m - 1] = (2.0 * t * f[m] + et) / (double)(2 * m - 1);
}

// One primitive pair of the bra (== ket) of the diagonal quartet.
struct SPrim {
  double zeta, kappa, c1, c2, inv2z;
  double P[3], PA[3];
};

// The class layout of one launch: the packed rolling window of the
// vertical recurrence (slab per ket level, e-offsets per (level, address))
// and the offsets of every work array inside a thread's slice.
struct SClass {
  int li, lj;             // shells i and j of the diagonal quartet
  int ne, nf, lt, n_e, n_f;
  int maxlevel;           // doubles per window slot
  int slab[9];            // per ket level k <= nf
  const int* eoff;        // [(nf+1) * n_e], device
  size_t o_prims, o_lev, o_cef, o_bra, o_prev, o_cur, o_kprev, o_kcur, o_blk, o_tmp, total;
};


// The lanes that evaluate one pair together: lane in [0, size), size 1 or
// a full warp.  Every element of a recurrence level, of a transform axis and
// of a contracted table is computed by one lane with the operations of the
// serial order (the primitive loops stay sequential and every sum keeps its
// order), so any team size gives the same bits; sync() separates the
// phases that read what other lanes wrote.
struct Team {
  int lane, size;
  SC_HD void sync() const {
#ifdef __CUDA_ARCH__
    if (size > 1) __syncwarp();
#endif
  }
};

// Degree of the Cartesian address a (sc_deg_below(d) <= a < sc_deg_below(d + 1)).
SC_HD int sc_degree(int a) {
  int d = 0;
  while (sc_deg_below(d + 1) <= a) ++d;
  return d;
}

// (ij|ij) of one team: shells given by centre, l, primitive count,
// exponents, effective coefficients and c2s matrix (nullptr: Cartesian);
// kappa = the host's exp(-(e1 e2 / z) |AB|^2) of every (i, j) primitive
// combination, i outer.  Returns Q = sqrt(max |(mu nu|mu nu)|) on every lane.
SC_HD double sc_schwarz(const BoysDev& B, const SClass& C, const Slice& W, const Team& T, const double* ca,
                        const double* cb, int npa, int npb, const double* ea, const double* wa, const double* eb,
                        const double* wb, const double* kappa, const double* c2a, const double* c2b) {
  const int la = C.li, lb = C.lj;
  const int ne = C.ne, nf = C.nf, lt = C.lt, n_e = C.n_e, n_f = C.n_f;
  const int L0 = T.lane, LS = T.size;
  // primitive pairs (src/engine/os_eri.rs:221-244), 11 doubles each
  int np = 0;
  for (int a = 0; a < npa; ++a)
    for (int b = 0; b < npb; ++b) {
      const double e1 = ea[a], e2 = eb[b];
      const double c1 = wa[a], c2 = wb[b];
      const double z = e1 + e2;
      const double kap = kappa[a * npb + b];
      if (kap * fabs(c1 * c2) < 1e-32) continue;
      if (L0 == 0) {
        const size_t o = C.o_prims + (size_t)np * 11;
        W[o + 0] = z;
        W[o + 1] = kap;
        W[o + 2] = c1;
        W[o + 3] = c2;
        W[o + 4] = 0.5 / z;
        for (int k = 0; k < 3; ++k) {
          const double P = (e1 * ca[k] + e2 * cb[k]) / z;
          W[o + 5 + k] = P;
          W[o + 8 + k] = P - ca[k];
        }
      }
      ++np;
    }
  const int na = sc_ncart(la), nb = sc_ncart(lb);
  const size_t nblk = (size_t)na * nb * na * nb;
  for (size_t q = L0; q < nblk; q += LS) W[C.o_blk + q] = 0.0;
  T.sync();
  if (lt == 0) {
    // (ss|ss) fast path (src/engine/os_eri.rs:500-536)
    if (L0 == 0) {
      const double two_pi_2_5 = 2.0 * kPi * kPi * ::sqrt(kPi);
      double acc = 0.0;
      for (int x = 0; x < np; ++x) {
        const size_t ob = C.o_prims + (size_t)x * 11;
        const double bc = W[ob + 2] * W[ob + 3];
        const double p = W[ob + 0];
        for (int y = 0; y < np; ++y) {
          const size_t ok = C.o_prims + (size_t)y * 11;
          const double q = W[ok + 0];
          const double pq = p + q;
          const double dx = W[ob + 5] - W[ok + 5], dy = W[ob + 6] - W[ok + 6], dz = W[ob + 7] - W[ok + 7];
          const double t = (p * q / pq) * (dx * dx + dy * dy + dz * dz);
          const double pref = two_pi_2_5 / (p * q * ::sqrt(pq)) * W[ob + 1] * W[ok + 1];
          double f0;
          sc_boys(B, 0, t, &f0);
          acc += (bc * W[ok + 2]) * W[ok + 3] * (pref * f0);
        }
      }
      W[C.o_blk] += acc;
    }
    T.sync();
  } else {
    for (size_t q = L0; q < (size_t)n_e * n_f; q += LS) W[C.o_cef + q] = 0.0;
    T.sync();
    auto L = [&](int k, int lf, int ae, int m) -> double& {
      return W[C.o_lev + (size_t)(k % 3) * C.maxlevel + (size_t)lf * C.slab[k] + C.eoff[k * n_e + ae] + m];
    };
    double fm[4 * 6 + 3];
    for (int x = 0; x < np; ++x) {
      const size_t ob = C.o_prims + (size_t)x * 11;
      const double bc = W[ob + 2] * W[ob + 3];
      for (int y = 0; y < np; ++y) {
        const size_t ok = C.o_prims + (size_t)y * 11;
        const double scale = (bc * W[ok + 2]) * W[ok + 3];
        // src/engine/os_eri.rs:2860-3020
        const double p = W[ob + 0], q = W[ok + 0];
        const double pq = p + q;
        const double rho = p * q / pq;
        const double bP[3] = {W[ob + 5], W[ob + 6], W[ob + 7]}, kP[3] = {W[ok + 5], W[ok + 6], W[ok + 7]};
        const double bPA[3] = {W[ob + 8], W[ob + 9], W[ob + 10]}, kPA[3] = {W[ok + 8], W[ok + 9], W[ok + 10]};
        const double d0 = bP[0] - kP[0], d1 = bP[1] - kP[1], d2 = bP[2] - kP[2];
        const double t = rho * (d0 * d0 + d1 * d1 + d2 * d2);
        double wv[3], wp[3], wq[3];
        for (int a = 0; a < 3; ++a) wv[a] = (p * bP[a] + q * kP[a]) / pq;
        for (int a = 0; a < 3; ++a) {
          wp[a] = wv[a] - bP[a];
          wq[a] = wv[a] - kP[a];
        }
        const double pref = 2.0 * kPi * kPi * ::sqrt(kPi) / (p * q * ::sqrt(pq)) * W[ob + 1] * W[ok + 1];
        sc_boys(B, lt, t, fm);
        for (int m = L0; m <= lt; m += LS) L(0, 0, 0, m) = pref * fm[m];
        T.sync();
        const double inv2pq = 0.5 / pq, q_pq = q / pq, p_pq = p / pq;
        const double inv2p = W[ob + 4], inv2q = W[ok + 4];
        for (int nd = 1; nd <= ne; ++nd) {
          for (int ti = L0; ti < sc_ncart(nd); ti += LS) {
            int x0, y0, z0;
            sc_triple(nd, ti, x0, y0, z0);
            const int i = sc_low_axis(x0, y0, z0);
            const int xi = sc_get(x0, y0, z0, i);
            const int a1 = sc_addr(x0 - (i == 0), y0 - (i == 1), z0 - (i == 2));
            const bool two = xi >= 2;
            const double c2 = (double)(xi - 1) * inv2p;
            const int a2 = two ? sc_addr(x0 - 2 * (i == 0), y0 - 2 * (i == 1), z0 - 2 * (i == 2)) : 0;
            const int ad = sc_addr(x0, y0, z0);
            for (int m = 0; m <= lt - nd; ++m) {
              double v = bPA[i] * L(0, 0, a1, m) + wp[i] * L(0, 0, a1, m + 1);
              if (two) v += c2 * (L(0, 0, a2, m) - q_pq * L(0, 0, a2, m + 1));
              L(0, 0, ad, m) = v;
            }
          }
          T.sync();
        }
        for (int ae = L0; ae < n_e; ae += LS) W[C.o_cef + (size_t)ae * n_f] += scale * L(0, 0, ae, 0);
        for (int kd = 1; kd <= nf; ++kd) {
          const int nfk = sc_ncart(kd);
          for (int idx = L0; idx < nfk * n_e; idx += LS) {
            const int fi = idx / n_e, ea_ = idx - fi * n_e;
            int fx, fy, fz;
            sc_triple(kd, fi, fx, fy, fz);
            const int j = sc_low_axis(fx, fy, fz);
            const int fj = sc_get(fx, fy, fz, j);
            const int gx = fx - (j == 0), gy = fy - (j == 1), gz = fz - (j == 2);
            const int lf1 = sc_within(gx, gy, gz);
            const bool two = fj >= 2;
            const double c2 = (double)(fj - 1) * inv2q;
            const int lf2 = two ? sc_within(gx - (j == 0), gy - (j == 1), gz - (j == 2)) : 0;
            const int lf = fi;
            const int nd = sc_degree(ea_);
            int x0, y0, z0;
            sc_triple(nd, ea_ - sc_deg_below(nd), x0, y0, z0);
            const int ej = sc_get(x0, y0, z0, j);
            const bool cross = ej >= 1;
            const double cc = cross ? (double)ej * inv2pq : 0.0;
            const int ax = cross ? sc_addr(x0 - (j == 0), y0 - (j == 1), z0 - (j == 2)) : 0;
            for (int m = 0; m <= lt - nd - kd; ++m) {
              double v = kPA[j] * L(kd - 1, lf1, ea_, m) + wq[j] * L(kd - 1, lf1, ea_, m + 1);
              if (two) v += c2 * (L(kd - 2, lf2, ea_, m) - p_pq * L(kd - 2, lf2, ea_, m + 1));
              if (cross) v += cc * L(kd - 1, lf1, ax, m + 1);
              L(kd, lf, ea_, m) = v;
            }
          }
          T.sync();
          for (int idx = L0; idx < nfk * n_e; idx += LS) {
            const int fi = idx / n_e, ae = idx - fi * n_e;
            int fx, fy, fz;
            sc_triple(kd, fi, fx, fy, fz);
            const int af = sc_addr(fx, fy, fz);
            W[C.o_cef + (size_t)ae * n_f + af] += scale * L(kd, fi, ae, 0);
          }
        }
        T.sync();
      }
    }
    // contracted HRR, bra then ket (src/engine/os_eri.rs:3040-3143)
    const double ab[3] = {ca[0] - cb[0], ca[1] - cb[1], ca[2] - cb[2]};
    const int fb = sc_deg_below(la);
    const int nfr = n_f - fb;
    size_t prev = C.o_prev, cur = C.o_cur;
    for (int fg = fb; fg < n_f; ++fg) {
      for (int ae = fb + L0; ae < sc_deg_below(ne + 1); ae += LS) W[prev + ae] = W[C.o_cef + (size_t)ae * n_f + fg];
      T.sync();
      for (int kb = 1; kb <= lb; ++kb) {
        const int cnt = sc_deg_below(ne - kb + 1) - fb;
        for (int idx = L0; idx < sc_ncart(kb) * cnt; idx += LS) {
          const int bi = idx / cnt, ae = fb + (idx - bi * cnt);
          int bx, by, bz;
          sc_triple(kb, bi, bx, by, bz);
          const int i = sc_low_axis(bx, by, bz);
          const int b1 = sc_within(bx - (i == 0), by - (i == 1), bz - (i == 2));
          const int dg = sc_degree(ae);
          int x0, y0, z0;
          sc_triple(dg, ae - sc_deg_below(dg), x0, y0, z0);
          const int a1 = sc_addr(x0 + (i == 0), y0 + (i == 1), z0 + (i == 2));
          W[cur + (size_t)bi * n_e + ae] = W[prev + (size_t)b1 * n_e + a1] + ab[i] * W[prev + (size_t)b1 * n_e + ae];
        }
        T.sync();
        const size_t t = prev;
        prev = cur;
        cur = t;
      }
      for (int idx = L0; idx < nb * na; idx += LS) {
        const int bi = idx / na, ai = idx - bi * na;
        W[C.o_bra + ((size_t)ai * nb + bi) * nfr + (fg - fb)] = W[prev + (size_t)bi * n_e + fb + ai];
      }
      T.sync();
    }
    const int nc = na, ndd = nb;
    for (int ai = 0; ai < na; ++ai)
      for (int bi = 0; bi < nb; ++bi) {
        const size_t row = ((size_t)ai * nb + bi) * nfr;
        size_t kp = C.o_kprev, kc = C.o_kcur;
        for (int ce = fb + L0; ce < sc_deg_below(nf + 1); ce += LS) W[kp + ce] = W[C.o_bra + row + (ce - fb)];
        T.sync();
        for (int kd = 1; kd <= lb; ++kd) {
          const int cnt = sc_deg_below(nf - kd + 1) - fb;
          for (int idx = L0; idx < sc_ncart(kd) * cnt; idx += LS) {
            const int di = idx / cnt, ce = fb + (idx - di * cnt);
            int dx, dy, dz;
            sc_triple(kd, di, dx, dy, dz);
            const int j = sc_low_axis(dx, dy, dz);
            const int d1 = sc_within(dx - (j == 0), dy - (j == 1), dz - (j == 2));
            const int dg = sc_degree(ce);
            int x0, y0, z0;
            sc_triple(dg, ce - sc_deg_below(dg), x0, y0, z0);
            const int c1 = sc_addr(x0 + (j == 0), y0 + (j == 1), z0 + (j == 2));
            W[kc + (size_t)di * n_f + ce] = W[kp + (size_t)d1 * n_f + c1] + ab[j] * W[kp + (size_t)d1 * n_f + ce];
          }
          T.sync();
          const size_t t = kp;
          kp = kc;
          kc = t;
        }
        for (int idx = L0; idx < nc * ndd; idx += LS) {
          const int ci = idx / ndd, di = idx - ci * ndd;
          W[C.o_blk + (((size_t)ai * nb + bi) * nc + ci) * ndd + di] += W[kp + (size_t)di * n_f + fb + ci];
        }
        T.sync();
      }
  }
  // per-axis c2s (src/spherical.rs:121-179), then the diagonal maximum;
  // every output element sums its inputs in the serial order from 0.0
  int dims[4] = {na, nb, na, nb};
  const double* mats[4] = {c2a, c2b, c2a, c2b};
  const int lsh[4] = {la, lb, la, lb};
  size_t cur = C.o_blk, oth = C.o_tmp;
  for (int axis = 0; axis < 4; ++axis) {
    if (!mats[axis]) continue;
    const int n_in = dims[axis], n_o = 2 * lsh[axis] + 1;
    size_t outer = 1, inner = 1;
    for (int q = 0; q < axis; ++q) outer *= dims[q];
    for (int q = axis + 1; q < 4; ++q) inner *= dims[q];
    const double* M = mats[axis];
    for (size_t idx = L0; idx < outer * n_o * inner; idx += LS) {
      const size_t s2 = idx % inner, t = idx / inner;
      const size_t r = t % n_o, o = t / n_o;
      double v = 0.0;
      for (int j = 0; j < n_in; ++j) {
        const double m = M[r * n_in + j];
        if (m == 0.0) continue;
        v += m * W[cur + (o * n_in + j) * inner + s2];
      }
      W[oth + idx] = v;
    }
    T.sync();
    dims[axis] = n_o;
    const size_t t = cur;
    cur = oth;
    oth = t;
  }
  const int ni = dims[0], nj = dims[1];
  double mx = 0.0;
  for (int idx = L0; idx < ni * nj; idx += LS) {
    const int mu = idx / nj, nu = idx - mu * nj;
    mx = fmax(mx, fabs(W[cur + (((size_t)mu * nj + nu) * ni + mu) * nj + nu]));
  }
#ifdef __CUDA_ARCH__
  if (LS > 1)
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
#endif
  T.sync();
  return ::sqrt(mx);
}

}  // namespace sc
}  // namespace igpu
