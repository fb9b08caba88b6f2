// Density-direct ERI nuclear gradient (DirectGradContractor,
// src/direct_grad.rs:394-485), one launch per angular class in evaluation
// orientation (la >= lb, lc >= ld, bra class >= ket class).
//
// For a canonical quartet with degeneracy-weighted two-particle density
// block W (src/direct_grad.rs:490-547, pulled back to Cartesian components),
// the derivative on the centre of position p is
//   g_p,x = sum W[..a..] * ( (..a+1x..)~ - a_x (..a-1x..) ),
// the raised block (..)~ built from primitives weighted by 2*alpha of
// position p, the lowered block from the plain ones (src/direct_grad.rs:
// 431-470).  Positions A, B, C are evaluated; D follows from translational
// invariance (src/direct_grad.rs:476-484).
//
// Nothing is stored between quartets: phase 1 recomputes the Rys 2D
// integrals of the quartet with one extra unit of angular momentum on the bra
// and on the ket and contracts, in one sweep over the primitive quartets,
// four [e0|f0] tables:
//   P  plain          e in [la-1, la+lb]   f in [lc-1, lc+ld]  (all lowered blocks)
//   A  2*alpha_A      e in [la+1, la+lb+1] f in [lc, lc+ld]
//   B  2*alpha_B      e in [la, la+lb+1]   f in [lc, lc+ld]
//   C  2*alpha_C      e in [la, la+lb]     f in [lc+1, lc+ld+1]
// (A and B share their rows: one product feeds both).  Phase 2 runs the
// horizontal recurrences of the six shifted blocks from these tables and
// dots each with W, so the gradient is the adjoint of the value path with
// the intermediates recomputed instead of kept.
#pragma once
#include "device_common.cuh"
#include "post.cuh"
#include "quartet.cuh"

namespace igpu {

// ------------------------------------------------------------ table shapes
// Segments of the phase-1 sweep: 0 = P, 1 = A and B, 2 = C.
__host__ __device__ constexpr bool g_low(int la, int lc) { return la > 0 || lc > 0; }
__host__ __device__ constexpr int g_ea(int la, int, int, int, int s) { return s == 0 ? (la > 0 ? la - 1 : 0) : la; }
__host__ __device__ constexpr int g_eb(int la, int lb, int, int, int s) { return s == 1 ? la + lb + 1 : la + lb; }
__host__ __device__ constexpr int g_fa(int, int, int lc, int, int s) {
  return s == 0 ? (lc > 0 ? lc - 1 : 0) : (s == 1 ? lc : lc + 1);
}
__host__ __device__ constexpr int g_fb(int, int, int lc, int ld, int s) { return s == 2 ? lc + ld + 1 : lc + ld; }
__host__ __device__ constexpr int g_rows(int la, int lb, int lc, int ld, int s) {
  return nrange(g_ea(la, lb, lc, ld, s), g_eb(la, lb, lc, ld, s));
}
__host__ __device__ constexpr int g_cols(int la, int lb, int lc, int ld, int s) {
  return nrange(g_fa(la, lb, lc, ld, s), g_fb(la, lb, lc, ld, s));
}
// accumulators per table entry of a segment
__host__ __device__ constexpr int g_nacc(int la, int, int lc, int, int s) {
  return s == 1 ? 2 : (s == 0 ? (g_low(la, lc) ? 1 : 0) : 1);
}
__host__ __device__ constexpr int g_acc_total(int la, int lb, int lc, int ld) {
  int t = 0;
  for (int s = 0; s < 3; ++s) t += g_nacc(la, lb, lc, ld, s) * g_rows(la, lb, lc, ld, s) * g_cols(la, lb, lc, ld, s);
  return t;
}

// Slot layout (doubles) of one gradient quartet: the four tables, two
// weight-block buffers, three HRR level buffers and the Cartesian block.
struct GradSlot {
  size_t off_p, off_a, off_b, off_c, ntab, W, S, blk, total;
};
__host__ __device__ inline GradSlot grad_slot_layout(int la, int lb, int lc, int ld) {
  GradSlot L;
  const size_t np = g_low(la, lc) ? (size_t)g_rows(la, lb, lc, ld, 0) * g_cols(la, lb, lc, ld, 0) : 0;
  const size_t na = (size_t)nrange(la + 1, la + lb + 1) * g_cols(la, lb, lc, ld, 1);
  const size_t nb = (size_t)g_rows(la, lb, lc, ld, 1) * g_cols(la, lb, lc, ld, 1);
  const size_t nc = (size_t)g_rows(la, lb, lc, ld, 2) * g_cols(la, lb, lc, ld, 2);
  L.off_p = 0;
  L.off_a = np;
  L.off_b = np + na;
  L.off_c = np + na + nb;
  L.ntab = np + na + nb + nc;
  L.W = (size_t)ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
  size_t S = 0, blk = 0;
  auto take = [&](int a, int b, int c, int d) {
    const SlotLayout s = slot_layout(a, b, c, d);
    S = s.S > S ? s.S : S;
    blk = s.blk > blk ? s.blk : blk;
  };
  take(la + 1, lb, lc, ld);
  take(la, lb + 1, lc, ld);
  take(la, lb, lc + 1, ld);
  if (la > 0) take(la - 1, lb, lc, ld);
  if (lb > 0) take(la, lb - 1, lc, ld);
  if (lc > 0) take(la, lb, lc - 1, ld);
  L.S = S;
  L.blk = blk;
  L.total = L.ntab + 2 * L.W + 3 * S + blk;
  return L;
}

// Lanes per quartet: one thread while all accumulators fit in registers,
// else the smallest team of 8, 16 or 32 lanes giving each lane at most one
// row of every segment (32 beyond that).  Measured against at most two rows
// per lane: fewer columns per lane means fewer passes, each of which
// recomputes the 2D tables of every primitive quartet.
__host__ __device__ constexpr int grad_team_for(int la, int lb, int lc, int ld) {
  if (g_acc_total(la, lb, lc, ld) <= 40) return 1;
  int mr = 0;
  for (int s = 0; s < 3; ++s)
    if (g_nacc(la, lb, lc, ld, s) > 0 && g_rows(la, lb, lc, ld, s) > mr) mr = g_rows(la, lb, lc, ld, s);
  for (int t = 8; t < 32; t *= 2)
    if ((mr + t - 1) / t <= 1) return t;
  return 32;
}

// Compile-time plan of the team sweep: items = (segment, column chunk);
// consecutive items are packed into passes of at most BUD accumulators per
// lane.  Every pass recomputes the Rys 2D tables of all primitive quartets.
constexpr int GPLAN_MAX = 96;
struct GradPassPlan {
  int nitems;
  int seg[GPLAN_MAX], f0[GPLAN_MAX], fw[GPLAN_MAX], off[GPLAN_MAX], rslot[GPLAN_MAX];
  int npass;
  int pbeg[GPLAN_MAX + 1];
  int pacc[GPLAN_MAX];
  int prows[GPLAN_MAX];
};
__host__ __device__ constexpr GradPassPlan make_grad_plan(int la, int lb, int lc, int ld, int T, int bud) {
  GradPassPlan p{};
  int n = 0;
  for (int s = 0; s < 3; ++s) {
    const int na = g_nacc(la, lb, lc, ld, s);
    if (na == 0) continue;
    const int rl = (g_rows(la, lb, lc, ld, s) + T - 1) / T;
    const int cols = g_cols(la, lb, lc, ld, s);
    int fch = bud / (rl * na);
    fch = fch < 1 ? 1 : (fch > cols ? cols : fch);
    for (int f0 = 0; f0 < cols; f0 += fch) {
      p.seg[n] = s;
      p.f0[n] = f0;
      p.fw[n] = cols - f0 < fch ? cols - f0 : fch;
      ++n;
    }
  }
  p.nitems = n;
  int np = 0, cur = 0, rows = 0;
  p.pbeg[0] = 0;
  for (int i = 0; i < n; ++i) {
    const int s = p.seg[i];
    const int rl = (g_rows(la, lb, lc, ld, s) + T - 1) / T;
    const int acc = rl * p.fw[i] * g_nacc(la, lb, lc, ld, s);
    if (cur > 0 && cur + acc > bud) {
      p.pacc[np] = cur;
      p.prows[np] = rows;
      ++np;
      p.pbeg[np] = i;
      cur = 0;
      rows = 0;
    }
    p.off[i] = cur;
    p.rslot[i] = rows;
    cur += acc;
    rows += rl;
  }
  p.pacc[np] = cur;
  p.prows[np] = rows;
  ++np;
  p.pbeg[np] = n;
  p.npass = np;
  return p;
}

template <int LA, int LB, int LC, int LD, typename R>
struct GradShape {
  static constexpr int NE = LA + LB, NF = LC + LD;
  static constexpr int NEV = NE + 1, NFV = NF + 1;  // raised VRR extents
  static constexpr int NR = (NE + NF + 1) / 2 + 1;
  static constexpr bool LOW = g_low(LA, LC);
  static constexpr int T = grad_team_for(LA, LB, LC, LD);
  // accumulators per lane per pass (measured: 80/112 beat 48/72 and 64/96)
  static constexpr int BUD = sizeof(R) == 8 ? 80 : 112;
  static constexpr GradPassPlan PL = make_grad_plan(LA, LB, LC, LD, T, BUD);
  static constexpr int GT = (NEV + 1) * (NFV + 1);
  // per primitive quartet in shared memory: roots, weights*prefactor, the
  // three raise factors 2*alpha_A, 2*alpha_B, 2*alpha_C, and 3*NR 2D tables
  static constexpr int PRIM_TAB = 2 * NR + 3 + 3 * NR * GT;
  static constexpr int BUDGET = (48 * 1024 / 128) * (T == 1 ? 1 : T) / (int)sizeof(R);
  static constexpr int BP0 = BUDGET / PRIM_TAB;
  static constexpr int BP = BP0 >= T ? T : (BP0 >= 16 ? 16 : (BP0 >= 8 ? 8 : (BP0 >= 4 ? 4 : (BP0 >= 2 ? 2 : 1))));
  static constexpr int SUB = T / BP;
  static constexpr int SMEM_PER_TEAM = T == 1 ? 0 : BP * PRIM_TAB;
};

// --------------------------------------------------- phase 1, one thread

template <int LA, int LB, int LC, int LD, typename R>
__device__ __forceinline__ void grad_tables_thread(const KernelArgs& A, const R* s_tab, const PairD& pb,
                                                   const PairD& pk, double* tab) {
  using GS = GradShape<LA, LB, LC, LD, R>;
  constexpr int NEV = GS::NEV, NFV = GS::NFV, NR = GS::NR;
  constexpr int R0 = g_rows(LA, LB, LC, LD, 0), C0 = g_cols(LA, LB, LC, LD, 0);
  constexpr int R1 = g_rows(LA, LB, LC, LD, 1), C1 = g_cols(LA, LB, LC, LD, 1);
  constexpr int R2 = g_rows(LA, LB, LC, LD, 2), C2 = g_cols(LA, LB, LC, LD, 2);
  constexpr int E0 = g_ea(LA, LB, LC, LD, 0), F0 = g_fa(LA, LB, LC, LD, 0);
  constexpr int E1 = g_ea(LA, LB, LC, LD, 1), F1 = g_fa(LA, LB, LC, LD, 1);
  constexpr int E2 = g_ea(LA, LB, LC, LD, 2), F2 = g_fa(LA, LB, LC, LD, 2);
  constexpr int NP = GS::LOW ? R0 * C0 : 0;
  R aP[NP > 0 ? NP : 1], aA[R1 * C1], aB[R1 * C1], aC[R2 * C2];
#pragma unroll
  for (int q = 0; q < (NP > 0 ? NP : 1); ++q) aP[q] = R(0);
#pragma unroll
  for (int q = 0; q < R1 * C1; ++q) aA[q] = aB[q] = R(0);
#pragma unroll
  for (int q = 0; q < R2 * C2; ++q) aC[q] = R(0);
  for (int ip = 0; ip < pb.nprim; ++ip) {
    const PrimPairD bp = A.prims[pb.prim_off + ip];
    const R wA = R(2) * R(bp.alpha), wB = R(2) * R(bp.beta);
    for (int kq = 0; kq < pk.nprim; ++kq) {
      const PrimPairD kp = A.prims[pk.prim_off + kq];
      const R wC = R(2) * R(kp.alpha);
      const QuartetHdr<R> h = quartet_header<R>(bp, kp, A.omega);
      R x[NR], w[NR];
      rys_roots_s<NR, R>(s_tab, h.T, x, w);
      const R inv_pq = R(1) / h.pq;
      const R qpq = h.q * inv_pq, ppq = h.p * inv_pq;
      const R inv2pq = R(0.5) * inv_pq, inv2p = R(0.5) / h.p, inv2q = R(0.5) / h.q;
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const R xr = x[r] * h.xs;
        const R b00 = xr * inv2pq;
        const R b10 = (R(1) - xr * qpq) * inv2p;
        const R b01 = (R(1) - xr * ppq) * inv2q;
        const R cq = xr * qpq, cp = xr * ppq;
        R gx[NEV + 1][NFV + 1], gy[NEV + 1][NFV + 1], gz[NEV + 1][NFV + 1];
        vrr_axis<NEV, NFV, R>(R(1), h.pax - cq * h.pqx, h.qcx + cp * h.pqx, b10, b01, b00, gx);
        vrr_axis<NEV, NFV, R>(R(1), h.pay - cq * h.pqy, h.qcy + cp * h.pqy, b10, b01, b00, gy);
        vrr_axis<NEV, NFV, R>(w[r] * h.pref, h.paz - cq * h.pqz, h.qcz + cp * h.pqz, b10, b01, b00, gz);
        if constexpr (GS::LOW) {
          static_for<R0>([&](auto e) {
            constexpr int ex = range_x(E0, decltype(e)::value), ey = range_y(E0, decltype(e)::value),
                          ez = range_z(E0, decltype(e)::value);
            static_for<C0>([&](auto f) {
              constexpr int fx = range_x(F0, decltype(f)::value), fy = range_y(F0, decltype(f)::value),
                            fz = range_z(F0, decltype(f)::value);
              aP[decltype(e)::value * C0 + decltype(f)::value] += gx[ex][fx] * gy[ey][fy] * gz[ez][fz];
            });
          });
        }
        static_for<R1>([&](auto e) {
          constexpr int ex = range_x(E1, decltype(e)::value), ey = range_y(E1, decltype(e)::value),
                        ez = range_z(E1, decltype(e)::value);
          static_for<C1>([&](auto f) {
            constexpr int fx = range_x(F1, decltype(f)::value), fy = range_y(F1, decltype(f)::value),
                          fz = range_z(F1, decltype(f)::value);
            const R v = gx[ex][fx] * gy[ey][fy] * gz[ez][fz];
            constexpr int q = decltype(e)::value * C1 + decltype(f)::value;
            aA[q] += wA * v;
            aB[q] += wB * v;
          });
        });
        static_for<R2>([&](auto e) {
          constexpr int ex = range_x(E2, decltype(e)::value), ey = range_y(E2, decltype(e)::value),
                        ez = range_z(E2, decltype(e)::value);
          static_for<C2>([&](auto f) {
            constexpr int fx = range_x(F2, decltype(f)::value), fy = range_y(F2, decltype(f)::value),
                          fz = range_z(F2, decltype(f)::value);
            aC[decltype(e)::value * C2 + decltype(f)::value] += wC * (gx[ex][fx] * gy[ey][fy] * gz[ez][fz]);
          });
        });
      }
    }
  }
  const GradSlot L = grad_slot_layout(LA, LB, LC, LD);
  if constexpr (GS::LOW) {
#pragma unroll
    for (int q = 0; q < NP; ++q) tab[L.off_p + q] = (double)aP[q];
  }
  constexpr int SKIP = ncart(LA);  // rows of degree la are not part of table A
#pragma unroll
  for (int q = SKIP * C1; q < R1 * C1; ++q) tab[L.off_a + q - SKIP * C1] = (double)aA[q];
#pragma unroll
  for (int q = 0; q < R1 * C1; ++q) tab[L.off_b + q] = (double)aB[q];
#pragma unroll
  for (int q = 0; q < R2 * C2; ++q) tab[L.off_c + q] = (double)aC[q];
}

// -------------------------------------------------------- phase 1, team

template <int LA, int LB, int LC, int LD, typename R, int PASS>
__device__ __forceinline__ void grad_team_pass(const KernelArgs& A, const R* s_tab, const PairD& pb, const PairD& pk,
                                               R* sm, int lane, unsigned tmask, double* tab) {
  using GS = GradShape<LA, LB, LC, LD, R>;
  constexpr int NEV = GS::NEV, NFV = GS::NFV, NR = GS::NR, T = GS::T, GT = GS::GT;
  constexpr int I0 = GS::PL.pbeg[PASS], I1 = GS::PL.pbeg[PASS + 1];
  constexpr int NACC = GS::PL.pacc[PASS], NROW = GS::PL.prows[PASS];
  R acc[NACC];
#pragma unroll
  for (int q = 0; q < NACC; ++q) acc[q] = R(0);
  // row offsets into the per-axis tables: e components of every row slot
  int ox[NROW], oy[NROW], oz[NROW];
  static_for<I1 - I0>([&](auto ii) {
    constexpr int I = I0 + decltype(ii)::value;
    constexpr int s = GS::PL.seg[I];
    constexpr int EA = g_ea(LA, LB, LC, LD, s), ROWS = g_rows(LA, LB, LC, LD, s);
    constexpr int RL = (ROWS + T - 1) / T, RS = GS::PL.rslot[I];
#pragma unroll
    for (int k = 0; k < RL; ++k) {
      const int row = lane + T * k;
      const int a = tri_below(EA) + (row < ROWS ? row : 0);
      ox[RS + k] = addr_lx(a) * (NFV + 1);
      oy[RS + k] = addr_ly(a) * (NFV + 1);
      oz[RS + k] = addr_lz(a) * (NFV + 1);
    }
  });
  constexpr int BP = GS::BP, SUB = GS::SUB, PT = GS::PRIM_TAB;
  const int npk = pk.nprim;
  const int npr = pb.nprim * npk;
  const int myp = lane % BP;
  const int sub = lane / BP;
  for (int base = 0; base < npr; base += BP) {
    const int nb = npr - base < BP ? npr - base : BP;
    const bool active = myp < nb;
    R* mys = sm + myp * PT;
    QuartetHdr<R> h;
    if (active) {
      const int pidx = base + myp;
      const int ip = pidx / npk, kq = pidx - ip * npk;
      const PrimPairD bp = A.prims[pb.prim_off + ip];
      const PrimPairD kp = A.prims[pk.prim_off + kq];
      h = quartet_header<R>(bp, kp, A.omega);
      for (int r = sub; r < NR; r += SUB) {
        R xr, wr;
        rys_root_one<NR, R>(s_tab, h.T, r, xr, wr);
        mys[r] = xr * h.xs;
        mys[NR + r] = wr * h.pref;
      }
      if (sub == 0) {
        mys[2 * NR] = R(2) * R(bp.alpha);
        mys[2 * NR + 1] = R(2) * R(bp.beta);
        mys[2 * NR + 2] = R(2) * R(kp.alpha);
      }
    }
    __syncwarp(tmask);
    if (active) {
      const R inv_pq = R(1) / h.pq;
      const R qpq = h.q * inv_pq, ppq = h.p * inv_pq;
      const R inv2p = R(0.5) / h.p, inv2q = R(0.5) / h.q;
      for (int t = sub; t < 3 * NR; t += SUB) {
        const int axis = t / NR, r = t - axis * NR;
        const R xr = mys[r];
        const R b00 = xr * R(0.5) * inv_pq;
        const R b10 = (R(1) - xr * qpq) * inv2p;
        const R b01 = (R(1) - xr * ppq) * inv2q;
        const R pqa = axis == 0 ? h.pqx : (axis == 1 ? h.pqy : h.pqz);
        const R paa = axis == 0 ? h.pax : (axis == 1 ? h.pay : h.paz);
        const R qca = axis == 0 ? h.qcx : (axis == 1 ? h.qcy : h.qcz);
        R g[NEV + 1][NFV + 1];
        vrr_axis<NEV, NFV, R>(axis == 2 ? mys[NR + r] : R(1), paa - xr * qpq * pqa, qca + xr * ppq * pqa, b10, b01,
                              b00, g);
        R* dst = mys + 2 * NR + 3 + (axis * NR + r) * GT;
#pragma unroll
        for (int n = 0; n <= NEV; ++n)
#pragma unroll
          for (int m = 0; m <= NFV; ++m) dst[n * (NFV + 1) + m] = g[n][m];
      }
    }
    __syncwarp(tmask);
    for (int p = 0; p < nb; ++p) {
      const R* pt = sm + p * PT;
      const R wA = pt[2 * NR], wB = pt[2 * NR + 1], wC = pt[2 * NR + 2];
      const R* gt = pt + 2 * NR + 3;
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const R* tx = gt + (0 * NR + r) * GT;
        const R* ty = gt + (1 * NR + r) * GT;
        const R* tz = gt + (2 * NR + r) * GT;
        static_for<I1 - I0>([&](auto ii) {
          constexpr int I = I0 + decltype(ii)::value;
          constexpr int s = GS::PL.seg[I], FF = GS::PL.f0[I], FW = GS::PL.fw[I], OFF = GS::PL.off[I];
          constexpr int FA = g_fa(LA, LB, LC, LD, s), ROWS = g_rows(LA, LB, LC, LD, s);
          constexpr int RL = (ROWS + T - 1) / T, RS = GS::PL.rslot[I];
#pragma unroll
          for (int k = 0; k < RL; ++k) {
            if (RL * T > ROWS && lane + T * k >= ROWS) continue;
            R rx[NFV + 1], ry[NFV + 1], rz[NFV + 1];
#pragma unroll
            for (int m = 0; m <= NFV; ++m) {
              rx[m] = tx[ox[RS + k] + m];
              ry[m] = ty[oy[RS + k] + m];
              rz[m] = tz[oz[RS + k] + m];
            }
            if constexpr (s == 2) {
#pragma unroll
              for (int m = 0; m <= NFV; ++m) rz[m] *= wC;
            }
            static_for<FW>([&](auto f) {
              constexpr int fi = FF + decltype(f)::value;
              constexpr int fx = range_x(FA, fi), fy = range_y(FA, fi), fz = range_z(FA, fi);
              const R v = rx[fx] * ry[fy] * rz[fz];
              if constexpr (s == 1) {
                acc[OFF + (k * FW + decltype(f)::value) * 2] += wA * v;
                acc[OFF + (k * FW + decltype(f)::value) * 2 + 1] += wB * v;
              } else {
                acc[OFF + k * FW + decltype(f)::value] += v;
              }
            });
          }
        });
      }
    }
    __syncwarp(tmask);
  }
  const GradSlot L = grad_slot_layout(LA, LB, LC, LD);
  static_for<I1 - I0>([&](auto ii) {
    constexpr int I = I0 + decltype(ii)::value;
    constexpr int s = GS::PL.seg[I], FF = GS::PL.f0[I], FW = GS::PL.fw[I], OFF = GS::PL.off[I];
    constexpr int ROWS = g_rows(LA, LB, LC, LD, s), COLS = g_cols(LA, LB, LC, LD, s);
    constexpr int RL = (ROWS + T - 1) / T;
#pragma unroll
    for (int k = 0; k < RL; ++k) {
      const int row = lane + T * k;
      if (row >= ROWS) continue;
#pragma unroll
      for (int f = 0; f < FW; ++f) {
        if constexpr (s == 0) {
          tab[L.off_p + (size_t)row * COLS + FF + f] = (double)acc[OFF + k * FW + f];
        } else if constexpr (s == 1) {
          tab[L.off_b + (size_t)row * COLS + FF + f] = (double)acc[OFF + (k * FW + f) * 2 + 1];
          if (row >= ncart(LA))
            tab[L.off_a + (size_t)(row - ncart(LA)) * COLS + FF + f] = (double)acc[OFF + (k * FW + f) * 2];
        } else {
          tab[L.off_c + (size_t)row * COLS + FF + f] = (double)acc[OFF + k * FW + f];
        }
      }
    }
  });
}

template <int LA, int LB, int LC, int LD, typename R, int PASS>
__device__ __forceinline__ void grad_team_passes(const KernelArgs& A, const R* s_tab, const PairD& pb,
                                                 const PairD& pk, R* sm, int lane, unsigned tmask, double* tab) {
  using GS = GradShape<LA, LB, LC, LD, R>;
  if constexpr (PASS < GS::PL.npass) {
    grad_team_pass<LA, LB, LC, LD, R, PASS>(A, s_tab, pb, pk, sm, lane, tmask, tab);
    __syncwarp(tmask);
    grad_team_passes<LA, LB, LC, LD, R, PASS + 1>(A, s_tab, pb, pk, sm, lane, tmask, tab);
  }
}

// ------------------------------------------------------------- phase 2

// Degeneracy-scaled two-particle density block of the quartet in
// evaluation orientation (src/direct_grad.rs:490-547).  Each element is
// evaluated with the AO indices of the reference orientation (i,j,k,l), so
// the block is the reference's even for non-symmetric term matrices; then
// every spherical axis is pulled back to Cartesian components through the
// transposed c2s matrix.  Returns the buffer holding the Cartesian block.
__device__ __forceinline__ const double* grad_weight_block(const KernelArgs& A, const PairD& pb, const PairD& pk,
                                                           const Screen& sc, double* W0, double* W1, int lane, int T,
                                                           unsigned tmask) {
  const DevShell d[4] = {A.shells[pb.a], A.shells[pb.b], A.shells[pk.a], A.shells[pk.b]};
  const int bb = sc.swapped ? 2 : 0, kb = sc.swapped ? 0 : 2;
  int rp[4];
  rp[0] = bb + (pb.a == pb.i ? 0 : 1);
  rp[1] = bb + (pb.a == pb.i ? 1 : 0);
  rp[2] = kb + (pk.a == pk.i ? 0 : 1);
  rp[3] = kb + (pk.a == pk.i ? 1 : 0);
  const int nf[4] = {d[0].nfunc, d[1].nfunc, d[2].nfunc, d[3].nfunc};
  const int total = nf[0] * nf[1] * nf[2] * nf[3];
  const size_t n = (size_t)A.nao;
  const GradDev& G = A.grad;
  const double deg = sc.degeneracy;
  for (int q = lane; q < total; q += T) {
    int f[4];
    f[3] = q % nf[3];
    int r = q / nf[3];
    f[2] = r % nf[2];
    r /= nf[2];
    f[1] = r % nf[1];
    f[0] = r / nf[1];
    size_t m[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) m[rp[p]] = (size_t)(d[p].off + f[p]);
    double w = 0.0;
    for (int t = 0; t < G.ncoul; ++t) {
      const double* Lm = G.cl[t];
      const double* Rm = G.cr[t];
      const double fac = 0.5 * deg * __ldg(G.cf + t);
      w += fac * (__ldg(Lm + m[0] * n + m[1]) * __ldg(Rm + m[2] * n + m[3]) +
                  __ldg(Rm + m[0] * n + m[1]) * __ldg(Lm + m[2] * n + m[3]));
    }
    for (int t = 0; t < G.nexch; ++t) {
      const double* Lm = G.xl[t];
      const double* Rm = G.xr[t];
      const double fac = 0.25 * deg * __ldg(G.xf + t);
      w += fac * (__ldg(Lm + m[0] * n + m[2]) * __ldg(Rm + m[1] * n + m[3]) +
                  __ldg(Lm + m[1] * n + m[2]) * __ldg(Rm + m[0] * n + m[3]) +
                  __ldg(Lm + m[0] * n + m[3]) * __ldg(Rm + m[1] * n + m[2]) +
                  __ldg(Lm + m[1] * n + m[3]) * __ldg(Rm + m[0] * n + m[2]));
    }
    W0[q] = w;
  }
  __syncwarp(tmask);
  int dims[4] = {nf[0], nf[1], nf[2], nf[3]};
  double* cur = W0;
  double* oth = W1;
  for (int axis = 0; axis < 4; ++axis) {
    if (!d[axis].spherical) continue;
    const int l = d[axis].l;
    const int n_in = dims[axis], n_out = ncart(l);
    const double* M = A.c2s + A.c2s_off[l];  // (2l+1) x ncart(l)
    int outer = 1, inner = 1;
    for (int q = 0; q < axis; ++q) outer *= dims[q];
    for (int q = axis + 1; q < 4; ++q) inner *= dims[q];
    const int tot = outer * n_out * inner;
    for (int q = lane; q < tot; q += T) {
      const int s = q % inner;
      const int r = q / inner;
      const int o = r / n_out, j = r % n_out;
      double acc = 0.0;
      for (int mm = 0; mm < n_in; ++mm) {
        const double c = __ldg(M + mm * n_out + j);
        if (c != 0.0) acc += c * cur[((size_t)o * n_in + mm) * inner + s];
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

// g[axis] += sum over the Cartesian W block of W * (raised or lowered block
// element of the shifted component on axis `pos`).
__device__ __forceinline__ void grad_dot(const double* W, const double* blk, const int ls[4], int pos, bool raised,
                                         double g[3], int lane, int T) {
  const int nc[4] = {ncart(ls[0]), ncart(ls[1]), ncart(ls[2]), ncart(ls[3])};
  int inner = 1;
  for (int q = pos + 1; q < 4; ++q) inner *= nc[q];
  const int np = nc[pos];
  const int total = nc[0] * nc[1] * nc[2] * nc[3];
  const int lp = ls[pos];
  const int nsh = raised ? ncart(lp + 1) : ncart(lp - 1);
  const int base = tri_below(lp);
  for (int q = lane; q < total; q += T) {
    const double w = W[q];
    if (w == 0.0) continue;
    const int s = q % inner;
    const int r = q / inner;
    const int a = r % np, o = r / np;
    const int ax = addr_lx(base + a), ay = addr_ly(base + a), az = addr_lz(base + a);
    const size_t rowb = (size_t)o * nsh;
    if (raised) {
      g[0] += w * blk[(rowb + cart_index3(ax + 1, ay, az)) * inner + s];
      g[1] += w * blk[(rowb + cart_index3(ax, ay + 1, az)) * inner + s];
      g[2] += w * blk[(rowb + cart_index3(ax, ay, az + 1)) * inner + s];
    } else {
      if (ax > 0) g[0] -= (double)ax * w * blk[(rowb + cart_index3(ax - 1, ay, az)) * inner + s];
      if (ay > 0) g[1] -= (double)ay * w * blk[(rowb + cart_index3(ax, ay - 1, az)) * inner + s];
      if (az > 0) g[2] -= (double)az * w * blk[(rowb + cart_index3(ax, ay, az - 1)) * inner + s];
    }
  }
}

// One shifted block: copy its [e0|f0] slice into the first HRR buffer, run
// the bra and ket recurrences, dot with W.
__device__ __forceinline__ void grad_shifted(const double* tabp, int tab_cols, int row_off, int nrows, int col_off,
                                             int ncols, const int bls[4], const int ls[4], int pos, bool raised,
                                             const double* W, double* buf[3], double* blk, const double ab[3],
                                             const double cd[3], double g[3], int lane, int T, unsigned tmask) {
  for (int q = lane; q < nrows * ncols; q += T) {
    const int r = q / ncols, c = q % ncols;
    buf[0][q] = tabp[(size_t)(row_off + r) * tab_cols + col_off + c];
  }
  __syncwarp(tmask);
  int cur = 0;
  hrr_bra(buf, cur, bls[0], bls[1], ncols, ab, lane, T, tmask);
  hrr_ket(buf, cur, blk, bls[0], bls[1], bls[2], bls[3], ncols, cd, lane, T, tmask);
  grad_dot(W, blk, ls, pos, raised, g, lane, T);
  __syncwarp(tmask);
}

// Phase 2 of one quartet: g[3*pos + axis] for evaluation positions 0..2
// (this lane's partial sums).
__device__ __forceinline__ void grad_post(const KernelArgs& A, int la, int lb, int lc, int ld, const PairD& pb,
                                          const PairD& pk, const Screen& sc, double* slot, double g[9], int lane,
                                          int T, unsigned tmask) {
  const GradSlot L = grad_slot_layout(la, lb, lc, ld);
  double* W0 = slot + L.ntab;
  double* W1 = W0 + L.W;
  double* buf[3] = {W1 + L.W, W1 + L.W + L.S, W1 + L.W + 2 * L.S};
  double* blk = W1 + L.W + 3 * L.S;
  const double* W = grad_weight_block(A, pb, pk, sc, W0, W1, lane, T, tmask);
  const double ab[3] = {pb.abx, pb.aby, pb.abz};
  const double cd[3] = {pk.abx, pk.aby, pk.abz};
  const int ls[4] = {la, lb, lc, ld};
  const int ne = la + lb, nf = lc + ld;
  const int ea0 = la > 0 ? la - 1 : 0, fa0 = lc > 0 ? lc - 1 : 0;
  const int colsP = nrange(fa0, nf);
  const int cols1 = nrange(lc, nf);
  const int cols2 = nrange(lc + 1, nf + 1);
#pragma unroll 1
  for (int q = 0; q < 9; ++q) g[q] = 0.0;
  // position A
  {
    const int b[4] = {la + 1, lb, lc, ld};
    grad_shifted(slot + L.off_a, cols1, 0, nrange(la + 1, ne + 1), 0, cols1, b, ls, 0, true, W, buf, blk, ab, cd, g,
                 lane, T, tmask);
  }
  if (la > 0) {
    const int b[4] = {la - 1, lb, lc, ld};
    grad_shifted(slot + L.off_p, colsP, 0, nrange(la - 1, ne - 1), tri_below(lc) - tri_below(fa0), cols1, b, ls, 0,
                 false, W, buf, blk, ab, cd, g, lane, T, tmask);
  }
  // position B
  {
    const int b[4] = {la, lb + 1, lc, ld};
    grad_shifted(slot + L.off_b, cols1, 0, nrange(la, ne + 1), 0, cols1, b, ls, 1, true, W, buf, blk, ab, cd, g + 3,
                 lane, T, tmask);
  }
  if (lb > 0) {
    const int b[4] = {la, lb - 1, lc, ld};
    grad_shifted(slot + L.off_p, colsP, tri_below(la) - tri_below(ea0), nrange(la, ne - 1),
                 tri_below(lc) - tri_below(fa0), cols1, b, ls, 1, false, W, buf, blk, ab, cd, g + 3, lane, T, tmask);
  }
  // position C
  {
    const int b[4] = {la, lb, lc + 1, ld};
    grad_shifted(slot + L.off_c, cols2, 0, nrange(la, ne), 0, cols2, b, ls, 2, true, W, buf, blk, ab, cd, g + 6, lane,
                 T, tmask);
  }
  if (lc > 0) {
    const int b[4] = {la, lb, lc - 1, ld};
    grad_shifted(slot + L.off_p, colsP, tri_below(la) - tri_below(ea0), nrange(la, ne), 0, nrange(lc - 1, nf - 1), b,
                 ls, 2, false, W, buf, blk, ab, cd, g + 6, lane, T, tmask);
  }
}

// ------------------------------------------ phase 2, Cartesian classes

__host__ __device__ constexpr int cidx(int lx, int ly, int lz) { return (ly + lz) * (ly + lz + 1) / 2 + lz; }

// Weight block of an all-Cartesian quartet with compile-time dims (same
// values as grad_weight_block).  The reference-orientation AO index of each
// element is picked by selects, not by indexing a local array.
template <int LA, int LB, int LC, int LD, int T>
__device__ __forceinline__ void grad_weight_block_cart(const KernelArgs& A, const PairD& pb, const PairD& pk,
                                                       const Screen& sc, double* W, int lane) {
  constexpr int N0 = ncart(LA), N1 = ncart(LB), N2 = ncart(LC), N3 = ncart(LD);
  const int o0 = A.shells[pb.a].off, o1 = A.shells[pb.b].off, o2 = A.shells[pk.a].off, o3 = A.shells[pk.b].off;
  // evaluation position of reference positions 0..3
  const int bb = sc.swapped ? 2 : 0, kb = sc.swapped ? 0 : 2;
  const bool bflip = pb.a != pb.i, kflip = pk.a != pk.i;
  const int e0 = bb == 0 ? (bflip ? 1 : 0) : (kflip ? 3 : 2);  // eval slot of reference i
  const int e1 = bb == 0 ? (bflip ? 0 : 1) : (kflip ? 2 : 3);  // of j
  const int e2 = kb == 2 ? (kflip ? 3 : 2) : (bflip ? 1 : 0);  // of k
  const int e3 = kb == 2 ? (kflip ? 2 : 3) : (bflip ? 0 : 1);  // of l
  const size_t n = (size_t)A.nao;
  const GradDev& G = A.grad;
  const double deg = sc.degeneracy;
  for (int q = lane; q < N0 * N1 * N2 * N3; q += T) {
    const int f3 = q % N3, f2 = (q / N3) % N2, f1 = (q / (N3 * N2)) % N1, f0 = q / (N3 * N2 * N1);
    const size_t x0 = o0 + f0, x1 = o1 + f1, x2 = o2 + f2, x3 = o3 + f3;
    auto pick = [&](int e) { return e == 0 ? x0 : (e == 1 ? x1 : (e == 2 ? x2 : x3)); };
    const size_t m0 = pick(e0), m1 = pick(e1), m2 = pick(e2), m3 = pick(e3);
    double w = 0.0;
    for (int t = 0; t < G.ncoul; ++t) {
      const double* Lm = G.cl[t];
      const double* Rm = G.cr[t];
      const double fac = 0.5 * deg * __ldg(G.cf + t);
      w += fac * (__ldg(Lm + m0 * n + m1) * __ldg(Rm + m2 * n + m3) + __ldg(Rm + m0 * n + m1) * __ldg(Lm + m2 * n + m3));
    }
    for (int t = 0; t < G.nexch; ++t) {
      const double* Lm = G.xl[t];
      const double* Rm = G.xr[t];
      const double fac = 0.25 * deg * __ldg(G.xf + t);
      w += fac * (__ldg(Lm + m0 * n + m2) * __ldg(Rm + m1 * n + m3) + __ldg(Lm + m1 * n + m2) * __ldg(Rm + m0 * n + m3) +
                  __ldg(Lm + m0 * n + m3) * __ldg(Rm + m1 * n + m2) + __ldg(Lm + m1 * n + m3) * __ldg(Rm + m0 * n + m2));
    }
    W[q] = w;
  }
}

// grad_dot with the shapes fixed at compile time: lanes take the (outer,
// inner) index pairs around axis POS, the components along POS are unrolled
// with their shifted indices known at compile time.
template <int L0, int L1, int L2, int L3, int POS, bool RAISED, int T>
__device__ __forceinline__ void grad_dot_ct(const double* W, const double* blk, double g[3], int lane) {
  constexpr int LS[4] = {L0, L1, L2, L3};
  constexpr int NC[4] = {ncart(L0), ncart(L1), ncart(L2), ncart(L3)};
  constexpr int LP = LS[POS], NP = NC[POS];
  constexpr int INNER = (POS < 3 ? NC[3] : 1) * (POS < 2 ? NC[2] : 1) * (POS < 1 ? NC[1] : 1);
  constexpr int OUTER = (NC[0] * NC[1] * NC[2] * NC[3]) / (NP * INNER);
  constexpr int NSH = RAISED ? ncart(LP + 1) : (LP > 0 ? ncart(LP - 1) : 1);
  for (int os = lane; os < OUTER * INNER; os += T) {
    const int o = os / INNER, s = os - (os / INNER) * INNER;
    const double* wr = W + (size_t)o * NP * INNER + s;
    const double* br = blk + (size_t)o * NSH * INNER + s;
    static_for<NP>([&](auto ai) {
      constexpr int a = decltype(ai)::value;
      constexpr int ax = comp_lx(LP, a), ay = comp_ly(LP, a), az = comp_lz(LP, a);
      const double w = wr[a * INNER];
      if constexpr (RAISED) {
        g[0] += w * br[cidx(ax + 1, ay, az) * INNER];
        g[1] += w * br[cidx(ax, ay + 1, az) * INNER];
        g[2] += w * br[cidx(ax, ay, az + 1) * INNER];
      } else {
        if constexpr (ax > 0) g[0] -= double(ax) * w * br[cidx(ax - 1, ay, az) * INNER];
        if constexpr (ay > 0) g[1] -= double(ay) * w * br[cidx(ax, ay - 1, az) * INNER];
        if constexpr (az > 0) g[2] -= double(az) * w * br[cidx(ax, ay, az - 1) * INNER];
      }
    });
  }
}

template <int L0, int L1, int L2, int L3, int POS, bool RAISED, int T>
__device__ __forceinline__ void grad_shifted_ct(const double* tabp, int tab_cols, int row_off, int nrows, int col_off,
                                                const double* W, double* buf[3], double* blk, const double ab[3],
                                                const double cd[3], double g[3], int lane, unsigned tmask) {
  constexpr int NCOLS = nrange(L2, L2 + L3);
  for (int q = lane; q < nrows * NCOLS; q += T) {
    const int r = q / NCOLS, c = q - (q / NCOLS) * NCOLS;
    buf[0][q] = tabp[(size_t)(row_off + r) * tab_cols + col_off + c];
  }
  __syncwarp(tmask);
  int cur = 0;
  hrr_bra(buf, cur, L0, L1, NCOLS, ab, lane, T, tmask);
  hrr_ket(buf, cur, blk, L0, L1, L2, L3, NCOLS, cd, lane, T, tmask);
  constexpr int LS[4] = {L0, L1, L2, L3};
  constexpr int D0 = POS == 0 ? (RAISED ? -1 : 1) : 0, D1 = POS == 1 ? (RAISED ? -1 : 1) : 0;
  constexpr int D2 = POS == 2 ? (RAISED ? -1 : 1) : 0;
  // W and the dot use the unshifted shells
  grad_dot_ct<L0 + D0, L1 + D1, L2 + D2, L3, POS, RAISED, T>(W, blk, g, lane);
  (void)LS;
  __syncwarp(tmask);
}

// Phase 2 of an all-Cartesian quartet (grad_post with compile-time shapes).
template <int LA, int LB, int LC, int LD, int T>
__device__ __forceinline__ void grad_post_cart(const KernelArgs& A, const PairD& pb, const PairD& pk, const Screen& sc,
                                               double* slot, double g[9], int lane, unsigned tmask) {
  const GradSlot L = grad_slot_layout(LA, LB, LC, LD);
  double* W = slot + L.ntab;
  double* buf[3] = {W + 2 * L.W, W + 2 * L.W + L.S, W + 2 * L.W + 2 * L.S};
  double* blk = W + 2 * L.W + 3 * L.S;
  grad_weight_block_cart<LA, LB, LC, LD, T>(A, pb, pk, sc, W, lane);
  __syncwarp(tmask);
  const double ab[3] = {pb.abx, pb.aby, pb.abz};
  const double cd[3] = {pk.abx, pk.aby, pk.abz};
  constexpr int NE = LA + LB, NF = LC + LD;
  constexpr int EA0 = LA > 0 ? LA - 1 : 0, FA0 = LC > 0 ? LC - 1 : 0;
  constexpr int COLSP = nrange(FA0, NF), COLS1 = nrange(LC, NF), COLS2 = nrange(LC + 1, NF + 1);
#pragma unroll 1
  for (int q = 0; q < 9; ++q) g[q] = 0.0;
  grad_shifted_ct<LA + 1, LB, LC, LD, 0, true, T>(slot + L.off_a, COLS1, 0, nrange(LA + 1, NE + 1), 0, W, buf, blk,
                                                  ab, cd, g, lane, tmask);
  if constexpr (LA > 0)
    grad_shifted_ct<LA - 1, LB, LC, LD, 0, false, T>(slot + L.off_p, COLSP, 0, nrange(LA - 1, NE - 1),
                                                     tri_below(LC) - tri_below(FA0), W, buf, blk, ab, cd, g, lane,
                                                     tmask);
  grad_shifted_ct<LA, LB + 1, LC, LD, 1, true, T>(slot + L.off_b, COLS1, 0, nrange(LA, NE + 1), 0, W, buf, blk, ab,
                                                  cd, g + 3, lane, tmask);
  if constexpr (LB > 0)
    grad_shifted_ct<LA, LB - 1, LC, LD, 1, false, T>(slot + L.off_p, COLSP, tri_below(LA) - tri_below(EA0),
                                                     nrange(LA, NE - 1), tri_below(LC) - tri_below(FA0), W, buf, blk,
                                                     ab, cd, g + 3, lane, tmask);
  grad_shifted_ct<LA, LB, LC + 1, LD, 2, true, T>(slot + L.off_c, COLS2, 0, nrange(LA, NE), 0, W, buf, blk, ab, cd,
                                                  g + 6, lane, tmask);
  if constexpr (LC > 0)
    grad_shifted_ct<LA, LB, LC - 1, LD, 2, false, T>(slot + L.off_p, COLSP, tri_below(LA) - tri_below(EA0),
                                                     nrange(LA, NE), 0, W, buf, blk, ab, cd, g + 6, lane, tmask);
}

// --------------------------------------------------------------- kernel

template <int LA, int LB, int LC, int LD, typename R>
__global__ void __launch_bounds__(128) grad_kernel(KernelArgs A) {
  using GS = GradShape<LA, LB, LC, LD, R>;
  constexpr int T = GS::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ R s_tab[GS::NR * RYS_MAX_SUB * 2 * RYS_NC];
  stage_rys_table<GS::NR, R>(s_tab);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int team = tid / T;
  const int lane = threadIdx.x % T;
  const unsigned tmask = T == 32 ? 0xffffffffu : (((1u << T) - 1u) << ((threadIdx.x % 32) / T * T));
  R* sm = reinterpret_cast<R*>(smem_raw) + (size_t)(threadIdx.x / T) * GS::SMEM_PER_TEAM;
  double* slot = A.scratch + (size_t)team * A.slot_doubles;
  QuartetCounters cnt;
  double* out = A.grad.out;
  // running derivative on the two bra centres (lane 0), flushed when the
  // team moves to another bra pair
  int cur_bra = -1, atom_a = 0, atom_b = 0;
  double gb[6] = {0, 0, 0, 0, 0, 0};
  auto flush_bra = [&]() {
    if (cur_bra >= 0) {
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        if (gb[x] != 0.0) atomicAdd(out + (size_t)atom_a * 3 + x, gb[x]);
        if (gb[3 + x] != 0.0) atomicAdd(out + (size_t)atom_b * 3 + x, gb[3 + x]);
        gb[x] = gb[3 + x] = 0.0;
      }
    }
  };
  constexpr int TPW = 32 / T;
  const int tw = (threadIdx.x & 31) / T;
  for (;;) {
    unsigned long long base = 0;
    if ((threadIdx.x & 31) == 0) base = atomicAdd(A.work_counter, A.chunk);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= A.task.total) break;
    const unsigned long long end = base + A.chunk < A.task.total ? base + A.chunk : A.task.total;
    TaskCursor cur;
    if (base + tw < end) cursor_seek(A.task, base + tw, cur);
    for (unsigned long long t = base + tw; t < end; t += TPW) {
      int pbi, pki;
      cursor_decode(A.task, t, cur, pbi, pki);
      const PairD pb = A.pairs[pbi];
      const PairD pk = A.pairs[pki];
      const Screen sc = screen_quartet(A, pb, pk);
      if (!sc.keep) continue;
      if (lane == 0) cnt.add(sc, pb, pk, A.fp32);
      if constexpr (T == 1)
        grad_tables_thread<LA, LB, LC, LD, R>(A, s_tab, pb, pk, slot);
      else
        grad_team_passes<LA, LB, LC, LD, R, 0>(A, s_tab, pb, pk, sm, lane, tmask, slot);
      __syncwarp(tmask);
      double g[9];
      if (A.kinds == 0)
        grad_post_cart<LA, LB, LC, LD, T>(A, pb, pk, sc, slot, g, lane, tmask);
      else
        grad_post(A, LA, LB, LC, LD, pb, pk, sc, slot, g, lane, T, tmask);
      if constexpr (T > 1) {
#pragma unroll
        for (int q = 0; q < 9; ++q)
#pragma unroll
          for (int o = T / 2; o > 0; o >>= 1) g[q] += __shfl_xor_sync(tmask, g[q], o, T);
      }
      if (lane == 0) {
        if (pbi != cur_bra) {
          flush_bra();
          cur_bra = pbi;
          atom_a = A.shells[pb.a].atom;
          atom_b = A.shells[pb.b].atom;
        }
#pragma unroll
        for (int x = 0; x < 6; ++x) gb[x] += g[x];
        const int atom_c = A.shells[pk.a].atom, atom_d = A.shells[pk.b].atom;
#pragma unroll
        for (int x = 0; x < 3; ++x) {
          atomicAdd(out + (size_t)atom_c * 3 + x, g[6 + x]);
          atomicAdd(out + (size_t)atom_d * 3 + x, -(g[x] + g[3 + x] + g[6 + x]));
        }
      }
      __syncwarp(tmask);
    }
  }
  if (lane == 0) flush_bra();
  cnt.flush(A.counters);
}

}  // namespace igpu
