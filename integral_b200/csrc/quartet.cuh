// Shell-quartet kernels of the two-electron path.
//
// One launch handles one angular class (la,lb|lc,ld) in evaluation
// orientation (la >= lb, lc >= ld, bra class >= ket class) over a task list
// of (bra pair, ket pair) quartets that survived the Schwarz product screen.
//
// Phase 1 builds the contracted table G[e][f] = sum over primitive quartets
// and Rys roots of Ix[ex][fx] Iy[ey][fy] Iz[ez][fz] (the [e0|f0] integrals,
// e of degree la..la+lb on A, f of degree lc..lc+ld on C) by Rys quadrature
// with the vertical recurrence of src/engine/rys.rs:234-268.  Doing the
// horizontal recurrence once per shell quartet on the contracted table is the
// early-contraction scheme of the reference's OS/HGP engine
// (src/engine/os_eri.rs:1-12) applied to Rys 2D integrals.
//   TEAM == 1 : one thread per quartet, everything in registers.
//   TEAM >= 2 : a team of TEAM lanes per quartet; roots and the 3*nroots
//               per-axis tables are built cooperatively in shared memory and
//               every lane accumulates its own rows e of G (register tiles
//               of FCH columns, the f range walked in chunks).
// The class's Rys Chebyshev table is staged in shared memory per block.
// Phase 2 (post.cuh) runs the horizontal recurrences, the Cartesian ->
// spherical transform and the mode-specific consumer on the team.
#pragma once
#include "device_common.cuh"
#include "post.cuh"
#include "post_thread.cuh"

namespace igpu {

template <int LA, int LB, int LC, int LD>
struct ClassShape {
  static constexpr int NE = LA + LB;
  static constexpr int NF = LC + LD;
  static constexpr int LT = NE + NF;
  static constexpr int NR = LT / 2 + 1;
  static constexpr int NEP = nrange(LA, NE);
  static constexpr int NFP = nrange(LC, NF);
  static constexpr int NG = NEP * NFP;
};

// Lanes per quartet: one thread while the whole G table fits in registers,
// otherwise the smallest team of 8, 16 or 32 lanes covering the rows (teams
// of 2 or 4 lanes measured slower: the per-primitive root and recurrence
// work is then spread over too few lanes).
__host__ __device__ constexpr int team_for(int nep, int nfp) {
  if (nep * nfp <= 81) return 1;
  if (nep <= 8) return 8;
  if (nep <= 16) return 16;
  return 32;
}
template <int LA, int LB, int LC, int LD>
__host__ __device__ constexpr int team_size() {
  return team_for(nrange(LA, LA + LB), nrange(LC, LC + LD));
}

// Phase-1 register footprint per lane: rows x FCH accumulators.
template <typename R>
__host__ __device__ constexpr int max_acc() { return sizeof(R) == 8 ? 64 : 96; }

template <int LA, int LB, int LC, int LD, typename R>
struct TeamShape {
  using S = ClassShape<LA, LB, LC, LD>;
  static constexpr int T = team_size<LA, LB, LC, LD>();
  static constexpr int ROWS = (S::NEP + T - 1) / T;
  static constexpr int FCH0 = max_acc<R>() / ROWS;
  static constexpr int FCH = FCH0 < 1 ? 1 : (FCH0 > S::NFP ? S::NFP : FCH0);
  static constexpr int NCHUNK = (S::NFP + FCH - 1) / FCH;
  // Primitive quartets set up per round: as many as fit a shared-memory
  // budget of 48 KB per 128-thread block (power of two, at most T).
  static constexpr int GTAB = (S::NE + 1) * (S::NF + 1);
  static constexpr int PRIM_TAB = 2 * S::NR + 3 * S::NR * GTAB;  // x, w, g[3][NR][GTAB]
  static constexpr int BUDGET = (48 * 1024 / 128) * (T == 1 ? 1 : T) / (int)sizeof(R);
  static constexpr int BP0 = BUDGET / PRIM_TAB;
  static constexpr int BP = BP0 >= T ? T : (BP0 >= 16 ? 16 : (BP0 >= 8 ? 8 : (BP0 >= 4 ? 4 : (BP0 >= 2 ? 2 : 1))));
  static constexpr int SUB = T / BP;  // lanes sharing one primitive quartet in a round
  static constexpr int SMEM_PER_TEAM = T == 1 ? 0 : BP * PRIM_TAB;  // in R units
  // Per-team shared memory: the primitive tables of phase 1, reused by the
  // post phase for the team's copy of the Cartesian block (16-byte multiple).
  // Classes whose copies would need more than 96 KB per 128-thread block
  // (f shells) read the block from the scratch slot instead.
  static constexpr int STAGE_BYTES0 = T == 1 ? 0 : jk_stage_doubles(LA, LB, LC, LD) * 8;
  static constexpr bool STAGE = T > 1 && (128 / T) * STAGE_BYTES0 <= 96 * 1024;
  static constexpr int STAGE_BYTES = STAGE ? STAGE_BYTES0 : 0;
  static constexpr int TAB_BYTES = SMEM_PER_TEAM * (int)sizeof(R);
  static constexpr int TEAM_BYTES = ((TAB_BYTES > STAGE_BYTES ? TAB_BYTES : STAGE_BYTES) + 15) / 16 * 16;
};

// Magnitude bound of one primitive quartet's contribution, |E_ab E_cd| times
// the Coulomb prefactor 2 pi^{5/2} / (p q sqrt(p + q)) (every Rys weight sum
// and Boys value is <= 1); evaluated in FP32 for the primitive screen of the
// FP32 launches.
__device__ __forceinline__ float prim_bound(const PrimPairF& b, const PrimPairF& k) {
  return fabsf(b.e * k.e) * (34.98683665f / (b.zeta * k.zeta * sqrtf(b.zeta + k.zeta)));
}

// Largest primitive-quartet count the team screen compacts (16 x 16 primitive
// pairs); quartets with more run every primitive quartet.
constexpr int MAX_SURV = 256;

// ------------------------------------------------------------- TEAM == 1

template <int LA, int LB, int LC, int LD, typename R>
__device__ __forceinline__ void accumulate_thread(const KernelArgs& A, const R* s_tab, const PairD& pb,
                                                  const PairD& pk, R (&G)[ClassShape<LA, LB, LC, LD>::NG]) {
  using S = ClassShape<LA, LB, LC, LD>;
  constexpr int NE = S::NE, NF = S::NF, NR = S::NR;
#pragma unroll
  for (int q = 0; q < S::NG; ++q) G[q] = R(0);
  const float cut = (sizeof(R) == 4 && A.fp32) ? (float)A.prim_cut : 0.f;
  float acx = 0.f, acy = 0.f, acz = 0.f;
  if constexpr (sizeof(R) == 4) {
    const DevShell& sa = A.shells[pb.a];
    const DevShell& sc = A.shells[pk.a];
    acx = (float)(sa.cx - sc.cx);
    acy = (float)(sa.cy - sc.cy);
    acz = (float)(sa.cz - sc.cz);
  }
  for (int ip = 0; ip < pb.nprim; ++ip) {
    for (int kq = 0; kq < pk.nprim; ++kq) {
      QuartetHdr<R> h;
      if constexpr (sizeof(R) == 4) {
        const PrimPairF bp = A.primsf[pb.prim_off + ip];
        const PrimPairF kp = A.primsf[pk.prim_off + kq];
        if (cut > 0.f && prim_bound(bp, kp) < cut) continue;
        h = quartet_header_f(bp, kp, acx, acy, acz, A.omega);
      } else {
        h = quartet_header<R>(A.prims[pb.prim_off + ip], A.prims[pk.prim_off + kq], A.omega);
      }
      R x[NR], w[NR];
      if constexpr (sizeof(R) == 4) {
        // FP32 launch: quadratures of five or more roots (high l) take
        // FP64 roots and weights
        if (roots_in_fp64<NR, R>(h.T)) {
          const double T64 = quartet_T64(A.prims[pb.prim_off + ip], A.prims[pk.prim_off + kq], A.omega);
#pragma unroll
          for (int r = 0; r < NR; ++r) {
            double xd, wd;
            rys_root_fp64<NR>(T64, r, xd, wd);
            x[r] = R(xd);
            w[r] = R(wd);
          }
        } else {
          rys_roots_s<NR, R>(s_tab, h.T, x, w);
        }
      } else {
        rys_roots_s<NR, R>(s_tab, h.T, x, w);
      }
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
        R gx[NE + 1][NF + 1], gy[NE + 1][NF + 1], gz[NE + 1][NF + 1];
        vrr_axis<NE, NF, R>(R(1), h.pax - cq * h.pqx, h.qcx + cp * h.pqx, b10, b01, b00, gx);
        vrr_axis<NE, NF, R>(R(1), h.pay - cq * h.pqy, h.qcy + cp * h.pqy, b10, b01, b00, gy);
        vrr_axis<NE, NF, R>(w[r] * h.pref, h.paz - cq * h.pqz, h.qcz + cp * h.pqz, b10, b01, b00, gz);
        static_for<S::NEP>([&](auto e) {
          constexpr int ex = range_x(LA, decltype(e)::value);
          constexpr int ey = range_y(LA, decltype(e)::value);
          constexpr int ez = range_z(LA, decltype(e)::value);
          static_for<S::NFP>([&](auto f) {
            constexpr int fx = range_x(LC, decltype(f)::value);
            constexpr int fy = range_y(LC, decltype(f)::value);
            constexpr int fz = range_z(LC, decltype(f)::value);
            G[decltype(e)::value * S::NFP + decltype(f)::value] += gx[ex][fx] * gy[ey][fy] * gz[ez][fz];
          });
        });
      }
    }
  }
}

// --------------------------------------------------------------- TEAM > 1

// Root r of the N-point quadrature from the shared-memory table.
template <int N, typename R>
__device__ __forceinline__ void rys_root_one(const R* s_tab, R T, int r, R& x, R& w) {
  const RysMeta m = c_rys[N];
  if (T >= R(m.t_hi)) {
    if constexpr (sizeof(R) == 8) {
      x = c_lag_x[N - 1][r] / T;
      w = c_lag_w[N - 1][r] * R(0.5) * rsqrt(T);
    } else {
      x = c_lag_xf[N - 1][r] / T;
      w = c_lag_wf[N - 1][r] * R(0.5) * rsqrt(T);
    }
    return;
  }
  R width = R(m.width);
  int s = (int)(T / width);
  s = s < 0 ? 0 : (s >= m.n_sub ? m.n_sub - 1 : s);
  R a = R(s) * width;
  R b = a + width;
  R xi = (R(2) * T - (a + b)) / (b - a);
  const R* base = s_tab + ((size_t)s * N + r) * 2 * RYS_NC;
  x = chebev_s<R>(base, xi);
  w = chebev_s<R>(base + RYS_NC, xi);
}

// One pass over all primitive quartets accumulating the columns
// [F0, F0 + FCH) of this lane's rows.
template <int LA, int LB, int LC, int LD, typename R, int F0>
__device__ __forceinline__ void team_pass(const KernelArgs& A, const R* s_tab, const PairD& pb, const PairD& pk,
                                          R* sm, int lane, unsigned tmask, double* G, const unsigned short* surv,
                                          int npr, bool g32) {
  using S = ClassShape<LA, LB, LC, LD>;
  using TS = TeamShape<LA, LB, LC, LD, R>;
  constexpr int NE = S::NE, NF = S::NF, NR = S::NR, T = TS::T;
  constexpr int FW = (F0 + TS::FCH <= S::NFP) ? TS::FCH : (S::NFP - F0);
  constexpr int GT = TS::GTAB;
  R acc[TS::ROWS][FW];
#pragma unroll
  for (int k = 0; k < TS::ROWS; ++k)
#pragma unroll
    for (int f = 0; f < FW; ++f) acc[k][f] = R(0);
  int ex[TS::ROWS], ey[TS::ROWS], ez[TS::ROWS];
#pragma unroll
  for (int k = 0; k < TS::ROWS; ++k) {
    int e = lane + T * k;
    int a = tri_below(LA) + (e < S::NEP ? e : 0);
    ex[k] = addr_lx(a);
    ey[k] = addr_ly(a);
    ez[k] = addr_lz(a);
  }
  // Rounds of BP primitive quartets: SUB lanes set up each one (roots, then
  // the 3*NR per-axis tables) into its shared-memory slot, then every lane
  // accumulates its rows over the whole round.
  constexpr int BP = TS::BP, SUB = TS::SUB, PT = TS::PRIM_TAB;
  const int npk = pk.nprim;
  const int myp = lane % BP;
  const int sub = lane / BP;
  float acx = 0.f, acy = 0.f, acz = 0.f;
  if constexpr (sizeof(R) == 4) {
    const DevShell& sa = A.shells[pb.a];
    const DevShell& sc = A.shells[pk.a];
    acx = (float)(sa.cx - sc.cx);
    acy = (float)(sa.cy - sc.cy);
    acz = (float)(sa.cz - sc.cz);
  }
  for (int base = 0; base < npr; base += BP) {
    const int nb = npr - base < BP ? npr - base : BP;
    const bool active = myp < nb;
    R* mys = sm + myp * PT;
    QuartetHdr<R> h;
    if (active) {
      const int pidx = surv ? (int)surv[base + myp] : base + myp;
      const int ip = pidx / npk, kq = pidx - ip * npk;
      if constexpr (sizeof(R) == 4)
        h = quartet_header_f(A.primsf[pb.prim_off + ip], A.primsf[pk.prim_off + kq], acx, acy, acz, A.omega);
      else
        h = quartet_header<R>(A.prims[pb.prim_off + ip], A.prims[pk.prim_off + kq], A.omega);
      // FP32 launch: quadratures of five or more roots (high l) take
      // FP64 roots and weights
      const bool r64 = roots_in_fp64<NR, R>(h.T);
      const double T64 = r64 ? quartet_T64(A.prims[pb.prim_off + ip], A.prims[pk.prim_off + kq], A.omega) : 0.0;
      for (int r = sub; r < NR; r += SUB) {
        R xr, wr;
        if (r64) {
          double xd, wd;
          rys_root_fp64<NR>(T64, r, xd, wd);
          xr = R(xd);
          wr = R(wd);
        } else {
          rys_root_one<NR, R>(s_tab, h.T, r, xr, wr);
        }
        mys[r] = xr * h.xs;
        mys[NR + r] = wr * h.pref;
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
        R g[NE + 1][NF + 1];
        vrr_axis<NE, NF, R>(axis == 2 ? mys[NR + r] : R(1), paa - xr * qpq * pqa, qca + xr * ppq * pqa, b10, b01,
                            b00, g);
        R* dst = mys + 2 * NR + (axis * NR + r) * GT;
#pragma unroll
        for (int n = 0; n <= NE; ++n)
#pragma unroll
          for (int m = 0; m <= NF; ++m) dst[n * (NF + 1) + m] = g[n][m];
      }
    }
    __syncwarp(tmask);
    for (int p = 0; p < nb; ++p) {
      const R* gt = sm + p * PT + 2 * NR;
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const R* tx = gt + (0 * NR + r) * GT;
        const R* ty = gt + (1 * NR + r) * GT;
        const R* tz = gt + (2 * NR + r) * GT;
#pragma unroll
        for (int k = 0; k < TS::ROWS; ++k) {
          if (TS::ROWS * T > S::NEP && lane + T * k >= S::NEP) continue;
          R rx[NF + 1], ry[NF + 1], rz[NF + 1];
#pragma unroll
          for (int m = 0; m <= NF; ++m) {
            rx[m] = tx[ex[k] * (NF + 1) + m];
            ry[m] = ty[ey[k] * (NF + 1) + m];
            rz[m] = tz[ez[k] * (NF + 1) + m];
          }
          static_for<FW>([&](auto f) {
            constexpr int fi = F0 + decltype(f)::value;
            constexpr int fx = range_x(LC, fi), fy = range_y(LC, fi), fz = range_z(LC, fi);
            acc[k][decltype(f)::value] += rx[fx] * ry[fy] * rz[fz];
          });
        }
      }
    }
    __syncwarp(tmask);
  }
#pragma unroll
  for (int k = 0; k < TS::ROWS; ++k) {
    int e = lane + T * k;
    if (e < S::NEP) {
      if (sizeof(R) == 4 && g32) {
        // FP32 post phase: the table stays in FP32
        float* Gf = reinterpret_cast<float*>(G);
#pragma unroll
        for (int f = 0; f < FW; ++f) Gf[(size_t)e * S::NFP + F0 + f] = (float)acc[k][f];
      } else {
#pragma unroll
        for (int f = 0; f < FW; ++f) G[(size_t)e * S::NFP + F0 + f] = (double)acc[k][f];
      }
    }
  }
}

template <int LA, int LB, int LC, int LD, typename R, int C>
__device__ __forceinline__ void team_chunks(const KernelArgs& A, const R* s_tab, const PairD& pb, const PairD& pk,
                                            R* sm, int lane, unsigned tmask, double* G, const unsigned short* surv,
                                            int npr, bool g32) {
  using TS = TeamShape<LA, LB, LC, LD, R>;
  if constexpr (C < TS::NCHUNK) {
    team_pass<LA, LB, LC, LD, R, C * TS::FCH>(A, s_tab, pb, pk, sm, lane, tmask, G, surv, npr, g32);
    __syncwarp(tmask);
    team_chunks<LA, LB, LC, LD, R, C + 1>(A, s_tab, pb, pk, sm, lane, tmask, G, surv, npr, g32);
  }
}

// Primitive screen of one quartet on a team of T lanes: the indices
// ip * nprim_ket + kq of the primitive quartets whose bound reaches `cut`,
// in order, into `list`; returns their count.
template <int T>
__device__ __forceinline__ int screen_prims(const KernelArgs& A, const PairD& pb, const PairD& pk, float cut,
                                            unsigned short* list, int lane, unsigned tmask) {
  const int npk = pk.nprim, npr = pb.nprim * npk;
  const int shift = ((threadIdx.x & 31) / T) * T;  // the team's first lane in the warp
  int n = 0;
  for (int b0 = 0; b0 < npr; b0 += T) {
    const int pidx = b0 + lane;
    bool keep = false;
    if (pidx < npr) {
      const int ip = pidx / npk, kq = pidx - ip * npk;
      keep = prim_bound(A.primsf[pb.prim_off + ip], A.primsf[pk.prim_off + kq]) >= cut;
    }
    const unsigned bal = (__ballot_sync(tmask, keep) & tmask) >> shift;
    if (keep) list[n + __popc(bal & ((1u << lane) - 1u))] = (unsigned short)pidx;
    n += __popc(bal);
  }
  __syncwarp(tmask);
  return n;
}

// ------------------------------------------------------------------ kernel

// Minimum resident 128-thread blocks per SM (register budget): team
// classes 3 (168 registers; measured faster than the unconstrained
// allocation, whose unrolled J/K sums take up to 255), thread-per-quartet
// classes by the size of their register-resident G table (spilling large
// tables costs more than the occupancy gains).
#ifndef IGPU_FP32_TEAM_MINB
#define IGPU_FP32_TEAM_MINB 3
#endif
template <int LA, int LB, int LC, int LD, typename R>
__host__ __device__ constexpr int quartet_min_blocks() {
  return team_size<LA, LB, LC, LD>() > 1
             ? (sizeof(R) == 4 ? IGPU_FP32_TEAM_MINB : 3)
             : (ClassShape<LA, LB, LC, LD>::NG <= 9 ? 5 : (ClassShape<LA, LB, LC, LD>::NG <= 27 ? 3 : 1));
}

template <int LA, int LB, int LC, int LD, typename R>
__global__ void __launch_bounds__(128, quartet_min_blocks<LA, LB, LC, LD, R>()) quartet_kernel(KernelArgs A) {
  using S = ClassShape<LA, LB, LC, LD>;
  using TS = TeamShape<LA, LB, LC, LD, R>;
  constexpr int T = TS::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ R s_tab[S::NR * RYS_MAX_SUB * 2 * RYS_NC];
  constexpr bool SCREEN = sizeof(R) == 4 && T > 1;
  __shared__ unsigned short s_surv[SCREEN ? (128 / T) * MAX_SURV : 1];
  constexpr bool CT_POST = ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD) <= 10000;
  __shared__ int s_hrr[(T > 1 && CT_POST) ? HrrTab<LA, LB, LC, LD>::TOTAL : 1];
  __shared__ R s_c2s[(T > 1 && CT_POST) ? 4 * C2S_TILE : 1];
  if constexpr (T > 1 && CT_POST) {
    build_hrr_tab<LA, LB, LC, LD>(s_hrr);
    stage_c2s<LA, LB, LC, LD, R>(A, s_c2s);
  }
  stage_rys_table<S::NR, R>(s_tab);  // its __syncthreads also publishes s_hrr, s_c2s
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int team = tid / T;
  const int lane = threadIdx.x % T;
  const int nteams = (gridDim.x * blockDim.x) / T;
  const unsigned tmask = T == 32 ? 0xffffffffu : (((1u << T) - 1u) << ((threadIdx.x % 32) / T * T));
  unsigned char* team_smem = smem_raw + (size_t)(threadIdx.x / T) * TS::TEAM_BYTES;
  R* sm = reinterpret_cast<R*>(team_smem);
  double* stage = TS::STAGE ? reinterpret_cast<double*>(team_smem) : nullptr;
  R* stage_r = TS::STAGE ? reinterpret_cast<R*>(team_smem) : nullptr;
  double* slot = A.scratch + (size_t)team * A.slot_doubles;
  QuartetCounters cnt;
  const ClassDims dims{LA, LB, LC, LD};
  (void)nteams;
  const bool use_acc = A.mode == MODE_JK && A.jk.symmetric;
  if (use_acc) {
    // the scratch slot is shared with earlier launches: clear the running
    // bra-block accumulators before first use
    double* acc = slot + A.acc_offset;
    const int nacc = A.jk.ndens * ncart(LA) * ncart(LB);
    for (int q = lane; q < nacc; q += T) acc[1 + q] = 0.0;
    if (lane == 0) acc[0] = -1.0;
  }
  __syncwarp(tmask);

  // Warps claim contiguous chunks of the task list; the teams of a warp
  // interleave inside a chunk, so consecutive quartets (same bra pair, same
  // primitive-pair count) stay on the same lanes.
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
    for (unsigned long long g = base + tw; g < end; g += TPW) {
      int pbi, pki;
      cursor_decode(A.task, g, cur, pbi, pki);
      const PairD pb = A.pairs[pbi];
      const PairD pk = A.pairs[pki];
      Screen sc = screen_quartet(A, pb, pk);
      if (!sc.keep) continue;
      if (lane == 0) cnt.add(sc, pb, pk, A.fp32);
      if constexpr (T == 1) {
        R G[S::NG];
        accumulate_thread<LA, LB, LC, LD, R>(A, s_tab, pb, pk, G);
        if (use_acc && A.kinds != 2) {
          // the post phase runs in the launch's arithmetic (FP32 launches
          // read the FP32 densities); J/K accumulate in FP64
          if (A.kinds == 0)
            thread_post_jk<LA, LB, LC, LD, false, R>(A, G, pb, pk, sc, slot + A.acc_offset, pbi);
          else
            thread_post_jk<LA, LB, LC, LD, true, R>(A, G, pb, pk, sc, slot + A.acc_offset, pbi);
          continue;
        }
#pragma unroll
        for (int q = 0; q < S::NG; ++q) slot[q] = (double)G[q];
      } else {
        const unsigned short* surv = nullptr;
        int npr = pb.nprim * pk.nprim;
        if constexpr (SCREEN) {
          if (A.fp32 && A.prim_cut > 0.0 && npr <= MAX_SURV) {
            unsigned short* list = s_surv + (threadIdx.x / T) * MAX_SURV;
            npr = screen_prims<T>(A, pb, pk, (float)A.prim_cut, list, lane, tmask);
            surv = list;
            if (npr == 0) continue;  // the whole quartet is below the screen
          }
        }
        team_chunks<LA, LB, LC, LD, R, 0>(A, s_tab, pb, pk, sm, lane, tmask, slot, surv, npr,
                                          CT_POST && use_acc && A.kinds != 2);
      }
      __syncwarp(tmask);
      // the compile-time shaped J/K sums unroll over the whole Cartesian
      // block, in the launch's arithmetic; blocks beyond (ff|ff) (g shells)
      // take the runtime post phase
      if constexpr (T > 1 && CT_POST) {
        if (use_acc && A.kinds == 0) {
          post_quartet_jk_cart<LA, LB, LC, LD, T, R>(A, pb, pk, sc, slot, lane, tmask, pbi, stage_r, s_hrr);
          continue;
        }
        if (use_acc && A.kinds == 1) {
          post_quartet_jk_sph<LA, LB, LC, LD, T, R>(A, pb, pk, sc, slot, lane, tmask, pbi, stage_r, s_hrr, s_c2s);
          continue;
        }
      }
      post_quartet(A, dims, pb, pk, sc, slot, lane, T, tmask, pbi, stage);
      __syncwarp(tmask);
    }
  }
  if (use_acc) flush_bra_acc(A, slot + A.acc_offset, lane, T, tmask);
  cnt.flush(A.counters);
}

}  // namespace igpu
