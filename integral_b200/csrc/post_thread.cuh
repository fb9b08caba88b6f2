// Register-resident post phase for one-thread-per-quartet classes: the
// horizontal recurrences, the spherical transform and the symmetric-density
// J/K contraction fully unrolled at compile time (every index below is a
// constant), so the block never leaves registers.  Same arithmetic as the
// team version in post.cuh.
#pragma once
#include "post.cuh"

namespace igpu {

__host__ __device__ constexpr int cart_index_c(int lx, int ly, int lz) { return (ly + lz) * (ly + lz + 1) / 2 + lz; }
__host__ __device__ constexpr int addr_c(int lx, int ly, int lz) { return tri_below(lx + ly + lz) + cart_index_c(lx, ly, lz); }
__host__ __device__ constexpr int first_axis(int x, int y, int z) { return x > 0 ? 0 : (y > 0 ? 1 : 2); }

// Bra level KB: (a, b | f) for b of degree KB, a of degree LA..NE-KB, from
// level KB-1 (src/engine/os_eri.rs:3083-3116).
template <int LA, int NE, int NFP, int KB, typename V>
__device__ __forceinline__ void bra_level(const V* src, V* dst, const V ab[3]) {
  constexpr int NBK = ncart(KB), NAK = nrange(LA, NE - KB), NAP = nrange(LA, NE - KB + 1);
  static_for<NBK>([&](auto ib_) {
    constexpr int ib = decltype(ib_)::value;
    constexpr int bx = comp_lx(KB, ib), by = comp_ly(KB, ib), bz = comp_lz(KB, ib);
    constexpr int ax = first_axis(bx, by, bz);
    constexpr int ib1 = cart_index_c(bx - (ax == 0), by - (ax == 1), bz - (ax == 2));
    static_for<NAK>([&](auto ia_) {
      constexpr int ia = decltype(ia_)::value;
      constexpr int px = range_x(LA, ia), py = range_y(LA, ia), pz = range_z(LA, ia);
      constexpr int ia1 = addr_c(px + (ax == 0), py + (ax == 1), pz + (ax == 2)) - tri_below(LA);
      static_for<NFP>([&](auto f_) {
        constexpr int f = decltype(f_)::value;
        dst[(ib * NAK + ia) * NFP + f] = src[(ib1 * NAP + ia1) * NFP + f] + ab[ax] * src[(ib1 * NAP + ia) * NFP + f];
      });
    });
  });
}

template <int LA, int LB, int NFP, int KB, typename V>
__device__ __forceinline__ void bra_hrr(const V* src, V* out, const V ab[3]) {
  if constexpr (LB == 0) {
#pragma unroll
    for (int q = 0; q < ncart(LA) * NFP; ++q) out[q] = src[q];
  } else {
    constexpr int NE = LA + LB;
    V dst[ncart(KB) * nrange(LA, NE - KB) * NFP];
    bra_level<LA, NE, NFP, KB, V>(src, dst, ab);
    if constexpr (KB == LB) {
#pragma unroll
      for (int q = 0; q < ncart(LB) * ncart(LA) * NFP; ++q) out[q] = dst[q];
    } else {
      bra_hrr<LA, LB, NFP, KB + 1, V>(dst, out, ab);
    }
  }
}

// Ket level KD of one (a,b) row: (c, d) for d of degree KD, c of degree
// LC..NF-KD.
template <int LC, int NF, int KD, typename V>
__device__ __forceinline__ void ket_level(const V* src, V* dst, const V cd[3]) {
  constexpr int NDK = ncart(KD), NCK = nrange(LC, NF - KD), NCP = nrange(LC, NF - KD + 1);
  static_for<NDK>([&](auto id_) {
    constexpr int id = decltype(id_)::value;
    constexpr int dx = comp_lx(KD, id), dy = comp_ly(KD, id), dz = comp_lz(KD, id);
    constexpr int ax = first_axis(dx, dy, dz);
    constexpr int id1 = cart_index_c(dx - (ax == 0), dy - (ax == 1), dz - (ax == 2));
    static_for<NCK>([&](auto ic_) {
      constexpr int ic = decltype(ic_)::value;
      constexpr int px = range_x(LC, ic), py = range_y(LC, ic), pz = range_z(LC, ic);
      constexpr int ic1 = addr_c(px + (ax == 0), py + (ax == 1), pz + (ax == 2)) - tri_below(LC);
      dst[id * NCK + ic] = src[id1 * NCP + ic1] + cd[ax] * src[id1 * NCP + ic];
    });
  });
}

template <int LC, int LD, int KD, typename V>
__device__ __forceinline__ void ket_hrr(const V* src, V* out, const V cd[3]) {
  constexpr int NF = LC + LD;
  if constexpr (LD == 0) {
#pragma unroll
    for (int q = 0; q < ncart(LC); ++q) out[q] = src[q];
  } else {
    V dst[ncart(KD) * nrange(LC, NF - KD)];
    ket_level<LC, NF, KD, V>(src, dst, cd);
    if constexpr (KD == LD) {
      // [d][c] -> [c][d]
#pragma unroll
      for (int c = 0; c < ncart(LC); ++c)
#pragma unroll
        for (int d = 0; d < ncart(LD); ++d) out[c * ncart(LD) + d] = dst[d * ncart(LC) + c];
    } else {
      ket_hrr<LC, LD, KD + 1, V>(dst, out, cd);
    }
  }
}

// Contract one axis of a [D0][D1][D2][D3] register block with the (2l+1) x
// n_cart matrix M (spherical.rs:121-179).
template <int AXIS, int D0, int D1, int D2, int D3, int NOUT, typename V>
__device__ __forceinline__ void c2s_axis(const V* in, V* out, const double* __restrict__ M) {
  constexpr int dims[4] = {D0, D1, D2, D3};
  constexpr int NIN = dims[AXIS];
  constexpr int outer = AXIS == 0 ? 1 : (AXIS == 1 ? D0 : (AXIS == 2 ? D0 * D1 : D0 * D1 * D2));
  constexpr int inner = AXIS == 0 ? D1 * D2 * D3 : (AXIS == 1 ? D2 * D3 : (AXIS == 2 ? D3 : 1));
  V m[NOUT * NIN];
#pragma unroll
  for (int q = 0; q < NOUT * NIN; ++q) m[q] = (V)__ldg(M + q);
#pragma unroll
  for (int o = 0; o < outer; ++o)
#pragma unroll
    for (int q = 0; q < NOUT; ++q)
#pragma unroll
      for (int s = 0; s < inner; ++s) {
        V acc = V(0);
#pragma unroll
        for (int j = 0; j < NIN; ++j) acc += m[q * NIN + j] * in[(o * NIN + j) * inner + s];
        out[(o * NOUT + q) * inner + s] = acc;
      }
}

template <int LA, int LB, int LC, int LD>
struct ThreadPost {
  static constexpr int NE = LA + LB, NF = LC + LD;
  static constexpr int NEP = nrange(LA, NE), NFP = nrange(LC, NF);
  static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  static constexpr int NBLK = NA * NB * NC * ND;
};

// G (registers) -> Cartesian block (registers).
template <int LA, int LB, int LC, int LD, typename V>
__device__ __forceinline__ void thread_block(const V* G, V* blk, const PairD& pb, const PairD& pk) {
  using P = ThreadPost<LA, LB, LC, LD>;
  const V ab[3] = {(V)pb.abx, (V)pb.aby, (V)pb.abz};
  const V cdv[3] = {(V)pk.abx, (V)pk.aby, (V)pk.abz};
  V H[P::NB * P::NA * P::NFP];  // [b][a][f]
  bra_hrr<LA, LB, P::NFP, 1, V>(G, H, ab);
  static_for<P::NA>([&](auto ia_) {
    constexpr int ia = decltype(ia_)::value;
    static_for<P::NB>([&](auto ib_) {
      constexpr int ib = decltype(ib_)::value;
      ket_hrr<LC, LD, 1, V>(H + (ib * P::NA + ia) * P::NFP, blk + (ia * P::NB + ib) * P::NC * P::ND, cdv);
    });
  });
}

// Symmetric-density J/K of one function-space block [N0][N1][N2][N3] in
// value type V (double, or float for the FP32 launches of the mixed path,
// which read the FP32 copy of the densities): bra-block J term into the
// running FP64 accumulators `acc`, the other five one-orientation terms
// atomically into the FP64 J', K'.
template <int N0, int N1, int N2, int N3, typename V>
__device__ __forceinline__ void thread_jk(const KernelArgs& A, const V* B, const int offs[4], unsigned w,
                                          uint64_t mask, double* acc) {
  auto W = [&](int p) { return (V)((w >> p) & 1u); };
  const V wab = W(0) + W(1) + W(2) + W(3), wcd = W(4) + W(5) + W(6) + W(7);
  const V wac = W(0) + W(4), wbc = W(1) + W(5), wad = W(2) + W(6), wbd = W(3) + W(7);
  const int nao = A.nao;
  const size_t n2 = (size_t)nao * nao;
  constexpr int S0 = N1 * N2 * N3, S1 = N2 * N3, S2 = N3;
  for (int d = 0; d < A.jk.ndens; ++d) {
    if (!((mask >> d) & 1ull)) continue;
    const V* Dm = dens_of<V>(A.jk) + d * n2;
    double* J = A.jk.J + d * n2;
    // J'[A a][B b] (accumulated over the bra's quartets)
    {
      V dcd[N2 * N3];
#pragma unroll
      for (int c = 0; c < N2; ++c)
#pragma unroll
        for (int e = 0; e < N3; ++e) dcd[c * N3 + e] = __ldg(Dm + (size_t)(offs[2] + c) * nao + offs[3] + e);
      double* a = acc + 1 + (size_t)d * N0 * N1;
#pragma unroll
      for (int i = 0; i < N0; ++i)
#pragma unroll
        for (int j = 0; j < N1; ++j) {
          V s = V(0);
#pragma unroll
          for (int q = 0; q < N2 * N3; ++q) s += B[i * S0 + j * S1 + q] * dcd[q];
          a[i * N1 + j] += (double)(wab * s);
        }
    }
    // J'[C c][D d]
    if (wcd != V(0)) {
      V dab[N0 * N1];
#pragma unroll
      for (int i = 0; i < N0; ++i)
#pragma unroll
        for (int j = 0; j < N1; ++j) dab[i * N1 + j] = __ldg(Dm + (size_t)(offs[0] + i) * nao + offs[1] + j);
#pragma unroll
      for (int c = 0; c < N2; ++c)
#pragma unroll
        for (int e = 0; e < N3; ++e) {
          V s = V(0);
#pragma unroll
          for (int q = 0; q < N0 * N1; ++q) s += B[q * S1 + c * S2 + e] * dab[q];
          atomicAdd(J + (size_t)(offs[2] + c) * nao + offs[3] + e, (double)(wcd * s));
        }
    }
    if (!A.jk.want_k) continue;
    double* K = A.jk.K + d * n2;
    // K'[A a][C c] = sum_{b,d} B D[B b][D d]
    if (wac != V(0)) {
      V m[N1 * N3];
#pragma unroll
      for (int j = 0; j < N1; ++j)
#pragma unroll
        for (int e = 0; e < N3; ++e) m[j * N3 + e] = __ldg(Dm + (size_t)(offs[1] + j) * nao + offs[3] + e);
#pragma unroll
      for (int i = 0; i < N0; ++i)
#pragma unroll
        for (int c = 0; c < N2; ++c) {
          V s = V(0);
#pragma unroll
          for (int j = 0; j < N1; ++j)
#pragma unroll
            for (int e = 0; e < N3; ++e) s += B[i * S0 + j * S1 + c * S2 + e] * m[j * N3 + e];
          atomicAdd(K + (size_t)(offs[0] + i) * nao + offs[2] + c, (double)(wac * s));
        }
    }
    // K'[B b][C c] = sum_{a,d} B D[A a][D d]
    if (wbc != V(0)) {
      V m[N0 * N3];
#pragma unroll
      for (int i = 0; i < N0; ++i)
#pragma unroll
        for (int e = 0; e < N3; ++e) m[i * N3 + e] = __ldg(Dm + (size_t)(offs[0] + i) * nao + offs[3] + e);
#pragma unroll
      for (int j = 0; j < N1; ++j)
#pragma unroll
        for (int c = 0; c < N2; ++c) {
          V s = V(0);
#pragma unroll
          for (int i = 0; i < N0; ++i)
#pragma unroll
            for (int e = 0; e < N3; ++e) s += B[i * S0 + j * S1 + c * S2 + e] * m[i * N3 + e];
          atomicAdd(K + (size_t)(offs[1] + j) * nao + offs[2] + c, (double)(wbc * s));
        }
    }
    // K'[A a][D d] = sum_{b,c} B D[B b][C c]
    if (wad != V(0)) {
      V m[N1 * N2];
#pragma unroll
      for (int j = 0; j < N1; ++j)
#pragma unroll
        for (int c = 0; c < N2; ++c) m[j * N2 + c] = __ldg(Dm + (size_t)(offs[1] + j) * nao + offs[2] + c);
#pragma unroll
      for (int i = 0; i < N0; ++i)
#pragma unroll
        for (int e = 0; e < N3; ++e) {
          V s = V(0);
#pragma unroll
          for (int j = 0; j < N1; ++j)
#pragma unroll
            for (int c = 0; c < N2; ++c) s += B[i * S0 + j * S1 + c * S2 + e] * m[j * N2 + c];
          atomicAdd(K + (size_t)(offs[0] + i) * nao + offs[3] + e, (double)(wad * s));
        }
    }
    // K'[B b][D d] = sum_{a,c} B D[A a][C c]
    if (wbd != V(0)) {
      V m[N0 * N2];
#pragma unroll
      for (int i = 0; i < N0; ++i)
#pragma unroll
        for (int c = 0; c < N2; ++c) m[i * N2 + c] = __ldg(Dm + (size_t)(offs[0] + i) * nao + offs[2] + c);
#pragma unroll
      for (int j = 0; j < N1; ++j)
#pragma unroll
        for (int e = 0; e < N3; ++e) {
          V s = V(0);
#pragma unroll
          for (int i = 0; i < N0; ++i)
#pragma unroll
            for (int c = 0; c < N2; ++c) s += B[i * S0 + j * S1 + c * S2 + e] * m[i * N2 + c];
          atomicAdd(K + (size_t)(offs[1] + j) * nao + offs[3] + e, (double)(wbd * s));
        }
    }
  }
}

// Whole post phase of a one-thread quartet for symmetric-density J/K with
// all four shells Cartesian (SPH = false) or all four spherical (SPH = true),
// in the launch's arithmetic V; J/K accumulate in FP64.
template <int LA, int LB, int LC, int LD, bool SPH, typename V>
__device__ __forceinline__ void thread_post_jk(const KernelArgs& A, const V* G, const PairD& pb, const PairD& pk,
                                               const Screen& sc, double* acc, int pbi) {
  using P = ThreadPost<LA, LB, LC, LD>;
  V blk[P::NBLK];
  thread_block<LA, LB, LC, LD, V>(G, blk, pb, pk);
  const int shl[4] = {pb.a, pb.b, pk.a, pk.b};
  const int offs[4] = {A.shells[shl[0]].off, A.shells[shl[1]].off, A.shells[shl[2]].off, A.shells[shl[3]].off};
  const unsigned w = distinct_perms(shl);
  if ((int)acc[0] != pbi) {
    flush_bra_acc(A, acc, 0, 1, 1u << (threadIdx.x & 31));
    acc[0] = (double)pbi;
  }
  if constexpr (!SPH) {
    thread_jk<P::NA, P::NB, P::NC, P::ND, V>(A, blk, offs, w, sc.mask, acc);
  } else {
    constexpr int F0 = 2 * LA + 1, F1 = 2 * LB + 1, F2 = 2 * LC + 1, F3 = 2 * LD + 1;
    V t1[F0 * P::NB * P::NC * P::ND];
    c2s_axis<0, P::NA, P::NB, P::NC, P::ND, F0, V>(blk, t1, A.c2s + A.c2s_off[LA]);
    V t2[F0 * F1 * P::NC * P::ND];
    c2s_axis<1, F0, P::NB, P::NC, P::ND, F1, V>(t1, t2, A.c2s + A.c2s_off[LB]);
    V t3[F0 * F1 * F2 * P::ND];
    c2s_axis<2, F0, F1, P::NC, P::ND, F2, V>(t2, t3, A.c2s + A.c2s_off[LC]);
    V t4[F0 * F1 * F2 * F3];
    c2s_axis<3, F0, F1, F2, P::ND, F3, V>(t3, t4, A.c2s + A.c2s_off[LD]);
    thread_jk<F0, F1, F2, F3, V>(A, t4, offs, w, sc.mask, acc);
  }
}

}  // namespace igpu
