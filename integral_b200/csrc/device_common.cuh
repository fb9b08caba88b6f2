// Device helpers shared by the quartet kernels: compile-time angular-momentum
// tables, Rys roots/weights from the Chebyshev tables, the per-axis Rys
// vertical recurrence, and small warp utilities.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <utility>

#include "igpu_internal.hpp"

namespace igpu {

// ------------------------------------------------------------ compile time

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int tri_below(int d) { return d * (d + 1) * (d + 2) / 6; }
__host__ __device__ constexpr int n_addr(int l) { return (l + 1) * (l + 2) * (l + 3) / 6; }
// Number of Cartesian triples with degree in [lo, hi].
__host__ __device__ constexpr int nrange(int lo, int hi) { return tri_below(hi + 1) - tri_below(lo); }

// Component i (canonical order: lx descending, then ly descending) of degree l.
__host__ __device__ constexpr int comp_lx(int l, int i) {
  int lx = l, rem = i;
  while (rem >= l - lx + 1) {
    rem -= l - lx + 1;
    --lx;
  }
  return lx;
}
__host__ __device__ constexpr int comp_ly(int l, int i) {
  int lx = l, rem = i;
  while (rem >= l - lx + 1) {
    rem -= l - lx + 1;
    --lx;
  }
  return (l - lx) - rem;
}
__host__ __device__ constexpr int comp_lz(int l, int i) { return l - comp_lx(l, i) - comp_ly(l, i); }
// Degree of the k-th triple in the range starting at degree lo.
__host__ __device__ constexpr int range_deg(int lo, int k) {
  int d = lo;
  while (k >= ncart(d)) {
    k -= ncart(d);
    ++d;
  }
  return d;
}
__host__ __device__ constexpr int range_idx(int lo, int k) {
  int d = lo;
  while (k >= ncart(d)) {
    k -= ncart(d);
    ++d;
  }
  return k;
}
__host__ __device__ constexpr int range_x(int lo, int k) { return comp_lx(range_deg(lo, k), range_idx(lo, k)); }
__host__ __device__ constexpr int range_y(int lo, int k) { return comp_ly(range_deg(lo, k), range_idx(lo, k)); }
__host__ __device__ constexpr int range_z(int lo, int k) { return comp_lz(range_deg(lo, k), range_idx(lo, k)); }

// Pair class pc = l_a(l_a+1)/2 + l_b (l_a >= l_b) and back.
__host__ __device__ constexpr int pc_la(int pc) {
  int la = 0;
  while ((la + 1) * (la + 2) / 2 <= pc) ++la;
  return la;
}
__host__ __device__ constexpr int pc_lb(int pc) { return pc - pc_la(pc) * (pc_la(pc) + 1) / 2; }

// cart_index / addr (src/math/am.rs:51-55, src/engine/os_eri.rs:129-137)
__host__ __device__ inline int cart_index3(int lx, int ly, int lz) {
  int d = ly + lz;
  return d * (d + 1) / 2 + lz;
}
__host__ __device__ inline int addr3(int lx, int ly, int lz) {
  return tri_below(lx + ly + lz) + cart_index3(lx, ly, lz);
}

template <int N, typename F, int... I>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}
// Calls f(std::integral_constant<int, i>) for i = 0 .. N-1, fully unrolled.
template <int N, typename F>
__device__ __forceinline__ void static_for(F&& f) {
  static_for_impl<N>(static_cast<F&&>(f), std::make_integer_sequence<int, N>{});
}

// ----------------------------------------------------------- device tables

// Each translation unit (one per bra pair class) is its own device module,
// so every module carries its own copy of these tables, filled by its
// upload_module_constants().
// Triples by global address (degree <= 20): packed lx | ly<<8 | lz<<16.
constexpr int ADDR_TAB_DEG = ADDR_TAB_DEG_HOST;
static __constant__ int c_addr_lxyz[n_addr(ADDR_TAB_DEG)];
static __constant__ RysMeta c_rys[MAX_ROOTS + 1];
static __constant__ double c_lag_x[MAX_ROOTS][MAX_ROOTS];
static __constant__ double c_lag_w[MAX_ROOTS][MAX_ROOTS];
static __constant__ float c_lag_xf[MAX_ROOTS][MAX_ROOTS];
static __constant__ float c_lag_wf[MAX_ROOTS][MAX_ROOTS];
static __constant__ const double* c_rys_tab;
static __constant__ const float* c_rys_tab_f;

static inline cudaError_t upload_module_constants(const ConstData& c) {
  cudaError_t e;
  if ((e = cudaMemcpyToSymbol(c_addr_lxyz, c.addr_lxyz, sizeof(int) * c.n_addr))) return e;
  if ((e = cudaMemcpyToSymbol(c_rys, c.meta, sizeof(RysMeta) * (MAX_ROOTS + 1)))) return e;
  if ((e = cudaMemcpyToSymbol(c_lag_x, c.lag_x, sizeof(double) * MAX_ROOTS * MAX_ROOTS))) return e;
  if ((e = cudaMemcpyToSymbol(c_lag_w, c.lag_w, sizeof(double) * MAX_ROOTS * MAX_ROOTS))) return e;
  if ((e = cudaMemcpyToSymbol(c_lag_xf, c.lag_xf, sizeof(float) * MAX_ROOTS * MAX_ROOTS))) return e;
  if ((e = cudaMemcpyToSymbol(c_lag_wf, c.lag_wf, sizeof(float) * MAX_ROOTS * MAX_ROOTS))) return e;
  if ((e = cudaMemcpyToSymbol(c_rys_tab, &c.tab, sizeof(c.tab)))) return e;
  if ((e = cudaMemcpyToSymbol(c_rys_tab_f, &c.tab_f, sizeof(c.tab_f)))) return e;
  return cudaSuccess;
}

__device__ __forceinline__ int addr_lx(int a) { return c_addr_lxyz[a] & 0xff; }
__device__ __forceinline__ int addr_ly(int a) { return (c_addr_lxyz[a] >> 8) & 0xff; }
__device__ __forceinline__ int addr_lz(int a) { return (c_addr_lxyz[a] >> 16) & 0xff; }

// ----------------------------------------------------------------- Rys

template <typename R>
__device__ __forceinline__ R chebev(const R* __restrict__ c, R xi) {
  R two_xi = R(2) * xi;
  R d = R(0), dd = R(0);
#pragma unroll
  for (int k = RYS_NC - 1; k >= 1; --k) {
    R sv = d;
    d = two_xi * d - dd + __ldg(c + k);
    dd = sv;
  }
  return xi * d - dd + R(0.5) * __ldg(c);
}

// Largest number of Chebyshev subintervals of any n (15 for n = 13).
constexpr int RYS_MAX_SUB = 16;

// Copy the N-root table (all subintervals) into shared memory; every thread
// of the block must call it.  Lookups of different T by the lanes of a warp
// are then shared-memory reads instead of scattered L1 sectors.
template <int N, typename R>
__device__ __forceinline__ void stage_rys_table(R* s_tab) {
  const RysMeta m = c_rys[N];
  const R* src;
  if constexpr (sizeof(R) == 8)
    src = c_rys_tab + m.off;
  else
    src = c_rys_tab_f + m.off;
  const int sub = m.n_sub < RYS_MAX_SUB ? m.n_sub : RYS_MAX_SUB;
  const int cnt = sub * N * 2 * RYS_NC;
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) s_tab[i] = __ldg(src + i);
  __syncthreads();
}

template <typename R>
__device__ __forceinline__ R chebev_s(const R* c, R xi) {
  R two_xi = R(2) * xi;
  R d = R(0), dd = R(0);
#pragma unroll
  for (int k = RYS_NC - 1; k >= 1; --k) {
    R sv = d;
    d = two_xi * d - dd + c[k];
    dd = sv;
  }
  return xi * d - dd + R(0.5) * c[0];
}

// Roots/weights from the shared-memory copy of the N-root table.
template <int N, typename R>
__device__ __forceinline__ void rys_roots_s(const R* s_tab, R T, R* x, R* w) {
  const RysMeta m = c_rys[N];
  if (T >= R(m.t_hi)) {
    R inv_t = R(1) / T;
    R sc = R(0.5) * rsqrt(T);
#pragma unroll
    for (int i = 0; i < N; ++i) {
      if constexpr (sizeof(R) == 8) {
        x[i] = c_lag_x[N - 1][i] * inv_t;
        w[i] = c_lag_w[N - 1][i] * sc;
      } else {
        x[i] = c_lag_xf[N - 1][i] * inv_t;
        w[i] = c_lag_wf[N - 1][i] * sc;
      }
    }
    return;
  }
  R width = R(m.width);
  int s = (int)(T / width);
  s = s < 0 ? 0 : (s >= m.n_sub ? m.n_sub - 1 : s);
  R a = R(s) * width;
  R b = a + width;
  R xi = (R(2) * T - (a + b)) / (b - a);
  const R* base = s_tab + (size_t)s * N * 2 * RYS_NC;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    x[i] = chebev_s<R>(base + (2 * i) * RYS_NC, xi);
    w[i] = chebev_s<R>(base + (2 * i + 1) * RYS_NC, xi);
  }
}

// N-point Rys quadrature at parameter T (src/math/rys.rs:174-215): the
// generalized-Laguerre(-1/2) limit above asymptotic_boundary(2N-1), else the
// piecewise Chebyshev interpolation.  x = squared roots, w = weights.
template <int N, typename R>
__device__ __forceinline__ void rys_roots(R T, R* x, R* w) {
  const RysMeta m = c_rys[N];
  if (T >= R(m.t_hi)) {
    R inv_t = R(1) / T;
    R sc = R(0.5) * rsqrt(T);
#pragma unroll
    for (int i = 0; i < N; ++i) {
      if constexpr (sizeof(R) == 8) {
        x[i] = c_lag_x[N - 1][i] * inv_t;
        w[i] = c_lag_w[N - 1][i] * sc;
      } else {
        x[i] = c_lag_xf[N - 1][i] * inv_t;
        w[i] = c_lag_wf[N - 1][i] * sc;
      }
    }
    return;
  }
  R width = R(m.width);
  int s = (int)(T / width);
  s = s < 0 ? 0 : (s >= m.n_sub ? m.n_sub - 1 : s);
  R a = R(s) * width;
  R b = a + width;
  R xi = (R(2) * T - (a + b)) / (b - a);
  const R* base;
  if constexpr (sizeof(R) == 8)
    base = c_rys_tab + m.off + (size_t)s * N * 2 * RYS_NC;
  else
    base = c_rys_tab_f + m.off + (size_t)s * N * 2 * RYS_NC;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    x[i] = chebev<R>(base + (2 * i) * RYS_NC, xi);
    w[i] = chebev<R>(base + (2 * i + 1) * RYS_NC, xi);
  }
}

// Per-axis Rys vertical recurrence g[n][m], n <= NE (bra power on A),
// m <= NF (ket power on C), seeded with g[0][0] = g00 (src/engine/rys.rs:
// 246-268; the seed scales the whole table, which folds the weight and
// prefactor into one axis).
template <int NE, int NF, typename R>
__device__ __forceinline__ void vrr_axis(R g00, R c00, R cp0, R b10, R b01, R b00,
                                         R (&g)[NE + 1][NF + 1]) {
  g[0][0] = g00;
  if constexpr (NE >= 1) g[1][0] = c00 * g00;
#pragma unroll
  for (int n = 1; n < NE; ++n) g[n + 1][0] = c00 * g[n][0] + R(n) * b10 * g[n - 1][0];
#pragma unroll
  for (int m = 0; m < NF; ++m) {
#pragma unroll
    for (int n = 0; n <= NE; ++n) {
      R t = cp0 * g[n][m];
      if (m >= 1) t += R(m) * b01 * g[n][m - 1];
      if (n >= 1) t += R(n) * b00 * g[n - 1][m];
      g[n][m + 1] = t;
    }
  }
}

// Per-primitive-quartet scalars of the Rys quadrature (src/engine/rys.rs:
// 140-166) in evaluation orientation.  For the long-range operator
// erf(omega r)/r (omega > 0, src/engine/rys.rs:163-175) the quadrature is
// taken at s*T with s = omega^2 / (rho + omega^2), every root scaled by s
// (xs) and every weight by sqrt(s) (folded into pref); omega = 0 is the
// Coulomb operator, with T and pref untouched and xs = 1.
template <typename R>
struct QuartetHdr {
  R T, pref, pq, p, q;
  R pqx, pqy, pqz;  // P - Q
  R pax, pay, paz;  // P - A
  R qcx, qcy, qcz;  // Q - C
  R xs;             // root scale (1 for Coulomb)
};

template <typename R>
__device__ __forceinline__ QuartetHdr<R> quartet_header(const PrimPairD& bp, const PrimPairD& kp,
                                                        double omega) {
  QuartetHdr<R> h;
  // 2 pi^{5/2}
  const double TWO_PI_2_5 = 34.98683665524972;
  R p = R(bp.zeta), q = R(kp.zeta);
  h.p = p;
  h.q = q;
  h.pq = p + q;
  R rho = p * q / h.pq;
  // centre differences in double first: absolute coordinates would lose
  // the separation to cancellation in FP32
  h.pqx = R(bp.px - kp.px);
  h.pqy = R(bp.py - kp.py);
  h.pqz = R(bp.pz - kp.pz);
  h.T = rho * (h.pqx * h.pqx + h.pqy * h.pqy + h.pqz * h.pqz);
  h.pref = R(TWO_PI_2_5) / (p * q * sqrt(h.pq)) * R(bp.e) * R(kp.e);
  h.pax = R(bp.pax);
  h.pay = R(bp.pay);
  h.paz = R(bp.paz);
  h.qcx = R(kp.pax);
  h.qcy = R(kp.pay);
  h.qcz = R(kp.paz);
  h.xs = R(1);
  if (omega > 0.0) {
    const R w2 = R(omega) * R(omega);
    const R sc = w2 / (rho + w2);
    h.T *= sc;
    h.pref *= sqrt(sc);
    h.xs = sc;
  }
  return h;
}

// The Rys parameter T of a primitive quartet in FP64 from the double pair
// data (the same expression as quartet_header, erf scaling included).
__device__ __forceinline__ double quartet_T64(const PrimPairD& bp, const PrimPairD& kp, double omega) {
  const double p = bp.zeta, q = kp.zeta, pq = p + q;
  const double rho = p * q / pq;
  const double dx = bp.px - kp.px, dy = bp.py - kp.py, dz = bp.pz - kp.pz;
  double T = rho * (dx * dx + dy * dy + dz * dz);
  if (omega > 0.0) T *= omega * omega / (rho + omega * omega);
  return T;
}

// Root r of the N-point quadrature at T, evaluated in FP64 from the double
// tables (the FP32 launches take this path for large T and high l).
template <int N>
__device__ __forceinline__ void rys_root_fp64(double T, int r, double& x, double& w) {
  const RysMeta m = c_rys[N];
  if (T >= m.t_hi) {
    x = c_lag_x[N - 1][r] / T;
    w = c_lag_w[N - 1][r] * 0.5 * rsqrt(T);
    return;
  }
  int s = (int)(T / m.width);
  s = s < 0 ? 0 : (s >= m.n_sub ? m.n_sub - 1 : s);
  const double a = (double)s * m.width, b = a + m.width;
  const double xi = (2.0 * T - (a + b)) / (b - a);
  const double* base = c_rys_tab + m.off + ((size_t)s * N + r) * 2 * RYS_NC;
  x = chebev<double>(base, xi);
  w = chebev<double>(base + RYS_NC, xi);
}

// The FP32 launches generate roots and weights in FP64 for every quadrature
// of five or more roots (high angular momentum, l_a + l_b + l_c + l_d >= 8):
// the n where Clenshaw sums lose digits just below the asymptotic crossover
// (the reference's own FP64 weights lose three to four there at n = 9, 11,
// 13, src/math/rys.rs:80-89) are all among them.  Above the crossover the
// roots and weights are the closed forms c_i / T and w_i T^{-1/2}, exact to
// FP32 rounding at every n.
constexpr int ROOTS64_NR = 5;
template <int N, typename R>
__device__ __forceinline__ bool roots_in_fp64(R) {
  return sizeof(R) == 4 && N >= ROOTS64_NR;
}

// quartet_header for the FP32 launches from the FP32 pair copies; ac = the
// bra's first evaluation shell centre minus the ket's, rounded once per
// quartet.
__device__ __forceinline__ QuartetHdr<float> quartet_header_f(const PrimPairF& bp, const PrimPairF& kp, float acx,
                                                              float acy, float acz, double omega) {
  QuartetHdr<float> h;
  const float p = bp.zeta, q = kp.zeta;
  h.p = p;
  h.q = q;
  h.pq = p + q;
  const float rho = p * q / h.pq;
  h.pqx = acx + (bp.pax - kp.pax);
  h.pqy = acy + (bp.pay - kp.pay);
  h.pqz = acz + (bp.paz - kp.paz);
  h.T = rho * (h.pqx * h.pqx + h.pqy * h.pqy + h.pqz * h.pqz);
  h.pref = 34.98683665524972f / (p * q * sqrtf(h.pq)) * bp.e * kp.e;
  h.pax = bp.pax;
  h.pay = bp.pay;
  h.paz = bp.paz;
  h.qcx = kp.pax;
  h.qcy = kp.pay;
  h.qcz = kp.paz;
  h.xs = 1.f;
  if (omega > 0.0) {
    const float w2 = float(omega) * float(omega);
    const float sc = w2 / (rho + w2);
    h.T *= sc;
    h.pref *= sqrtf(sc);
    h.xs = sc;
  }
  return h;
}

// ----------------------------------------------------------- misc device

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
// Identity of one screened canonical quartet with its density mask; the sum
// over the list (mod 2^64) fingerprints the list independent of order.
__device__ __forceinline__ uint64_t quartet_key(int i, int j, int k, int l, uint64_t mask) {
  uint64_t id = ((((uint64_t)i * 65536u + (uint64_t)j) * 65536u + (uint64_t)k) * 65536u) + (uint64_t)l;
  return splitmix64(id ^ splitmix64(mask + 0x5851F42D4C957F2Dull));
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace igpu
