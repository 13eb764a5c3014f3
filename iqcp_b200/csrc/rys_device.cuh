// Device Boys function and Rys quadrature.
//
// Rys rule (roots as t^2 in [0,1), weights) for n roots at argument T: the
// same quantities rys_roots returns in the reference (rys/mod.rs:253), which
// computes them per call from moments with Schmidt orthogonalisation and a
// companion-matrix QR (rys/mod.rs:468-790).  On the device a per-call
// eigen-solve diverges across lanes, so the rule is read from tables instead:
// degree-11 Chebyshev series on unit intervals of T up to Tasym(n), and the
// large-T Hermite limit (roots y_i/T, weights W_i/sqrt(T)) beyond it.  The
// tables (rys_tables.inc, made by gen_rys_tables.cpp in binary128) are exact
// to ~3e-16 relative, i.e. closer to the true rule than the reference's own
// FP64 moment method.
//
// Boys F_0..F_m(T): the reference's regime split (boys/mod.rs:587-618: series
// at the highest order plus downward recurrence below the m_max turnover,
// erf + upward recurrence above it), with CUDA's erf/exp.
#pragma once
#include <cuda_runtime.h>

#define RYS_TAB_QUAL __device__ const
#include "rys_tables.inc"
#undef RYS_TAB_QUAL

namespace iqcp {

// unit intervals below Tasym(n)
__host__ __device__ constexpr int rys_nint(int n) {
  constexpr int t[RYS_TAB_MAXN + 1] = RYS_TAB_NINT;
  return t[n];
}
// Shared-memory copy of the order-N table: [interval][root 0..N-1, weight
// 0..N-1][coefficient], interval stride padded to an odd number of doubles so
// that lanes reading different intervals fall on different bank pairs.
template <int N>
__host__ __device__ constexpr int rys_tab_stride() { return 2 * N * (RYS_TAB_DEG + 1) + 1; }
template <int N>
__host__ __device__ constexpr int rys_tab_doubles() { return rys_nint(N) * rys_tab_stride<N>(); }

// Copy the order-N table into shared memory (all threads of the block).  Each
// lane reads the interval of its own T, so table reads are scattered: from
// shared memory they cost a few bank wavefronts, from L1 one cache line per lane.
template <int N>
__device__ __forceinline__ void rys_stage_table(double* __restrict__ s) {
  constexpr int W = 2 * N * (RYS_TAB_DEG + 1);
  const double* g = kRysCheb + kRysOffset[N];
  for (int i = threadIdx.x; i < rys_nint(N) * W; i += blockDim.x) {
    const int k = i / W;
    s[k * rys_tab_stride<N>() + (i - k * W)] = __ldg(g + i);
  }
}

__device__ __forceinline__ double cheb_clenshaw_s(const double* c, double x2) {
  double b1 = 0.0, b2 = 0.0;
#pragma unroll
  for (int j = RYS_TAB_DEG; j >= 1; --j) {
    const double t = fma(x2, b1, c[j] - b2);
    b2 = b1;
    b1 = t;
  }
  return fma(0.5 * x2, b1, c[0] - b2);
}

// rys_rule with the order-N table staged in shared memory at `s`
template <int N>
__device__ __forceinline__ void rys_rule_tab(double T, const double* s, double* __restrict__ r,
                                             double* __restrict__ w) {
  constexpr int NI = rys_nint(N);
  if (T >= double(NI)) {
    const double it = 1.0 / T;
    const double is = 1.0 / sqrt(T);
    const int base = (N * (N - 1)) / 2;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      r[i] = __ldg(kRysAsymRoot + base + i) * it;
      w[i] = __ldg(kRysAsymWeight + base + i) * is;
    }
    return;
  }
  const int k = int(T);
  const double x2 = 2.0 * (2.0 * (T - double(k)) - 1.0);
  const double* c = s + k * rys_tab_stride<N>();
#pragma unroll
  for (int i = 0; i < N; ++i) {
    r[i] = cheb_clenshaw_s(c + i * (RYS_TAB_DEG + 1), x2);
    w[i] = cheb_clenshaw_s(c + (N + i) * (RYS_TAB_DEG + 1), x2);
  }
}

__device__ __forceinline__ double cheb_clenshaw(const double* __restrict__ c, double x2) {
  // x2 = 2x; sum_j c_j T_j(x)
  double b1 = 0.0, b2 = 0.0;
#pragma unroll
  for (int j = RYS_TAB_DEG; j >= 1; --j) {
    const double t = fma(x2, b1, __ldg(c + j) - b2);
    b2 = b1;
    b1 = t;
  }
  return fma(0.5 * x2, b1, __ldg(c) - b2);
}

template <int N>
__device__ __forceinline__ void rys_rule(double T, double* __restrict__ r, double* __restrict__ w) {
  static_assert(N >= 1 && N <= RYS_TAB_MAXN, "unsupported Rys order");
  if (T >= double(kRysTasym[N])) {
    const double it = 1.0 / T;
    const double is = 1.0 / sqrt(T);
    const int base = (N * (N - 1)) / 2;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      r[i] = __ldg(kRysAsymRoot + base + i) * it;
      w[i] = __ldg(kRysAsymWeight + base + i) * is;
    }
    return;
  }
  const int k = int(T);  // unit-width intervals
  const double x2 = 2.0 * (2.0 * (T - double(k)) - 1.0);
  const double* c = kRysCheb + kRysOffset[N] + k * (2 * N * (RYS_TAB_DEG + 1));
#pragma unroll
  for (int i = 0; i < N; ++i) {
    r[i] = cheb_clenshaw(c + i * (RYS_TAB_DEG + 1), x2);
    w[i] = cheb_clenshaw(c + (N + i) * (RYS_TAB_DEG + 1), x2);
  }
}

// Runtime-order dispatch (tests / batch entry point)
__device__ inline void rys_rule_n(int n, double T, double* r, double* w) {
  switch (n) {
    case 1: rys_rule<1>(T, r, w); break;
    case 2: rys_rule<2>(T, r, w); break;
    case 3: rys_rule<3>(T, r, w); break;
    case 4: rys_rule<4>(T, r, w); break;
    case 5: rys_rule<5>(T, r, w); break;
    case 6: rys_rule<6>(T, r, w); break;
    case 7: rys_rule<7>(T, r, w); break;
    default: break;
  }
}

__device__ __forceinline__ double boys_turnover(int m) {
  // boys/mod.rs:67-108 (m-dependent series/recurrence switch)
  const double tab[16] = {0.0, 0.0, 0.866025403784, 1.295010032056, 1.705493613097,
                          2.106432965305, 2.501471934009, 2.892473348218, 3.280525047072,
                          3.666320693281, 4.05033123037, 4.432891808508, 4.814249856864,
                          5.194593501454, 5.574069276051, 5.952793645111};
  return m < 16 ? tab[m] : 5.952793645111 + 0.372 * double(m - 15);
}

// F_0..F_m(T) into f[0..m] (m <= 31)
__device__ inline void boys_all_dev(int m, double T, double* f) {
  if (T < 1e-14) {
    for (int i = 0; i <= m; ++i) f[i] = 1.0 / (2.0 * i + 1.0);
    return;
  }
  if (T < boys_turnover(m)) {
    const double b = m + 0.5;
    const double e = 0.5 * exp(-T);
    double term = e, sum = e, den = b + 1.0;
    const double tol = 1.1102230246251565e-16 * e;
    for (int it = 0; it < 200 && term > tol; ++it) {
      term *= T / den;
      sum += term;
      den += 1.0;
    }
    f[m] = sum / b;
    double bc = b;
    for (int i = m; i >= 1; --i) {
      bc -= 1.0;
      f[i - 1] = (e + T * f[i]) / bc;
    }
  } else {
    const double st = sqrt(T);
    f[0] = 0.88622692545275801365 / st * erf(st);
    const double e = exp(-T);
    const double h = 0.5 / T;
    for (int i = 1; i <= m; ++i) f[i] = h * ((2 * i - 1) * f[i - 1] - e);
  }
}

}  // namespace iqcp
