// CPU oracle (TEST INFRASTRUCTURE ONLY): Boys function and Rys quadrature.
//
// Restates, operation by operation, the reference's FP64 algorithms:
//   * boys_all   <- crates/qc-core/src/boys/mod.rs:587-618 (boys_all_internal),
//                   series :481-540, erf + upward recurrence :557-579,
//                   turnover table :67-108 (regime chosen by the HIGHEST order).
//   * rys_roots  <- crates/qc-core/src/rys/mod.rs:253-286 (moments F_0..F_2n),
//                   rdk_rys_roots :468-562, schmidt_orthogonalize :585-660,
//                   polynomial_roots :687-790, hessenberg_qr :801-878,
//                   qr_step :881-950, bisection_refine :953-1039.
// erf is glibc's, which shares fdlibm's s_erf.c algorithm with the Rust `libm`
// 0.2.16 crate the reference calls (boys/mod.rs:649-651).
//
// The pipeline is written once over its working type F.  F = double is the
// reference's arithmetic and what every parity fixture uses.  F = long double
// (x87 extended, 64-bit significand) runs the same steps with tolerances
// scaled to that precision and rounds the result to double: the moment method
// loses about cond(Hankel) digits (relative root errors ~2e-11 at 5 roots and
// ~5e-10 at 6 in double), so the extended form gives a second, more accurate
// reading of the same algorithm, to tell the reference's own rounding apart
// from a device-side error (set_root_precision).
#include <cmath>
#include <cfloat>
#include <cstring>

#include "oracle_internal.h"

namespace oracle {
namespace {

// boys/mod.rs:67-108 -- m-dependent switch between series and erf recurrence.
const double kTurnover[40] = {
    0.0, 0.0, 0.866025403784, 1.295010032056, 1.705493613097, 2.106432965305,
    2.501471934009, 2.892473348218, 3.280525047072, 3.666320693281, 4.05033123037,
    4.432891808508, 4.814249856864, 5.194593501454, 5.574069276051, 5.952793645111,
    6.330860773135, 6.708347923415, 7.08531930745, 7.461828891625, 7.837922483937,
    8.213639312398, 8.589013237349, 8.964073695432, 9.338846443746, 9.713354153046,
    10.08761688545, 10.46165248270, 10.83547688448, 11.20910439128, 11.58254788331,
    11.95581900374, 12.32892831326, 12.70188542111, 13.07469909673, 13.44737736550,
    13.81992759110, 14.19235654675, 14.56467047710, 14.93687515212};

double turnover(int m) {
  if (m < 40) return kTurnover[m];
  return 14.93687515212 + 0.372 * (double(m) - 39.0);
}

constexpr double kSqrtPiOver4 = 0.8862269254527580136490837416705725913987747280611935641069038949264;

// Working-precision constants: the reference's for double (THRESHOLD_ZERO,
// the QR and root tolerances of rys/mod.rs), three orders of magnitude
// tighter for the extended type.
template <typename F> struct Prec;
template <> struct Prec<double> {
  static constexpr double kEps = DBL_EPSILON;
  static constexpr double kSqrtPiOver4 = oracle::kSqrtPiOver4;
  static constexpr double kThresholdZero = DBL_EPSILON * 8.0;
  static constexpr int kQrMaxIter = 30;
  static constexpr double kQrEps = 1e-15;
  static constexpr double kRootAccuracy = 1e-15;
};
template <> struct Prec<long double> {
  static constexpr long double kEps = LDBL_EPSILON;
  static constexpr long double kSqrtPiOver4 =
      0.8862269254527580136490837416705725913987747280611935641069038949264L;
  static constexpr long double kThresholdZero = LDBL_EPSILON * 8.0L;
  static constexpr int kQrMaxIter = 60;
  static constexpr long double kQrEps = 1e-18L;
  static constexpr long double kRootAccuracy = 1e-18L;
};

int g_root_precision = 0;  // 0: double (the reference's), 1: extended

}  // namespace

template <typename F>
void boys_all_t(int m_max, F t, F* f) {
  if (t < 1e-14) {                       // NEAR_ZERO_THRESHOLD
    for (int i = 0; i <= m_max; ++i) f[i] = 1.0 / (2.0 * F(i) + 1.0);
    return;
  }
  if (t < turnover(m_max)) {
    // Series at the top order, then downward recurrence.
    const F b = F(m_max) + 0.5;
    const F e = 0.5 * std::exp(-t);
    F term = e, sum = e;
    const F tol = (Prec<F>::kEps * 0.5) * e;
    F den = b + 1.0;
    while (term > tol) {
      term *= t / den;
      sum += term;
      den += 1.0;
    }
    f[m_max] = sum / b;
    F bc = b;
    for (int i = m_max; i >= 1; --i) {
      bc -= 1.0;
      f[i - 1] = (e + t * f[i]) / bc;
    }
  } else {
    const F st = std::sqrt(t);
    f[0] = Prec<F>::kSqrtPiOver4 / st * std::erf(st);
    const F e = std::exp(-t);
    const F h = 0.5 / t;
    for (int i = 1; i <= m_max; ++i) f[i] = h * (F(2 * i - 1) * f[i - 1] - e);
  }
}

void boys_all(int m_max, double t, double* f) { boys_all_t<double>(m_max, t, f); }

namespace {

constexpr int kBisectMaxIter = 200;

enum {
  kErrSchmidt = -1,
  kErrRootFinding = -2,
  kErrRange = -3,
  kErrWeight = -4,
};

// Gram-Schmidt on the monomials with the moment inner product; cs is
// column-major (cs[i + j*n] = coefficient of x^i in P_j).
template <typename F>
int schmidt(F* cs, const F* mu, int n) {
  F v[kMaxRoots + 1];
  cs[0] = 1.0 / std::sqrt(mu[0]);
  const F fac1 = -mu[1] / mu[0];
  const F t1 = mu[2] + fac1 * mu[1];
  if (t1 <= 0.0) return kErrSchmidt;
  const F r1 = 1.0 / std::sqrt(t1);
  cs[n] = fac1 * r1;
  cs[1 + n] = r1;
  for (int j = 2; j < n; ++j) {
    for (int i = 0; i < j; ++i) v[i] = 0.0;
    F fac = mu[2 * j];
    for (int k = 0; k < j; ++k) {
      F dot = 0.0;
      for (int i = 0; i <= k; ++i) dot += cs[i + k * n] * mu[i + j];
      for (int i = 0; i <= k; ++i) v[i] -= dot * cs[i + k * n];
      fac -= dot * dot;
    }
    if (fac <= 0.0) {
      if (fac == 0.0) {
        for (int jj = j; jj < n; ++jj)
          for (int ii = 0; ii <= jj; ++ii) cs[ii + jj * n] = 0.0;
        return 0;
      }
      return kErrSchmidt;
    }
    const F r = 1.0 / std::sqrt(fac);
    cs[j + j * n] = r;
    for (int k = 0; k < j; ++k) cs[k + j * n] = r * v[k];
  }
  return 0;
}

// One shifted QR sweep (Givens) on the active block [n0, n1) of the
// row-major nr x nr Hessenberg matrix a.
template <typename F>
void qr_sweep(F* a, int nr, int n0, int n1, F shift) {
  const int m1 = n0 + 1;
  F cv = a[n0 * nr + n0] - shift;
  F sv = a[m1 * nr + n0];
  F v = std::sqrt(cv * cv + sv * sv);
  F c = 1.0, s = 0.0;
  if (v != 0.0) { c = cv / v; s = sv / v; }
  for (int k = n0; k < nr; ++k) {
    const F x = a[n0 * nr + k], y = a[m1 * nr + k];
    a[n0 * nr + k] = c * x + s * y;
    a[m1 * nr + k] = c * y - s * x;
  }
  int m3 = n1 < n0 + 3 ? n1 : n0 + 3;
  for (int k = 0; k < m3; ++k) {
    const F x = a[k * nr + n0], y = a[k * nr + m1];
    a[k * nr + n0] = c * x + s * y;
    a[k * nr + m1] = c * y - s * x;
  }
  for (int j = n0; j < n1 - 2; ++j) {
    const int j1 = j + 1, j2 = j + 2;
    cv = a[j1 * nr + j];
    sv = a[j2 * nr + j];
    v = std::sqrt(cv * cv + sv * sv);
    a[j1 * nr + j] = v;
    a[j2 * nr + j] = 0.0;
    c = 1.0; s = 0.0;
    if (v != 0.0) { c = cv / v; s = sv / v; }
    for (int k = j1; k < nr; ++k) {
      const F x = a[j1 * nr + k], y = a[j2 * nr + k];
      a[j1 * nr + k] = c * x + s * y;
      a[j2 * nr + k] = c * y - s * x;
    }
    m3 = n1 < j + 4 ? n1 : j + 4;
    for (int k = 0; k < m3; ++k) {
      const F x = a[k * nr + j1], y = a[k * nr + j2];
      a[k * nr + j1] = c * x + s * y;
      a[k * nr + j2] = c * y - s * x;
    }
  }
}

template <typename F>
int hessenberg_eig(F* a, int nr) {
  int n0 = 0, n1 = nr, its = 0;
  for (int ic = 0; ic < nr * Prec<F>::kQrMaxIter; ++ic) {
    int k = n0;
    while (k + 1 < n1) {
      const F s = std::fabs(a[k * nr + k]) + std::fabs(a[(k + 1) * nr + k + 1]);
      if (std::fabs(a[(k + 1) * nr + k]) < Prec<F>::kQrEps * s) break;
      ++k;
    }
    const int k1 = k + 1;
    if (k1 < n1) {
      a[k1 * nr + k] = 0.0;
      n0 = k1;
      its = 0;
      if (n0 + 1 >= n1) {
        n0 = 0;
        n1 = k1;
        if (n1 < 2) return 0;
      }
    } else {
      const int m1 = n1 - 1, m2 = n1 - 2;
      const F a11 = a[m1 * nr + m1], a22 = a[m2 * nr + m2];
      const F tr = a11 + a22;
      F disc = (a11 - a22) * (a11 - a22);
      disc += 4.0 * a[m1 * nr + m2] * a[m2 * nr + m1];
      F shift;
      if (disc > 0.0) {
        const F sq = std::sqrt(disc);
        const F r1 = (tr + sq) * 0.5, r2 = (tr - sq) * 0.5;
        shift = std::fabs(a11 - r1) > std::fabs(a11 - r2) ? r2 : r1;
      } else {
        if (n1 == 2) return kErrRootFinding;
        shift = tr * 0.5;
      }
      ++its;
      qr_sweep(a, nr, n0, n1, shift);
      if (its > Prec<F>::kQrMaxIter) return kErrRootFinding;
    }
  }
  return kErrRootFinding;
}

template <typename F>
F horner(const F* c, int order, F x) {
  F p = c[order];
  for (int i = 1; i <= order; ++i) p = p * x + c[order - i];
  return p;
}

template <typename F>
int bisect_refine(const F* cs, F* roots, int order, int n1) {
  const F* a = cs + order * n1;
  F x1i = 0.0, p1i = a[0];
  for (int m = 0; m < order; ++m) {
    const F x0i = x1i, p0i = p1i;
    x1i = roots[m];
    p1i = horner(a, order, x1i);
    if (p1i == 0.0) continue;
    if (p0i * p1i > 0.0) return kErrRootFinding;
    F x0, x1, p0, p1;
    if (x0i <= x1i) { x0 = x0i; x1 = x1i; p0 = p0i; p1 = p1i; }
    else { x0 = x1i; x1 = x0i; p0 = p1i; p1 = p0i; }
    if (p1 == 0.0) { roots[m] = x1; continue; }
    if (p0 == 0.0) { roots[m] = x0; continue; }
    F xi = x0 + (x0 - x1) / (p1 - p0) * p0;
    for (int it = 0; it < kBisectMaxIter; ++it) {
      if (std::fabs(x1 - x0) <= x1 * Prec<F>::kRootAccuracy) break;
      F pi = horner(a, order, xi);
      if (pi == 0.0) break;
      if (p0 * pi <= 0.0) { x1 = xi; p1 = pi; xi = x0 * 0.25 + xi * 0.75; }
      else { x0 = xi; p0 = pi; xi = xi * 0.75 + x1 * 0.25; }
      pi = horner(a, order, xi);
      if (pi == 0.0) break;
      if (p0 * pi <= 0.0) { x1 = xi; p1 = pi; }
      else { x0 = xi; p0 = pi; }
      xi = x0 + (x0 - x1) / (p1 - p0) * p0;
    }
    roots[m] = xi;
  }
  return 0;
}

template <typename F>
int poly_roots(F* roots, const F* cs, int nr, int n1) {
  if (nr == 1) {
    roots[0] = -cs[n1] / cs[1 + n1];
    return 0;
  }
  if (nr == 2) {
    const F a = cs[2 + 2 * n1], b = cs[1 + 2 * n1], c = cs[2 * n1];
    const F disc = b * b - 4.0 * a * c;
    if (disc < 0.0) return kErrRootFinding;
    const F sq = std::sqrt(disc);
    roots[0] = (-b - sq) / (2.0 * a);
    roots[1] = (-b + sq) / (2.0 * a);
    return 0;
  }
  F a[kMaxRoots * kMaxRoots];
  std::memset(a, 0, sizeof(a));
  const F lead = cs[nr + nr * n1];
  if (std::fabs(lead) < Prec<F>::kThresholdZero) return kErrRootFinding;
  const F fac = -1.0 / lead;
  for (int i = 0; i < nr; ++i) a[nr - 1 - i] = cs[nr * n1 + i] * fac;
  for (int i = 0; i < nr - 1; ++i) a[(i + 1) * nr + i] = 1.0;
  if (hessenberg_eig(a, nr) == 0) {
    for (int i = 0; i < nr; ++i) roots[nr - 1 - i] = a[i * nr + i];
    return 0;
  }
  // QR gave up: seed from the quadratic and bisect orders 3..nr.
  const F qa = cs[2 + 2 * n1], qb = cs[1 + 2 * n1], qc = cs[2 * n1];
  const F disc = qb * qb - 4.0 * qa * qc;
  const F sq = disc >= 0.0 ? std::sqrt(disc) : 0.0;
  roots[0] = 0.5 * (-qb - sq) / qa;
  roots[1] = 0.5 * (-qb + sq) / qa;
  for (int i = 2; i < nr; ++i) roots[i] = 1.0;
  for (int k = 2; k < nr; ++k) {
    const int rc = bisect_refine(cs, roots, k + 1, n1);
    if (rc) return rc;
  }
  return 0;
}

template <typename F>
int rys_roots_t(int nroots, F t, F* roots, F* weights) {
  if (nroots < 1 || nroots > kMaxRoots) return -10;
  if (t < 0.0) return -11;
  F mu[2 * kMaxRoots + 1];
  boys_all_t<F>(2 * nroots, t, mu);

  if (std::fabs(mu[0]) < Prec<F>::kThresholdZero) {
    for (int i = 0; i < nroots; ++i) roots[i] = weights[i] = 0.0;
    return 0;
  }
  if (nroots == 1) {
    const F ratio = mu[1] / (mu[0] - mu[1]);
    roots[0] = ratio >= 0.0 ? ratio / (1.0 + ratio) : 0.0;
    weights[0] = mu[0];
    return 0;  // special method: not validated in the reference either
  }
  const int n1 = nroots + 1;
  F cs[(kMaxRoots + 1) * (kMaxRoots + 1)];
  std::memset(cs, 0, sizeof(cs));
  int rc = schmidt(cs, mu, n1);
  if (rc) return rc;
  F r[kMaxRoots] = {0};
  rc = poly_roots(r, cs, nroots, n1);
  if (rc) return rc;
  F w[kMaxRoots] = {0};
  for (int k = 0; k < nroots; ++k) {
    const F x = r[k];
    if (std::fabs(x - 1.0) < Prec<F>::kThresholdZero) {
      r[k] = 0.0;
      w[k] = 0.0;
      continue;
    }
    F dum = 1.0 / mu[0];
    for (int j = 1; j < nroots; ++j) {
      const F p = horner(cs + j * n1, j, x);
      dum += p * p;
    }
    w[k] = 1.0 / dum;
  }
  for (int k = 0; k < nroots; ++k) {
    if (!(r[k] >= 0.0 && r[k] < 1.0)) return kErrRange;
    if (w[k] < 0.0) return kErrWeight;
  }
  for (int k = 0; k < nroots; ++k) { roots[k] = r[k]; weights[k] = w[k]; }
  return 0;
}

}  // namespace

void set_root_precision(int extended) { g_root_precision = extended ? 1 : 0; }
int root_precision() { return g_root_precision; }

int rys_roots(int nroots, double t, double* roots, double* weights) {
  if (!g_root_precision) return rys_roots_t<double>(nroots, t, roots, weights);
  long double r[kMaxRoots], w[kMaxRoots];
  const int rc = rys_roots_t<long double>(nroots, (long double)t, r, w);
  if (rc == 0)
    for (int i = 0; i < nroots; ++i) { roots[i] = double(r[i]); weights[i] = double(w[i]); }
  return rc;
}

}  // namespace oracle
