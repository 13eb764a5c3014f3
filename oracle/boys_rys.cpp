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

const double kSqrtPiOver4 = 0.8862269254527580136490837416705725913987747280611935641069038949264;

}  // namespace

void boys_all(int m_max, double t, double* f) {
  if (t < 1e-14) {                       // NEAR_ZERO_THRESHOLD
    for (int i = 0; i <= m_max; ++i) f[i] = 1.0 / (2.0 * double(i) + 1.0);
    return;
  }
  if (t < turnover(m_max)) {
    // Series at the top order, then downward recurrence.
    const double b = double(m_max) + 0.5;
    const double e = 0.5 * std::exp(-t);
    double term = e, sum = e;
    const double tol = (DBL_EPSILON * 0.5) * e;
    double den = b + 1.0;
    while (term > tol) {
      term *= t / den;
      sum += term;
      den += 1.0;
    }
    f[m_max] = sum / b;
    double bc = b;
    for (int i = m_max; i >= 1; --i) {
      bc -= 1.0;
      f[i - 1] = (e + t * f[i]) / bc;
    }
  } else {
    const double st = std::sqrt(t);
    f[0] = kSqrtPiOver4 / st * std::erf(st);
    const double e = std::exp(-t);
    const double h = 0.5 / t;
    for (int i = 1; i <= m_max; ++i) f[i] = h * (double(2 * i - 1) * f[i - 1] - e);
  }
}

namespace {

constexpr double kThresholdZero = DBL_EPSILON * 8.0;
constexpr int kQrMaxIter = 30;
constexpr double kQrEps = 1e-15;
constexpr double kRootAccuracy = 1e-15;
constexpr int kBisectMaxIter = 200;

enum {
  kErrSchmidt = -1,
  kErrRootFinding = -2,
  kErrRange = -3,
  kErrWeight = -4,
};

// Gram-Schmidt on the monomials with the moment inner product; cs is
// column-major (cs[i + j*n] = coefficient of x^i in P_j).
int schmidt(double* cs, const double* mu, int n) {
  double v[kMaxRoots + 1];
  cs[0] = 1.0 / std::sqrt(mu[0]);
  const double fac1 = -mu[1] / mu[0];
  const double t1 = mu[2] + fac1 * mu[1];
  if (t1 <= 0.0) return kErrSchmidt;
  const double r1 = 1.0 / std::sqrt(t1);
  cs[n] = fac1 * r1;
  cs[1 + n] = r1;
  for (int j = 2; j < n; ++j) {
    for (int i = 0; i < j; ++i) v[i] = 0.0;
    double fac = mu[2 * j];
    for (int k = 0; k < j; ++k) {
      double dot = 0.0;
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
    const double r = 1.0 / std::sqrt(fac);
    cs[j + j * n] = r;
    for (int k = 0; k < j; ++k) cs[k + j * n] = r * v[k];
  }
  return 0;
}

// One shifted QR sweep (Givens) on the active block [n0, n1) of the
// row-major nr x nr Hessenberg matrix a.
void qr_sweep(double* a, int nr, int n0, int n1, double shift) {
  const int m1 = n0 + 1;
  double cv = a[n0 * nr + n0] - shift;
  double sv = a[m1 * nr + n0];
  double v = std::sqrt(cv * cv + sv * sv);
  double c = 1.0, s = 0.0;
  if (v != 0.0) { c = cv / v; s = sv / v; }
  for (int k = n0; k < nr; ++k) {
    const double x = a[n0 * nr + k], y = a[m1 * nr + k];
    a[n0 * nr + k] = c * x + s * y;
    a[m1 * nr + k] = c * y - s * x;
  }
  int m3 = n1 < n0 + 3 ? n1 : n0 + 3;
  for (int k = 0; k < m3; ++k) {
    const double x = a[k * nr + n0], y = a[k * nr + m1];
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
      const double x = a[j1 * nr + k], y = a[j2 * nr + k];
      a[j1 * nr + k] = c * x + s * y;
      a[j2 * nr + k] = c * y - s * x;
    }
    m3 = n1 < j + 4 ? n1 : j + 4;
    for (int k = 0; k < m3; ++k) {
      const double x = a[k * nr + j1], y = a[k * nr + j2];
      a[k * nr + j1] = c * x + s * y;
      a[k * nr + j2] = c * y - s * x;
    }
  }
}

int hessenberg_eig(double* a, int nr) {
  int n0 = 0, n1 = nr, its = 0;
  for (int ic = 0; ic < nr * kQrMaxIter; ++ic) {
    int k = n0;
    while (k + 1 < n1) {
      const double s = std::fabs(a[k * nr + k]) + std::fabs(a[(k + 1) * nr + k + 1]);
      if (std::fabs(a[(k + 1) * nr + k]) < kQrEps * s) break;
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
      const double a11 = a[m1 * nr + m1], a22 = a[m2 * nr + m2];
      const double tr = a11 + a22;
      double disc = (a11 - a22) * (a11 - a22);
      disc += 4.0 * a[m1 * nr + m2] * a[m2 * nr + m1];
      double shift;
      if (disc > 0.0) {
        const double sq = std::sqrt(disc);
        const double r1 = (tr + sq) * 0.5, r2 = (tr - sq) * 0.5;
        shift = std::fabs(a11 - r1) > std::fabs(a11 - r2) ? r2 : r1;
      } else {
        if (n1 == 2) return kErrRootFinding;
        shift = tr * 0.5;
      }
      ++its;
      qr_sweep(a, nr, n0, n1, shift);
      if (its > kQrMaxIter) return kErrRootFinding;
    }
  }
  return kErrRootFinding;
}

double horner(const double* c, int order, double x) {
  double p = c[order];
  for (int i = 1; i <= order; ++i) p = p * x + c[order - i];
  return p;
}

int bisect_refine(const double* cs, double* roots, int order, int n1) {
  const double* a = cs + order * n1;
  double x1i = 0.0, p1i = a[0];
  for (int m = 0; m < order; ++m) {
    const double x0i = x1i, p0i = p1i;
    x1i = roots[m];
    p1i = horner(a, order, x1i);
    if (p1i == 0.0) continue;
    if (p0i * p1i > 0.0) return kErrRootFinding;
    double x0, x1, p0, p1;
    if (x0i <= x1i) { x0 = x0i; x1 = x1i; p0 = p0i; p1 = p1i; }
    else { x0 = x1i; x1 = x0i; p0 = p1i; p1 = p0i; }
    if (p1 == 0.0) { roots[m] = x1; continue; }
    if (p0 == 0.0) { roots[m] = x0; continue; }
    double xi = x0 + (x0 - x1) / (p1 - p0) * p0;
    for (int it = 0; it < kBisectMaxIter; ++it) {
      if (std::fabs(x1 - x0) <= x1 * kRootAccuracy) break;
      double pi = horner(a, order, xi);
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

int poly_roots(double* roots, const double* cs, int nr, int n1) {
  if (nr == 1) {
    roots[0] = -cs[n1] / cs[1 + n1];
    return 0;
  }
  if (nr == 2) {
    const double a = cs[2 + 2 * n1], b = cs[1 + 2 * n1], c = cs[2 * n1];
    const double disc = b * b - 4.0 * a * c;
    if (disc < 0.0) return kErrRootFinding;
    const double sq = std::sqrt(disc);
    roots[0] = (-b - sq) / (2.0 * a);
    roots[1] = (-b + sq) / (2.0 * a);
    return 0;
  }
  double a[kMaxRoots * kMaxRoots];
  std::memset(a, 0, sizeof(a));
  const double lead = cs[nr + nr * n1];
  if (std::fabs(lead) < kThresholdZero) return kErrRootFinding;
  const double fac = -1.0 / lead;
  for (int i = 0; i < nr; ++i) a[nr - 1 - i] = cs[nr * n1 + i] * fac;
  for (int i = 0; i < nr - 1; ++i) a[(i + 1) * nr + i] = 1.0;
  if (hessenberg_eig(a, nr) == 0) {
    for (int i = 0; i < nr; ++i) roots[nr - 1 - i] = a[i * nr + i];
    return 0;
  }
  // QR gave up: seed from the quadratic and bisect orders 3..nr.
  const double qa = cs[2 + 2 * n1], qb = cs[1 + 2 * n1], qc = cs[2 * n1];
  const double disc = qb * qb - 4.0 * qa * qc;
  const double sq = disc >= 0.0 ? std::sqrt(disc) : 0.0;
  roots[0] = 0.5 * (-qb - sq) / qa;
  roots[1] = 0.5 * (-qb + sq) / qa;
  for (int i = 2; i < nr; ++i) roots[i] = 1.0;
  for (int k = 2; k < nr; ++k) {
    const int rc = bisect_refine(cs, roots, k + 1, n1);
    if (rc) return rc;
  }
  return 0;
}

}  // namespace

int rys_roots(int nroots, double t, double* roots, double* weights) {
  if (nroots < 1 || nroots > kMaxRoots) return -10;
  if (t < 0.0) return -11;
  double mu[2 * kMaxRoots + 1];
  boys_all(2 * nroots, t, mu);

  if (std::fabs(mu[0]) < kThresholdZero) {
    for (int i = 0; i < nroots; ++i) roots[i] = weights[i] = 0.0;
    return 0;
  }
  if (nroots == 1) {
    const double ratio = mu[1] / (mu[0] - mu[1]);
    roots[0] = ratio >= 0.0 ? ratio / (1.0 + ratio) : 0.0;
    weights[0] = mu[0];
    return 0;  // special method: not validated in the reference either
  }
  const int n1 = nroots + 1;
  double cs[(kMaxRoots + 1) * (kMaxRoots + 1)];
  std::memset(cs, 0, sizeof(cs));
  int rc = schmidt(cs, mu, n1);
  if (rc) return rc;
  double r[kMaxRoots] = {0};
  rc = poly_roots(r, cs, nroots, n1);
  if (rc) return rc;
  double w[kMaxRoots] = {0};
  for (int k = 0; k < nroots; ++k) {
    const double x = r[k];
    if (std::fabs(x - 1.0) < kThresholdZero) {
      r[k] = 0.0;
      w[k] = 0.0;
      continue;
    }
    double dum = 1.0 / mu[0];
    for (int j = 1; j < nroots; ++j) {
      const double p = horner(cs + j * n1, j, x);
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

}  // namespace oracle
