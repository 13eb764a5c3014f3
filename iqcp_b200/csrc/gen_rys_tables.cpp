// Offline generator for the device Rys quadrature tables (rys_tables.inc).
//
// For n = 1..kMaxN roots, the n-point Rys rule over x = t^2 on [0, 1) with
// weight  x^{-1/2} exp(-T x) / 2  (moments F_k(T), the Boys function) is
// computed in IEEE binary128 by
//   * moments F_0..F_2n(T) from the convergent Kummer series,
//   * the Chebyshev (modified-moment free) algorithm for the three-term
//     recurrence coefficients (Gautschi, "Orthogonal Polynomials", 2.1.7),
//   * eigenvalues of the Jacobi matrix by Sturm-sequence bisection,
//   * Christoffel numbers w_i = 1 / sum_j p_j(x_i)^2 (orthonormal p_j).
// Roots and weights are then fitted piecewise on T in [0, Tasym(n)) with
// Chebyshev series of fixed degree on unit-width intervals.  Beyond Tasym(n)
// the rule is the large-T limit: roots y_i / T and weights W_i / sqrt(T), with
// (y_i, W_i) the Gauss rule for the weight y^{-1/2} e^{-y} / 2 on [0, inf).
// Tasym(n) is the first integer T from which that limit agrees with the exact
// rule to the target accuracy everywhere in the sampled range.
//
// Build/run:  g++ -O2 -o /tmp/gen gen_rys_tables.cpp -lquadmath && /tmp/gen rys_tables.inc
#include <quadmath.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

typedef __float128 q;

static const int kMaxN = 7;
static const int kDeg = 11;          // Chebyshev degree per interval
static const double kWidth = 1.0;    // interval width in T

// F_k(T) = int_0^1 t^{2k} e^{-T t^2} dt, k = 0..m, by the series of F_m and
// downward recurrence (all terms positive, no cancellation).
static void boys_q(int m, q T, q* F) {
  const q e = expq(-T);
  q term = 1.0Q / (2 * m + 1), sum = term;
  for (int k = 1; k < 100000; ++k) {
    term *= 2 * T / (2 * m + 2 * k + 1);
    sum += term;
    if (term < sum * 1e-40Q) break;
  }
  F[m] = e * sum;
  for (int k = m; k >= 1; --k) F[k - 1] = (2 * T * F[k] + e) / (2 * k - 1);
}

// Gauss rule from moments mu_0..mu_2n via the Chebyshev algorithm.
static void gauss_from_moments(int n, const q* mu, q* x, q* w) {
  // sigma_{k,l} recursion (Gautschi 2004, Alg. 2.1)
  std::vector<q> a(n), b(n);
  const int L = 2 * n;
  std::vector<q> sm1(L + 1, 0), s0(L + 1), s1(L + 1);
  for (int l = 0; l <= L - 1; ++l) s0[l] = mu[l];
  a[0] = mu[1] / mu[0];
  b[0] = mu[0];
  for (int k = 1; k < n; ++k) {
    for (int l = k; l <= L - k - 1; ++l)
      s1[l] = s0[l + 1] - a[k - 1] * s0[l] - b[k - 1] * sm1[l];
    a[k] = s1[k + 1] / s1[k] - s0[k] / s0[k - 1];
    b[k] = s1[k] / s0[k - 1];
    sm1 = s0;
    s0 = s1;
  }
  // eigenvalues of the Jacobi matrix J (diag a, offdiag sqrt(b_k)), bisection
  auto count_below = [&](q lam) {
    int cnt = 0;
    q d = a[0] - lam;
    if (d < 0) ++cnt;
    for (int k = 1; k < n; ++k) {
      if (d == 0) d = 1e-60Q;
      d = a[k] - lam - b[k] / d;
      if (d < 0) ++cnt;
    }
    return cnt;
  };
  // Gershgorin bounds of the Jacobi matrix
  q lo = a[0], hi = a[0];
  for (int k = 0; k < n; ++k) {
    const q r = (k > 0 ? sqrtq(b[k]) : 0) + (k + 1 < n ? sqrtq(b[k + 1]) : 0);
    if (a[k] - r < lo) lo = a[k] - r;
    if (a[k] + r > hi) hi = a[k] + r;
  }
  lo -= 1e-3Q;
  hi += 1e-3Q;
  for (int i = 0; i < n; ++i) {
    q l = lo, h = hi;
    for (int it = 0; it < 240; ++it) {
      q m = 0.5Q * (l + h);
      if (count_below(m) > i) h = m; else l = m;
    }
    x[i] = 0.5Q * (l + h);
  }
  // orthonormal polynomials p_0 = 1/sqrt(b0); sqrt(b_{k+1}) p_{k+1} = (x-a_k) p_k - sqrt(b_k) p_{k-1}
  for (int i = 0; i < n; ++i) {
    q pm1 = 0, p0 = 1 / sqrtq(b[0]), s = p0 * p0;
    for (int k = 0; k < n - 1; ++k) {
      q p1 = ((x[i] - a[k]) * p0 - (k > 0 ? sqrtq(b[k]) * pm1 : 0)) / sqrtq(b[k + 1]);
      s += p1 * p1;
      pm1 = p0;
      p0 = p1;
    }
    w[i] = 1 / s;
  }
}

static void exact_rule(int n, q T, q* x, q* w) {
  q F[2 * kMaxN + 2];
  boys_q(2 * n, T, F);
  gauss_from_moments(n, F, x, w);
}

// Large-T rule: weight y^{-1/2} e^{-y}/2 on [0, inf), moments Gamma(k+1/2)/2
static void asym_base(int n, q* y, q* W) {
  q mu[2 * kMaxN + 2];
  q g = sqrtq(M_PIq);  // Gamma(1/2)
  for (int k = 0; k <= 2 * n; ++k) {
    mu[k] = g / 2;
    g *= (k + 0.5Q);
  }
  gauss_from_moments(n, mu, y, W);
}

static double cheb_eval(const double* c, double xx) {
  double b1 = 0, b2 = 0;
  for (int j = kDeg; j >= 1; --j) {
    double t = c[j] + 2 * xx * b1 - b2;
    b2 = b1;
    b1 = t;
  }
  return c[0] + xx * b1 - b2;
}

int main(int argc, char** argv) {
  if (argc < 2) { fprintf(stderr, "usage: gen out.inc\n"); return 1; }
  const double tol = 2e-15;
  int tasym[kMaxN + 1];
  std::vector<double> asy_y, asy_w;
  std::vector<double> coef;       // [n][interval][func 2n][deg+1]
  std::vector<int> offset(kMaxN + 2, 0);
  for (int n = 1; n <= kMaxN; ++n) {
    q y[kMaxN], W[kMaxN], x[kMaxN], w[kMaxN];
    asym_base(n, y, W);
    for (int i = 0; i < n; ++i) { asy_y.push_back((double)y[i]); asy_w.push_back((double)W[i]); }
    // smallest integer Ta with relative agreement for all sampled T >= Ta
    int Ta = 0;
    for (int T0 = 200; T0 >= 1; --T0) {
      bool ok = true;
      for (int s = 0; s < 8 && ok; ++s) {
        q T = T0 + s * 0.125Q;
        exact_rule(n, T, x, w);
        for (int i = 0; i < n; ++i) {
          q xa = y[i] / T, wa = W[i] / sqrtq(T);
          if (fabsq(xa - x[i]) > tol * x[i] || fabsq(wa - w[i]) > tol * w[i]) ok = false;
        }
      }
      if (!ok) { Ta = T0 + 1; break; }
    }
    tasym[n] = Ta;
    const int nint = int(std::ceil(Ta / kWidth));
    offset[n] = int(coef.size());
    for (int k = 0; k < nint; ++k) {
      const double t0 = k * kWidth;
      // Chebyshev interpolation at deg+1 Chebyshev points of the 1st kind
      const int np = kDeg + 1;
      std::vector<q> vals(size_t(np) * 2 * n);
      for (int j = 0; j < np; ++j) {
        q th = M_PIq * (j + 0.5Q) / np;
        q xx = cosq(th);
        q T = t0 + (xx + 1) * 0.5Q * kWidth;
        exact_rule(n, T, x, w);
        for (int i = 0; i < n; ++i) {
          vals[size_t(j) * 2 * n + i] = x[i];
          vals[size_t(j) * 2 * n + n + i] = w[i];
        }
      }
      for (int f = 0; f < 2 * n; ++f)
        for (int m = 0; m <= kDeg; ++m) {
          q s = 0;
          for (int j = 0; j < np; ++j)
            s += vals[size_t(j) * 2 * n + f] * cosq(m * M_PIq * (j + 0.5Q) / np);
          s *= (m == 0 ? 1.0Q : 2.0Q) / np;
          coef.push_back((double)s);
        }
    }
    // accuracy report on a dense grid
    double worst = 0;
    for (int k = 0; k < nint; ++k)
      for (int s = 0; s < 23; ++s) {
        const double T = k * kWidth + (s + 0.37) / 23.0 * kWidth;
        exact_rule(n, T, x, w);
        const double* c = &coef[offset[n] + size_t(k) * 2 * n * (kDeg + 1)];
        const double xx = 2 * (T - k * kWidth) / kWidth - 1;
        for (int f = 0; f < 2 * n; ++f) {
          const double v = cheb_eval(c + f * (kDeg + 1), xx);
          const double ex = (double)(f < n ? x[f] : w[f - n]);
          worst = std::fmax(worst, std::fabs(v - ex) / std::fabs(ex));
        }
      }
    fprintf(stderr, "n=%d Tasym=%d intervals=%d worst rel err %.3e\n", n, Ta, nint, worst);
  }
  offset[kMaxN + 1] = int(coef.size());
  FILE* f = fopen(argv[1], "w");
  fprintf(f, "// Generated by gen_rys_tables.cpp (binary128 Rys rules, Chebyshev fits). Do not edit.\n");
  fprintf(f, "#define RYS_TAB_MAXN %d\n#define RYS_TAB_DEG %d\n#define RYS_TAB_WIDTH %.1f\n", kMaxN, kDeg, kWidth);
  fprintf(f, "#ifndef RYS_TAB_QUAL\n#define RYS_TAB_QUAL static const\n#endif\n");
  fprintf(f, "#define RYS_TAB_NINT {0");
  for (int n = 1; n <= kMaxN; ++n) fprintf(f, ", %d", tasym[n]);
  fprintf(f, "}\n");
  fprintf(f, "RYS_TAB_QUAL int kRysTasym[%d] = {0", kMaxN + 1);
  for (int n = 1; n <= kMaxN; ++n) fprintf(f, ", %d", tasym[n]);
  fprintf(f, "};\nRYS_TAB_QUAL int kRysOffset[%d] = {0", kMaxN + 2);
  for (int n = 1; n <= kMaxN + 1; ++n) fprintf(f, ", %d", offset[n]);
  fprintf(f, "};\n// large-T rule per n (n entries each, n = 1..%d concatenated)\n", kMaxN);
  fprintf(f, "RYS_TAB_QUAL double kRysAsymRoot[%zu] = {\n", asy_y.size());
  for (double v : asy_y) fprintf(f, "  %.17e,\n", v);
  fprintf(f, "};\nRYS_TAB_QUAL double kRysAsymWeight[%zu] = {\n", asy_w.size());
  for (double v : asy_w) fprintf(f, "  %.17e,\n", v);
  fprintf(f, "};\n// [n][interval][root 0..n-1, weight 0..n-1][Chebyshev coefficient 0..DEG]\n");
  fprintf(f, "RYS_TAB_QUAL double kRysCheb[%zu] = {\n", coef.size());
  for (size_t i = 0; i < coef.size(); ++i) fprintf(f, "%.17e,%s", coef[i], (i % 4 == 3) ? "\n" : " ");
  fprintf(f, "};\n");
  fclose(f);
  return 0;
}
