// CPU oracle (TEST INFRASTRUCTURE ONLY): contracted shell-quartet ERIs and
// their first derivatives, restating the reference's Rys path:
//   * cart_powers       <- integrals/cartesian.rs:113-136 (i desc, then j desc)
//   * cart_norm         <- integrals/overlap.rs:343-400 (per-component primitive
//                          normalisation; no contracted-shell renormalisation)
//   * pair data         <- integrals/eri/gaussian_product_2e.rs:260-340
//   * root coefficients <- integrals/eri/rys_coefficients.rs:94-180 (t^2 -> t^2/(1-t^2))
//   * 2D VRR            <- integrals/eri/vrr_2d.rs:143-205
//   * HTR               <- integrals/eri/htr_4d.rs:70-256 (recursive when j+l<=4)
//   * shell_eri         <- integrals/eri/mod.rs:458-854 (K screens :603/:611,
//                          T~0 fallback on a RysError :642-737)
//   * shell_eri_deriv   <- integrals/eri/mod.rs:2035-2548 (+1 on bra and ket,
//                          nroots=(L+2)/2+1, nabla identity on all 4 centres),
//                          T~0 path :3024-3190
//   * schwarz_bounds    <- integrals/eri/mod.rs:1263-1290
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle_internal.h"

namespace oracle {

void cart_powers(int l, int idx, int pw[3]) {
  int n = 0;
  for (int i = l; i >= 0; --i)
    for (int j = l - i; j >= 0; --j) {
      if (n == idx) { pw[0] = i; pw[1] = j; pw[2] = l - i - j; return; }
      ++n;
    }
}

static unsigned long long dfact(int n) {
  unsigned long long r = 1;
  for (int k = n; k > 1; k -= 2) r *= (unsigned long long)k;
  return r;
}

double cart_norm(double alpha, const int pw[3]) {
  const double tap = 2.0 * alpha / M_PI;
  const double base = std::sqrt(std::sqrt(tap * tap * tap));
  const int L = pw[0] + pw[1] + pw[2];
  if (L == 0) return base;
  const double fa = 4.0 * alpha;
  double num;
  switch (L) {
    case 1: num = std::sqrt(fa); break;
    case 2: num = fa; break;
    case 3: num = fa * std::sqrt(fa); break;
    case 4: num = fa * fa; break;
    default: num = std::pow(fa, double(L) / 2.0);
  }
  const double di = double(dfact(pw[0] > 0 ? 2 * pw[0] - 1 : 0));
  const double dj = double(dfact(pw[1] > 0 ? 2 * pw[1] - 1 : 0));
  const double dk = double(dfact(pw[2] > 0 ? 2 * pw[2] - 1 : 0));
  return base * num / std::sqrt(di * dj * dk);
}

Basis make_basis(int n_shells, const int* l, const int* nprim, const int* atom_of_shell,
                 const double* center, const double* exps, const double* coefs,
                 int natoms, const double* atom_xyz, const int* z) {
  Basis bs;
  int p = 0, off = 0;
  for (int s = 0; s < n_shells; ++s) {
    Shell sh;
    sh.l = l[s];
    sh.atom = atom_of_shell[s];
    for (int d = 0; d < 3; ++d) sh.center[d] = center[3 * s + d];
    sh.exps.assign(exps + p, exps + p + nprim[s]);
    sh.coefs.assign(coefs + p, coefs + p + nprim[s]);
    p += nprim[s];
    bs.offsets.push_back(off);
    off += ncart(sh.l);
    bs.shells.push_back(std::move(sh));
  }
  bs.nbf = off;
  bs.natoms = natoms;
  bs.atom_xyz.assign(atom_xyz, atom_xyz + 3 * natoms);
  bs.atom_z.assign(z, z + natoms);
  return bs;
}

namespace {

struct Pair2e {       // gaussian_product_2e.rs:40-115
  double p, q, pa[3], qc[3], ab[3], cd[3], pq[3], rho, t, pref;
};

Pair2e make_pair2e(double ai, const double* A, double aj, const double* B, double ak,
                   const double* C, double al, const double* D, const double ab[3],
                   const double cd[3], double kij, double kkl) {
  Pair2e g;
  g.p = ai + aj;
  double P[3], Q[3];
  for (int d = 0; d < 3; ++d) {
    P[d] = (ai * A[d] + aj * B[d]) / g.p;
    g.pa[d] = P[d] - A[d];
  }
  g.q = ak + al;
  for (int d = 0; d < 3; ++d) {
    Q[d] = (ak * C[d] + al * D[d]) / g.q;
    g.qc[d] = Q[d] - C[d];
  }
  for (int d = 0; d < 3; ++d) {
    g.pq[d] = P[d] - Q[d];
    g.ab[d] = ab[d];
    g.cd[d] = cd[d];
  }
  const double pq2 = g.pq[0] * g.pq[0] + g.pq[1] * g.pq[1] + g.pq[2] * g.pq[2];
  g.rho = g.p * g.q / (g.p + g.q);
  g.t = g.rho * pq2;
  g.pref = 2.0 * M_PI * M_PI * std::sqrt(M_PI) / (g.p * g.q * std::sqrt(g.p + g.q)) * kij * kkl;
  return g;
}

struct RootCoef { double b00, b10, b01, c00[3], c0p[3]; };

RootCoef root_coef(const Pair2e& g, double u) {   // rys_coefficients.rs:94-180
  RootCoef c;
  const double a1 = g.p * g.q;
  const double ut = u < 1.0 - 1e-15 ? u / (1.0 - u) : 1e15;
  const double u2 = g.rho * ut;
  const double tmp4 = 0.5 / (u2 * (g.p + g.q) + a1);
  const double tmp5 = u2 * tmp4;
  c.b00 = tmp5;
  c.b10 = tmp5 + tmp4 * g.q;
  c.b01 = tmp5 + tmp4 * g.p;
  const double t2 = 2.0 * tmp5 * g.q, t3 = 2.0 * tmp5 * g.p;
  for (int d = 0; d < 3; ++d) {
    c.c00[d] = g.pa[d] - t2 * g.pq[d];
    c.c0p[d] = g.qc[d] + t3 * g.pq[d];
  }
  return c;
}

RootCoef root_coef_t0(const Pair2e& g) {   // rys_coefficients.rs:183-215
  RootCoef c;
  const double tmp4 = 0.5 / (g.p * g.q);
  c.b00 = 0.0;
  c.b10 = tmp4 * g.q;
  c.b01 = tmp4 * g.p;
  for (int d = 0; d < 3; ++d) { c.c00[d] = g.pa[d]; c.c0p[d] = g.qc[d]; }
  return c;
}

// g[n*(nk+1)+m], n<=nb, m<=nk  (vrr_2d.rs:143-205)
void vrr(double* g, int nb, int nk, double c00, double c0p, double b00, double b10,
         double b01) {
  const int cols = nk + 1;
  for (int i = 0; i < (nb + 1) * cols; ++i) g[i] = 0.0;
  g[0] = 1.0;
  if (nb == 0 && nk == 0) return;
  if (nb > 0) {
    g[cols] = c00;
    for (int n = 1; n < nb; ++n)
      g[(n + 1) * cols] = c00 * g[n * cols] + double(n) * b10 * g[(n - 1) * cols];
  }
  for (int m = 0; m < nk; ++m) {
    if (m == 0) g[1] = c0p * g[0];
    else g[m + 1] = c0p * g[m] + double(m) * b01 * g[m - 1];
    for (int n = 1; n <= nb; ++n) {
      const double gnm = g[n * cols + m];
      const double gnm1 = m > 0 ? g[n * cols + m - 1] : 0.0;
      const double gn1m = g[(n - 1) * cols + m];
      g[n * cols + m + 1] = c0p * gnm + double(m) * b01 * gnm1 + double(n) * b00 * gn1m;
    }
  }
}

double htr_rec(const double* g, int nk, int i, int j, int k, int l, double ab, double cd) {
  if (j == 0 && l == 0) return g[i * (nk + 1) + k];
  if (l > 0)
    return htr_rec(g, nk, i, j, k + 1, l - 1, ab, cd) + cd * htr_rec(g, nk, i, j, k, l - 1, ab, cd);
  return htr_rec(g, nk, i + 1, j - 1, k, l, ab, cd) + ab * htr_rec(g, nk, i, j - 1, k, l, ab, cd);
}

double htr_iter(const double* g, int nk, int i, int j, int k, int l, double ab, double cd) {
  // ket transfer for each bra index nn = i..i+j, then bra transfer
  double prev[16], curr[16];
  if (l == 0) {
    for (int nn = i; nn <= i + j; ++nn) prev[nn - i] = g[nn * (nk + 1) + k];
  } else {
    double kp[64], kc[64];
    const int w = l + 1;
    for (int nn = i; nn <= i + j; ++nn)
      for (int kk = k; kk <= k + l; ++kk) kp[(nn - i) * w + (kk - k)] = g[nn * (nk + 1) + kk];
    for (int ll = 1; ll <= l; ++ll) {
      const int range = l - ll + 1;
      for (int ni = 0; ni <= j; ++ni)
        for (int ko = 0; ko < range; ++ko)
          kc[ni * w + ko] = kp[ni * w + ko + 1] + cd * kp[ni * w + ko];
      std::memcpy(kp, kc, sizeof(kp));
    }
    for (int ni = 0; ni <= j; ++ni) prev[ni] = kp[ni * w];
  }
  if (j == 0) return prev[0];
  for (int jj = 1; jj <= j; ++jj) {
    const int ns = j + 1 - jj;
    for (int o = 0; o < ns; ++o) curr[o] = prev[o + 1] + ab * prev[o];
    std::memcpy(prev, curr, sizeof(prev));
  }
  return prev[0];
}

inline double htr(const double* g, int nk, int i, int j, int k, int l, double ab, double cd) {
  if (j == 0 && l == 0) return g[i * (nk + 1) + k];
  if (j + l <= 4) return htr_rec(g, nk, i, j, k, l, ab, cd);
  return htr_iter(g, nk, i, j, k, l, ab, cd);
}

struct QuartetSetup {
  int n[4];
  std::vector<int> pw[4];                  // powers, 3 per component
  std::vector<double> norms[4];            // [prim * ncomp + comp]
  double ab[3], cd[3];
  std::vector<double> kij, kkl;
};

void setup(const Shell* s[4], QuartetSetup& q) {
  for (int c = 0; c < 4; ++c) {
    q.n[c] = ncart(s[c]->l);
    q.pw[c].resize(3 * q.n[c]);
    for (int i = 0; i < q.n[c]; ++i) cart_powers(s[c]->l, i, &q.pw[c][3 * i]);
    const int np = int(s[c]->exps.size());
    q.norms[c].resize(np * q.n[c]);
    for (int p = 0; p < np; ++p)
      for (int i = 0; i < q.n[c]; ++i)
        q.norms[c][p * q.n[c] + i] = cart_norm(s[c]->exps[p], &q.pw[c][3 * i]);
  }
  double ab2 = 0, cd2 = 0;
  for (int d = 0; d < 3; ++d) {
    q.ab[d] = s[0]->center[d] - s[1]->center[d];
    q.cd[d] = s[2]->center[d] - s[3]->center[d];
  }
  ab2 = q.ab[0] * q.ab[0] + q.ab[1] * q.ab[1] + q.ab[2] * q.ab[2];
  cd2 = q.cd[0] * q.cd[0] + q.cd[1] * q.cd[1] + q.cd[2] * q.cd[2];
  const int ni = int(s[0]->exps.size()), nj = int(s[1]->exps.size());
  const int nk = int(s[2]->exps.size()), nl = int(s[3]->exps.size());
  q.kij.resize(ni * nj);
  q.kkl.resize(nk * nl);
  for (int a = 0; a < ni; ++a)
    for (int b = 0; b < nj; ++b) {
      const double ea = s[0]->exps[a], eb = s[1]->exps[b];
      q.kij[a * nj + b] = std::exp(-(ea * eb / (ea + eb)) * ab2);
    }
  for (int a = 0; a < nk; ++a)
    for (int b = 0; b < nl; ++b) {
      const double ea = s[2]->exps[a], eb = s[3]->exps[b];
      q.kkl[a * nl + b] = std::exp(-(ea * eb / (ea + eb)) * cd2);
    }
}

}  // namespace

void shell_eri(const Shell& A, const Shell& B, const Shell& C, const Shell& D, double* out,
               EriCounters* cnt) {
  const Shell* s[4] = {&A, &B, &C, &D};
  QuartetSetup q;
  setup(s, q);
  const int n_i = q.n[0], n_j = q.n[1], n_k = q.n[2], n_l = q.n[3];
  const int ntot = n_i * n_j * n_k * n_l;
  std::fill(out, out + ntot, 0.0);
  const int L = A.l + B.l + C.l + D.l;
  const int nroots = L / 2 + 1;
  const int nb = A.l + B.l, nk = C.l + D.l;
  double gx[64], gy[64], gz[64];
  double roots[kMaxRoots], weights[kMaxRoots];
  const int npi = int(A.exps.size()), npj = int(B.exps.size());
  const int npk = int(C.exps.size()), npl = int(D.exps.size());

  for (int pi = 0; pi < npi; ++pi)
    for (int pj = 0; pj < npj; ++pj) {
      const double kij = q.kij[pi * npj + pj];
      if (kij < 1e-15) continue;
      for (int pk = 0; pk < npk; ++pk)
        for (int pl = 0; pl < npl; ++pl) {
          const double kkl = q.kkl[pk * npl + pl];
          if (kij * kkl < 1e-15) continue;
          const Pair2e g = make_pair2e(A.exps[pi], A.center, B.exps[pj], B.center, C.exps[pk],
                                       C.center, D.exps[pl], D.center, q.ab, q.cd, kij, kkl);
          const double cb = A.coefs[pi] * B.coefs[pj] * C.coefs[pk] * D.coefs[pl];
          int nr = nroots;
          const int rc = rys_roots(nroots, g.t, roots, weights);
          bool t0 = false;
          if (rc != 0) {
            if (cnt) cnt->rys_failures++;
            if (!(g.t < 1e-15)) continue;
            if (cnt) cnt->t_zero_fallbacks++;
            t0 = true;
            nr = 1;
          }
          if (cnt) cnt->prim_quartets++;
          for (int r = 0; r < nr; ++r) {
            const RootCoef c = t0 ? root_coef_t0(g) : root_coef(g, roots[r]);
            vrr(gx, nb, nk, c.c00[0], c.c0p[0], c.b00, c.b10, c.b01);
            vrr(gy, nb, nk, c.c00[1], c.c0p[1], c.b00, c.b10, c.b01);
            vrr(gz, nb, nk, c.c00[2], c.c0p[2], c.b00, c.b10, c.b01);
            const double wp = t0 ? g.pref * cb : g.pref * weights[r] * cb;
            for (int ii = 0; ii < n_i; ++ii) {
              const int* pa = &q.pw[0][3 * ii];
              const double na = q.norms[0][pi * n_i + ii];
              for (int jj = 0; jj < n_j; ++jj) {
                const int* pb = &q.pw[1][3 * jj];
                const double nbn = q.norms[1][pj * n_j + jj];
                for (int kk = 0; kk < n_k; ++kk) {
                  const int* pc = &q.pw[2][3 * kk];
                  const double nc = q.norms[2][pk * n_k + kk];
                  for (int ll = 0; ll < n_l; ++ll) {
                    const int* pd = &q.pw[3][3 * ll];
                    const double nd = q.norms[3][pl * n_l + ll];
                    const double ix = htr(gx, nk, pa[0], pb[0], pc[0], pd[0], g.ab[0], g.cd[0]);
                    const double iy = htr(gy, nk, pa[1], pb[1], pc[1], pd[1], g.ab[1], g.cd[1]);
                    const double iz = htr(gz, nk, pa[2], pb[2], pc[2], pd[2], g.ab[2], g.cd[2]);
                    out[((ii * n_j + jj) * n_k + kk) * n_l + ll] +=
                        wp * na * nbn * nc * nd * ix * iy * iz;
                  }
                }
              }
            }
          }
        }
    }
}

void shell_eri_deriv(const Shell& A, const Shell& B, const Shell& C, const Shell& D,
                     double* out13, EriCounters* cnt) {
  const Shell* s[4] = {&A, &B, &C, &D};
  QuartetSetup q;
  setup(s, q);
  const int n_i = q.n[0], n_j = q.n[1], n_k = q.n[2], n_l = q.n[3];
  const int ntot = n_i * n_j * n_k * n_l;
  std::fill(out13, out13 + 13 * ntot, 0.0);
  const int Lext = A.l + B.l + C.l + D.l + 2;
  const int nroots = Lext / 2 + 1;
  const int nb = A.l + B.l + 1, nk = C.l + D.l + 1;
  double gt[3][64];
  double roots[kMaxRoots], weights[kMaxRoots];
  const int npi = int(A.exps.size()), npj = int(B.exps.size());
  const int npk = int(C.exps.size()), npl = int(D.exps.size());

  for (int pi = 0; pi < npi; ++pi)
    for (int pj = 0; pj < npj; ++pj) {
      const double kij = q.kij[pi * npj + pj];
      if (kij < 1e-15) continue;
      for (int pk = 0; pk < npk; ++pk)
        for (int pl = 0; pl < npl; ++pl) {
          const double kkl = q.kkl[pk * npl + pl];
          if (kij * kkl < 1e-15) continue;
          const Pair2e g = make_pair2e(A.exps[pi], A.center, B.exps[pj], B.center, C.exps[pk],
                                       C.center, D.exps[pl], D.center, q.ab, q.cd, kij, kkl);
          const double cb = A.coefs[pi] * B.coefs[pj] * C.coefs[pk] * D.coefs[pl];
          const double ex[4] = {A.exps[pi], B.exps[pj], C.exps[pk], D.exps[pl]};
          int nr = nroots;
          const int rc = rys_roots(nroots, g.t, roots, weights);
          bool t0 = false;
          if (rc != 0) {
            if (cnt) cnt->rys_failures++;
            if (!(g.t < 1e-15)) continue;
            if (cnt) cnt->t_zero_fallbacks++;
            t0 = true;
            nr = 1;
          }
          if (cnt) cnt->prim_quartets++;
          for (int r = 0; r < nr; ++r) {
            const RootCoef c = t0 ? root_coef_t0(g) : root_coef(g, roots[r]);
            for (int d = 0; d < 3; ++d) vrr(gt[d], nb, nk, c.c00[d], c.c0p[d], c.b00, c.b10, c.b01);
            const double wp = t0 ? g.pref * cb : g.pref * weights[r] * cb;
            for (int ii = 0; ii < n_i; ++ii)
              for (int jj = 0; jj < n_j; ++jj)
                for (int kk = 0; kk < n_k; ++kk)
                  for (int ll = 0; ll < n_l; ++ll) {
                    const int* pw4[4] = {&q.pw[0][3 * ii], &q.pw[1][3 * jj], &q.pw[2][3 * kk],
                                         &q.pw[3][3 * ll]};
                    const double an = wp * q.norms[0][pi * n_i + ii] * q.norms[1][pj * n_j + jj] *
                                      q.norms[2][pk * n_k + kk] * q.norms[3][pl * n_l + ll];
                    double reg[3];
                    for (int d = 0; d < 3; ++d)
                      reg[d] = htr(gt[d], nk, pw4[0][d], pw4[1][d], pw4[2][d], pw4[3][d], g.ab[d],
                                   g.cd[d]);
                    const int idx = ((ii * n_j + jj) * n_k + kk) * n_l + ll;
                    out13[idx] += an * reg[0] * reg[1] * reg[2];
                    for (int cen = 0; cen < 4; ++cen) {
                      const double e2 = 2.0 * ex[cen];
                      for (int d = 0; d < 3; ++d) {
                        int up[4] = {pw4[0][d], pw4[1][d], pw4[2][d], pw4[3][d]};
                        up[cen] += 1;
                        const double plus =
                            htr(gt[d], nk, up[0], up[1], up[2], up[3], g.ab[d], g.cd[d]);
                        double minus = 0.0;
                        if (pw4[cen][d] > 0) {
                          int dn[4] = {pw4[0][d], pw4[1][d], pw4[2][d], pw4[3][d]};
                          dn[cen] -= 1;
                          minus = htr(gt[d], nk, dn[0], dn[1], dn[2], dn[3], g.ab[d], g.cd[d]);
                        }
                        const double d1 = e2 * plus - double(pw4[cen][d]) * minus;
                        double val;
                        if (d == 0) val = d1 * reg[1] * reg[2];
                        else if (d == 1) val = reg[0] * d1 * reg[2];
                        else val = reg[0] * reg[1] * d1;
                        out13[(1 + 3 * cen + d) * ntot + idx] += an * val;
                      }
                    }
                  }
          }
        }
    }
}

std::vector<double> schwarz_bounds(const Basis& bs) {
  const int ns = int(bs.shells.size());
  std::vector<double> q(size_t(ns) * ns, 0.0);
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < ns; ++i) {
    std::vector<double> blk(1296);
    for (int j = 0; j <= i; ++j) {
      const Shell &a = bs.shells[i], &b = bs.shells[j];
      const int n = ncart(a.l) * ncart(b.l) * ncart(a.l) * ncart(b.l);
      shell_eri(a, b, a, b, blk.data(), nullptr);
      double mx = 0.0;
      for (int k = 0; k < n; ++k) mx = std::max(mx, std::fabs(blk[k]));
      q[size_t(i) * ns + j] = q[size_t(j) * ns + i] = std::sqrt(mx);
    }
  }
  return q;
}

}  // namespace oracle
