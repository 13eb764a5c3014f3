// CPU oracle (TEST INFRASTRUCTURE ONLY): stored-ERI and direct J/K builds and
// the fused two-electron gradient, restating:
//   * eri_compressed  <- integrals/eri/mod.rs:946-1070 (pair_index, eri_index,
//                        loop si>=sj x sk>=sl with the Schwarz skip :1028)
//   * build_fock      <- scf/mod.rs:825-881 (G = sum D[(mn|ls) - 1/2 (ml|ns)],
//                        mu>=nu, sigma<lambda doubled for J)
//   * build_jk        <- dft/ks_scf.rs:1306-1395 (J and K from stored ERIs)
//   * jk_direct       -- the same shell_eri numerics and screening, digested per
//                        unique quartet with 8-fold degeneracy weights (the
//                        reference stores ERIs instead; this is the direct form
//                        the GPU path computes, needed where storage cannot fit)
//   * eri_gradient    <- scf/gradient.rs:1430-1566 (unique quartets, Q_ij and
//                        Q_ij*Q_kl screens, |w|<1e-15 skip) with
//                        compute_symmetry_weight :1570-1640.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle_internal.h"

namespace oracle {

static inline size_t pair_idx(size_t i, size_t j) {
  if (i < j) std::swap(i, j);
  return i * (i + 1) / 2 + j;
}
static inline size_t eri_idx(size_t i, size_t j, size_t k, size_t l) {
  size_t p = pair_idx(i, j), q = pair_idx(k, l);
  if (p < q) std::swap(p, q);
  return p * (p + 1) / 2 + q;
}

void eri_compressed(const Basis& bs, double* eri, EriCounters* cnt) {
  const size_t n = bs.nbf;
  const size_t np = n * (n + 1) / 2;
  std::memset(eri, 0, sizeof(double) * (np * (np + 1) / 2));
  const std::vector<double> Q = schwarz_bounds(bs);
  const int ns = int(bs.shells.size());
  long long fails = 0, t0 = 0, pq = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : fails, t0, pq)
  for (int si = 0; si < ns; ++si) {
    std::vector<double> blk(1296);
    EriCounters c;
    for (int sj = 0; sj <= si; ++sj) {
      const double qij = Q[size_t(si) * ns + sj];
      for (int sk = 0; sk < ns; ++sk)
        for (int sl = 0; sl <= sk; ++sl) {
          if (qij * Q[size_t(sk) * ns + sl] < kSchwarzThreshold) continue;
          const Shell &A = bs.shells[si], &B = bs.shells[sj], &C = bs.shells[sk],
                      &D = bs.shells[sl];
          shell_eri(A, B, C, D, blk.data(), &c);
          const int ni = ncart(A.l), nj = ncart(B.l), nk = ncart(C.l), nl = ncart(D.l);
          for (int a = 0; a < ni; ++a)
            for (int b = 0; b < nj; ++b) {
              const size_t i = bs.offsets[si] + a, j = bs.offsets[sj] + b;
              if (i < j) continue;
              for (int c2 = 0; c2 < nk; ++c2)
                for (int d = 0; d < nl; ++d) {
                  const size_t k = bs.offsets[sk] + c2, l = bs.offsets[sl] + d;
                  if (k < l) continue;
                  // both bra/ket orders of a quartet write the same value
                  eri[eri_idx(i, j, k, l)] = blk[((a * nj + b) * nk + c2) * nl + d];
                }
            }
        }
    }
    fails += c.rys_failures;
    t0 += c.t_zero_fallbacks;
    pq += c.prim_quartets;
  }
  if (cnt) {
    cnt->rys_failures += fails;
    cnt->t_zero_fallbacks += t0;
    cnt->prim_quartets += pq;
  }
}

// D and F are row-major here (the reference's DMatrix is column-major, but D
// and G are symmetric, so the element order is the same).
void build_fock(int nbf, const double* H, const double* D, const double* eri, double* F) {
  const size_t n = nbf;
  std::memcpy(F, H, sizeof(double) * n * n);
#pragma omp parallel for schedule(dynamic)
  for (long mu = 0; mu < long(n); ++mu)
    for (size_t nu = 0; nu <= size_t(mu); ++nu) {
      double g = 0.0;
      for (size_t la = 0; la < n; ++la) {
        {
          const double dll = D[la * n + la];
          const double jint = eri[eri_idx(mu, nu, la, la)];
          const double kint = eri[eri_idx(mu, la, nu, la)];
          g += dll * (jint - 0.5 * kint);
        }
        for (size_t si = 0; si < la; ++si) {
          const double dls = D[la * n + si];
          const double jint = eri[eri_idx(mu, nu, la, si)];
          const double k1 = eri[eri_idx(mu, la, nu, si)];
          const double k2 = eri[eri_idx(mu, si, nu, la)];
          g += dls * (2.0 * jint - 0.5 * (k1 + k2));
        }
      }
      F[mu * n + nu] += g;
      if (size_t(mu) != nu) F[nu * n + mu] += g;
    }
}

// J_mn = sum_ls D_ls (mn|ls); K_mn = sum_ls D_ls (ml|ns)  (ks_scf.rs:1306-1395)
void build_jk_stored(int nbf, const double* D, const double* eri, double* J, double* K) {
  const size_t n = nbf;
#pragma omp parallel for schedule(dynamic)
  for (long mu = 0; mu < long(n); ++mu)
    for (size_t nu = 0; nu < n; ++nu) {
      double j = 0.0, k = 0.0;
      for (size_t la = 0; la < n; ++la)
        for (size_t si = 0; si < n; ++si) {
          const double d = D[la * n + si];
          j += d * eri[eri_idx(mu, nu, la, si)];
          k += d * eri[eri_idx(mu, la, nu, si)];
        }
      J[mu * n + nu] = j;
      if (K) K[mu * n + nu] = k;
    }
}

// Direct J/K over unique quartets (si>=sj, sk>=sl, pair(si,sj)>=pair(sk,sl)).
// `quartet_stride`/`quartet_phase` restrict the work to every stride-th bra
// shell pair so the CPU baseline can time a bounded, evenly spread sample.
void jk_direct(const Basis& bs, const double* D, double* J, double* K, int quartet_stride,
               int quartet_phase, EriCounters* cnt, long long* n_quartets) {
  const int ns = int(bs.shells.size());
  const size_t n = bs.nbf;
  const std::vector<double> Q = schwarz_bounds(bs);
  std::vector<std::pair<int, int>> pairs;
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j <= i; ++j) pairs.push_back({i, j});
  std::fill(J, J + n * n, 0.0);
  if (K) std::fill(K, K + n * n, 0.0);
  long long fails = 0, t0 = 0, pq = 0, nq = 0;
#pragma omp parallel reduction(+ : fails, t0, pq, nq)
  {
    std::vector<double> Jl(n * n, 0.0), Kl(n * n, 0.0), blk(1296);
    EriCounters c;
#pragma omp for schedule(dynamic)
    for (long P = 0; P < long(pairs.size()); ++P) {
      if (quartet_stride > 1 && (P % quartet_stride) != quartet_phase) continue;
      const int si = pairs[P].first, sj = pairs[P].second;
      const double qij = Q[size_t(si) * ns + sj];
      for (long Qp = 0; Qp <= P; ++Qp) {
        const int sk = pairs[Qp].first, sl = pairs[Qp].second;
        if (qij * Q[size_t(sk) * ns + sl] < kSchwarzThreshold) continue;
        const Shell &A = bs.shells[si], &B = bs.shells[sj], &C = bs.shells[sk],
                    &Dd = bs.shells[sl];
        shell_eri(A, B, C, Dd, blk.data(), &c);
        ++nq;
        double f = 1.0;
        if (si == sj) f *= 0.5;
        if (sk == sl) f *= 0.5;
        if (P == Qp) f *= 0.5;
        const int ni = ncart(A.l), nj = ncart(B.l), nk = ncart(C.l), nl = ncart(Dd.l);
        for (int a = 0; a < ni; ++a)
          for (int b = 0; b < nj; ++b) {
            const size_t i = bs.offsets[si] + a, j = bs.offsets[sj] + b;
            for (int c2 = 0; c2 < nk; ++c2)
              for (int d = 0; d < nl; ++d) {
                const size_t k = bs.offsets[sk] + c2, l = bs.offsets[sl] + d;
                const double v = f * blk[((a * nj + b) * nk + c2) * nl + d];
                Jl[i * n + j] += 2.0 * v * D[k * n + l];
                Jl[k * n + l] += 2.0 * v * D[i * n + j];
                Kl[i * n + k] += v * D[j * n + l];
                Kl[j * n + k] += v * D[i * n + l];
                Kl[i * n + l] += v * D[j * n + k];
                Kl[j * n + l] += v * D[i * n + k];
              }
          }
      }
    }
#pragma omp critical
    {
      for (size_t x = 0; x < n * n; ++x) {
        J[x] += Jl[x];
        if (K) K[x] += Kl[x];
      }
    }
    fails += c.rys_failures;
    t0 += c.t_zero_fallbacks;
    pq += c.prim_quartets;
  }
  // symmetrise: J = Jt + Jt^T, K = Kt + Kt^T
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j <= i; ++j) {
      const double js = J[i * n + j] + J[j * n + i];
      J[i * n + j] = J[j * n + i] = js;
      if (K) {
        const double ks = K[i * n + j] + K[j * n + i];
        K[i * n + j] = K[j * n + i] = ks;
      }
    }
  if (cnt) {
    cnt->rys_failures += fails;
    cnt->t_zero_fallbacks += t0;
    cnt->prim_quartets += pq;
  }
  if (n_quartets) *n_quartets = nq;
}

static inline double sym_weight(const double* D, size_t n, size_t i, size_t j, size_t k, size_t l,
                                bool ij_same, bool kl_same, bool bk_same, double c) {
  auto w = [&](size_t p, size_t q, size_t r, size_t s) {
    return 0.5 * D[p * n + q] * D[r * n + s] - c * D[p * n + r] * D[q * n + s];
  };
  double t = w(i, j, k, l);
  if (!ij_same) t += w(j, i, k, l);
  if (!kl_same) t += w(i, j, l, k);
  if (!ij_same && !kl_same) t += w(j, i, l, k);
  if (!bk_same) {
    t += w(k, l, i, j);
    if (!kl_same) t += w(l, k, i, j);
    if (!ij_same) t += w(k, l, j, i);
    if (!ij_same && !kl_same) t += w(l, k, j, i);
  }
  return t;
}

// grad is natoms x 3, accumulated (+=).  D is the factor-2 RHF density.
void eri_gradient(const Basis& bs, const double* D, double hf_frac, double* grad,
                  int quartet_stride, int quartet_phase, EriCounters* cnt) {
  const int ns = int(bs.shells.size());
  const size_t n = bs.nbf;
  const double xs = hf_frac * 0.25;
  const std::vector<double> Q = schwarz_bounds(bs);
  std::vector<std::pair<int, int>> pairs;
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j <= i; ++j) pairs.push_back({i, j});
  const int na = bs.natoms;
  long long fails = 0, t0 = 0, pq = 0;
  std::vector<double> gsum(3 * na, 0.0);
#pragma omp parallel reduction(+ : fails, t0, pq)
  {
    std::vector<double> gl(3 * na, 0.0), blk(13 * 1296);
    EriCounters c;
#pragma omp for schedule(dynamic)
    for (long P = 0; P < long(pairs.size()); ++P) {
      if (quartet_stride > 1 && (P % quartet_stride) != quartet_phase) continue;
      const int si = pairs[P].first, sj = pairs[P].second;
      const double qij = Q[size_t(si) * ns + sj];
      if (qij < kSchwarzThreshold) continue;
      for (long Qp = 0; Qp <= P; ++Qp) {
        const int sk = pairs[Qp].first, sl = pairs[Qp].second;
        if (qij * Q[size_t(sk) * ns + sl] < kSchwarzThreshold) continue;
        const Shell &A = bs.shells[si], &B = bs.shells[sj], &C = bs.shells[sk],
                    &Dd = bs.shells[sl];
        shell_eri_deriv(A, B, C, Dd, blk.data(), &c);
        const int ni = ncart(A.l), nj = ncart(B.l), nk = ncart(C.l), nl = ncart(Dd.l);
        const int ntot = ni * nj * nk * nl;
        const int atoms[4] = {A.atom, B.atom, C.atom, Dd.atom};
        for (int a = 0; a < ni; ++a)
          for (int b = 0; b < nj; ++b)
            for (int c2 = 0; c2 < nk; ++c2)
              for (int d = 0; d < nl; ++d) {
                const size_t i = bs.offsets[si] + a, j = bs.offsets[sj] + b;
                const size_t k = bs.offsets[sk] + c2, l = bs.offsets[sl] + d;
                const double w =
                    sym_weight(D, n, i, j, k, l, si == sj, sk == sl, P == Qp, xs);
                if (std::fabs(w) < 1e-15) continue;
                const int idx = ((a * nj + b) * nk + c2) * nl + d;
                for (int cen = 0; cen < 4; ++cen)
                  for (int dir = 0; dir < 3; ++dir)
                    gl[3 * atoms[cen] + dir] += w * blk[(1 + 3 * cen + dir) * ntot + idx];
              }
      }
    }
#pragma omp critical
    for (int x = 0; x < 3 * na; ++x) gsum[x] += gl[x];
    fails += c.rys_failures;
    t0 += c.t_zero_fallbacks;
    pq += c.prim_quartets;
  }
  for (int x = 0; x < 3 * na; ++x) grad[x] += gsum[x];
  if (cnt) {
    cnt->rys_failures += fails;
    cnt->t_zero_fallbacks += t0;
    cnt->prim_quartets += pq;
  }
}

}  // namespace oracle
