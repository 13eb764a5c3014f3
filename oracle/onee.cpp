// CPU oracle (TEST INFRASTRUCTURE ONLY): one-electron support integrals.
//
// The reference computes S, T, V and H = T + V (integrals/overlap.rs:647,
// kinetic.rs, nuclear.rs:68-305, hcore.rs:103) and their nuclear derivatives
// (scf/gradient.rs:188-700, integrals/deriv1.rs) over the same normalised
// Cartesian primitives as the ERIs.  They are not on the Fock-build hot path;
// the oracle restates what they compute (not how: McMurchie-Davidson Hermite
// expansions here) so that SCF energies and full RHF gradients can be checked
// against the reference's published values.
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle_internal.h"

namespace oracle {
namespace {

constexpr int kMaxL = 5;  // powers up to l+2 for kinetic / derivatives

// Hermite expansion coefficients E[i][j][t] for one Cartesian direction.
struct Herm1 {
  double E[kMaxL + 3][kMaxL + 3][2 * kMaxL + 7];
};

void hermite(double a, double b, double Ax, double Bx, int imax, int jmax, Herm1& h) {
  const double p = a + b, mu = a * b / p;
  const double X = Ax - Bx;
  const double XPA = -b / p * X, XPB = a / p * X;
  const double o2p = 0.5 / p;
  std::memset(&h, 0, sizeof(h));
  h.E[0][0][0] = std::exp(-mu * X * X);
  for (int i = 0; i <= imax; ++i)
    for (int j = 0; j <= jmax; ++j) {
      if (i == 0 && j == 0) continue;
      for (int t = 0; t <= i + j; ++t) {
        double v;
        if (i > 0) {
          v = XPA * h.E[i - 1][j][t];
          if (t > 0) v += o2p * h.E[i - 1][j][t - 1];
          if (t + 1 <= i + j - 1) v += double(t + 1) * h.E[i - 1][j][t + 1];
        } else {
          v = XPB * h.E[i][j - 1][t];
          if (t > 0) v += o2p * h.E[i][j - 1][t - 1];
          if (t + 1 <= i + j - 1) v += double(t + 1) * h.E[i][j - 1][t + 1];
        }
        h.E[i][j][t] = v;
      }
    }
}

// R^0_{tuv}(p, PC) for t+u+v <= N
void hermite_coulomb(double p, const double PC[3], int N, std::vector<double>& R) {
  const int S = N + 1;
  std::vector<double> Rn(size_t(S) * S * S * S, 0.0);
  auto at = [&](int n, int t, int u, int v) -> double& {
    return Rn[((size_t(n) * S + t) * S + u) * S + v];
  };
  const double T = p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
  double F[32];
  boys_all(N, T, F);
  double fac = 1.0;
  for (int n = 0; n <= N; ++n) {
    at(n, 0, 0, 0) = fac * F[n];
    fac *= -2.0 * p;
  }
  for (int n = N - 1; n >= 0; --n) {
    const int lim = N - n;
    for (int t = 0; t <= lim; ++t)
      for (int u = 0; u <= lim - t; ++u)
        for (int v = 0; v <= lim - t - u; ++v) {
          if (t + u + v == 0) continue;
          double val;
          if (t > 0) {
            val = PC[0] * at(n + 1, t - 1, u, v);
            if (t > 1) val += double(t - 1) * at(n + 1, t - 2, u, v);
          } else if (u > 0) {
            val = PC[1] * at(n + 1, t, u - 1, v);
            if (u > 1) val += double(u - 1) * at(n + 1, t, u - 2, v);
          } else {
            val = PC[2] * at(n + 1, t, u, v - 1);
            if (v > 1) val += double(v - 1) * at(n + 1, t, u, v - 2);
          }
          at(n, t, u, v) = val;
        }
  }
  R.assign(size_t(S) * S * S, 0.0);
  for (int t = 0; t <= N; ++t)
    for (int u = 0; u <= N - t; ++u)
      for (int v = 0; v <= N - t - u; ++v) R[(size_t(t) * S + u) * S + v] = at(0, t, u, v);
}

// Primitive integrals over raw (unnormalised) Cartesian Gaussians with powers
// pa, pb.  kind: 0 overlap, 1 kinetic, 2 nuclear attraction (all nuclei),
// 3 derivative of the nuclear attraction w.r.t. nucleus `cn`, direction `dir`
// (Hellmann-Feynman operator term).
double prim1e(int kind, double a, const double* A, const int pa[3], double b, const double* B,
              const int pb[3], const Basis& bs, int cn, int dir) {
  const double p = a + b;
  Herm1 h[3];
  for (int d = 0; d < 3; ++d) hermite(a, b, A[d], B[d], pa[d] + 1, pb[d] + 2, h[d]);
  const double sp = std::sqrt(M_PI / p);
  if (kind == 0) return h[0].E[pa[0]][pb[0]][0] * h[1].E[pa[1]][pb[1]][0] *
                        h[2].E[pa[2]][pb[2]][0] * sp * sp * sp;
  if (kind == 1) {
    double s1[3], t1[3];
    for (int d = 0; d < 3; ++d) {
      const int i = pa[d], j = pb[d];
      s1[d] = h[d].E[i][j][0] * sp;
      double v = -2.0 * b * double(2 * j + 1) * h[d].E[i][j][0] + 4.0 * b * b * h[d].E[i][j + 2][0];
      if (j >= 2) v += double(j * (j - 1)) * h[d].E[i][j - 2][0];
      t1[d] = -0.5 * v * sp;
    }
    return t1[0] * s1[1] * s1[2] + s1[0] * t1[1] * s1[2] + s1[0] * s1[1] * t1[2];
  }
  double P[3];
  for (int d = 0; d < 3; ++d) P[d] = (a * A[d] + b * B[d]) / p;
  const int N = pa[0] + pb[0] + pa[1] + pb[1] + pa[2] + pb[2] + (kind == 3 ? 1 : 0);
  const int S = N + 1;
  double total = 0.0;
  std::vector<double> R;
  const int c0 = kind == 3 ? cn : 0, c1 = kind == 3 ? cn + 1 : bs.natoms;
  for (int c = c0; c < c1; ++c) {
    const double PC[3] = {P[0] - bs.atom_xyz[3 * c], P[1] - bs.atom_xyz[3 * c + 1],
                          P[2] - bs.atom_xyz[3 * c + 2]};
    hermite_coulomb(p, PC, N, R);
    double s = 0.0;
    for (int t = 0; t <= pa[0] + pb[0]; ++t)
      for (int u = 0; u <= pa[1] + pb[1]; ++u)
        for (int v = 0; v <= pa[2] + pb[2]; ++v) {
          int tt = t, uu = u, vv = v;
          if (kind == 3) (dir == 0 ? tt : dir == 1 ? uu : vv) += 1;
          s += h[0].E[pa[0]][pb[0]][t] * h[1].E[pa[1]][pb[1]][u] * h[2].E[pa[2]][pb[2]][v] *
               R[(size_t(tt) * S + uu) * S + vv];
        }
    // V_C = -Z 2pi/p sum E R ; d/dC_x of R_{tuv}(P-C) = -R_{t+1,u,v}
    const double z = double(bs.atom_z[c]);
    total += (kind == 3 ? z : -z) * 2.0 * M_PI / p * s;
  }
  return total;
}

// Contracted matrix element between component ca of shell A and cb of shell B,
// optionally differentiating the bra function w.r.t. its centre in direction
// dbra (-1: no derivative).
double contracted(int kind, const Shell& SA, int ca, const Shell& SB, int cb, const Basis& bs,
                  int dbra, int cn, int dir) {
  int pa[3], pb[3];
  cart_powers(SA.l, ca, pa);
  cart_powers(SB.l, cb, pb);
  double sum = 0.0;
  for (size_t i = 0; i < SA.exps.size(); ++i) {
    const double na = SA.coefs[i] * cart_norm(SA.exps[i], pa);
    for (size_t j = 0; j < SB.exps.size(); ++j) {
      const double nb = SB.coefs[j] * cart_norm(SB.exps[j], pb);
      double v;
      if (dbra < 0) {
        v = prim1e(kind, SA.exps[i], SA.center, pa, SB.exps[j], SB.center, pb, bs, cn, dir);
      } else {
        int up[3] = {pa[0], pa[1], pa[2]};
        up[dbra] += 1;
        v = 2.0 * SA.exps[i] *
            prim1e(kind, SA.exps[i], SA.center, up, SB.exps[j], SB.center, pb, bs, cn, dir);
        if (pa[dbra] > 0) {
          int dn[3] = {pa[0], pa[1], pa[2]};
          dn[dbra] -= 1;
          v -= double(pa[dbra]) *
               prim1e(kind, SA.exps[i], SA.center, dn, SB.exps[j], SB.center, pb, bs, cn, dir);
        }
      }
      sum += na * nb * v;
    }
  }
  return sum;
}

}  // namespace

// out: nbf x nbf row-major
void one_electron(const Basis& bs, int kind, double* out) {
  const int ns = int(bs.shells.size());
  const size_t n = bs.nbf;
#pragma omp parallel for schedule(dynamic)
  for (int a = 0; a < ns; ++a)
    for (int b = 0; b < ns; ++b) {
      const Shell &SA = bs.shells[a], &SB = bs.shells[b];
      for (int ca = 0; ca < ncart(SA.l); ++ca)
        for (int cb = 0; cb < ncart(SB.l); ++cb)
          out[(bs.offsets[a] + ca) * n + bs.offsets[b] + cb] =
              contracted(kind, SA, ca, SB, cb, bs, -1, 0, 0);
    }
}

// One-electron part of the RHF gradient: sum D dH - sum W dS, plus the
// nuclear repulsion gradient.  grad (natoms x 3) is overwritten.
void one_electron_gradient(const Basis& bs, const double* D, const double* W, double* grad) {
  const int ns = int(bs.shells.size());
  const size_t n = bs.nbf;
  const int na = bs.natoms;
  std::vector<double> g(3 * na, 0.0);
  // nuclear repulsion
  for (int i = 0; i < na; ++i)
    for (int j = 0; j < na; ++j) {
      if (i == j) continue;
      double r[3], r2 = 0;
      for (int d = 0; d < 3; ++d) {
        r[d] = bs.atom_xyz[3 * i + d] - bs.atom_xyz[3 * j + d];
        r2 += r[d] * r[d];
      }
      const double rr = std::sqrt(r2);
      for (int d = 0; d < 3; ++d)
        g[3 * i + d] -= double(bs.atom_z[i] * bs.atom_z[j]) * r[d] / (rr * rr * rr);
    }
#pragma omp parallel
  {
    std::vector<double> gl(3 * na, 0.0);
#pragma omp for schedule(dynamic)
    for (int a = 0; a < ns; ++a) {
      const Shell& SA = bs.shells[a];
      for (int b = 0; b < ns; ++b) {
        const Shell& SB = bs.shells[b];
        for (int ca = 0; ca < ncart(SA.l); ++ca)
          for (int cb = 0; cb < ncart(SB.l); ++cb) {
            const size_t mu = bs.offsets[a] + ca, nu = bs.offsets[b] + cb;
            const double dmn = D[mu * n + nu], wmn = W[mu * n + nu];
            for (int dir = 0; dir < 3; ++dir) {
              // basis-function derivative of bra (ket term equal by symmetry)
              const double ds = contracted(0, SA, ca, SB, cb, bs, dir, 0, 0);
              const double dt = contracted(1, SA, ca, SB, cb, bs, dir, 0, 0);
              const double dv = contracted(2, SA, ca, SB, cb, bs, dir, 0, 0);
              gl[3 * SA.atom + dir] += 2.0 * (dmn * (dt + dv) - wmn * ds);
            }
          }
      }
    }
    // Hellmann-Feynman: derivative of the nuclear attraction operator
#pragma omp for schedule(dynamic)
    for (int c = 0; c < na; ++c)
      for (int a = 0; a < ns; ++a)
        for (int b = 0; b < ns; ++b) {
          const Shell &SA = bs.shells[a], &SB = bs.shells[b];
          for (int ca = 0; ca < ncart(SA.l); ++ca)
            for (int cb = 0; cb < ncart(SB.l); ++cb) {
              const size_t mu = bs.offsets[a] + ca, nu = bs.offsets[b] + cb;
              for (int dir = 0; dir < 3; ++dir)
                gl[3 * c + dir] += D[mu * n + nu] * contracted(3, SA, ca, SB, cb, bs, -1, c, dir);
            }
        }
#pragma omp critical
    for (int x = 0; x < 3 * na; ++x) g[x] += gl[x];
  }
  for (int x = 0; x < 3 * na; ++x) grad[x] = g[x];
}

double nuclear_repulsion(const Basis& bs) {
  double e = 0.0;
  for (int i = 0; i < bs.natoms; ++i)
    for (int j = 0; j < i; ++j) {
      double r2 = 0;
      for (int d = 0; d < 3; ++d) {
        const double x = bs.atom_xyz[3 * i + d] - bs.atom_xyz[3 * j + d];
        r2 += x * x;
      }
      e += double(bs.atom_z[i] * bs.atom_z[j]) / std::sqrt(r2);
    }
  return e;
}

}  // namespace oracle
