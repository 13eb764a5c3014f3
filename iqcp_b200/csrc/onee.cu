// One-electron integrals on the device: overlap S, kinetic T and nuclear
// attraction V over the same normalised Cartesian primitives as the ERIs.
// They stand in for overlap_matrix (integrals/overlap.rs:647), the kinetic
// and nuclear builders behind hcore_matrix (integrals/hcore.rs:103,
// nuclear.rs:68-305): H = T + V.  Evaluated with McMurchie-Davidson Hermite
// expansions, one thread per (shell a, shell b) block, all component pairs.
// one_electron_grad_kernel contracts their nuclear derivatives with D and W.
#include <cuda_runtime.h>

#include "engine.cuh"
#include "rys_device.cuh"

namespace iqcp {

namespace {

constexpr int kE = 5;        // powers up to l + 2 (kinetic) with l <= 2
constexpr int kT = 2 * kE;   // Hermite index range

// E[i][j][t] for one direction, i <= ia_max < NI, j <= jb_max
template <int NI>
__device__ void hermite_e(double a, double b, double X, int imax, int jmax, double E[NI][kE][kT]) {
  const double p = a + b, mu = a * b / p;
  const double XPA = -b / p * X, XPB = a / p * X, o2p = 0.5 / p;
  for (int i = 0; i <= imax; ++i)
    for (int j = 0; j <= jmax; ++j)
      for (int t = 0; t < kT; ++t) E[i][j][t] = 0.0;
  E[0][0][0] = exp(-mu * X * X);
  for (int i = 0; i <= imax; ++i)
    for (int j = 0; j <= jmax; ++j) {
      if (i == 0 && j == 0) continue;
      for (int t = 0; t <= i + j; ++t) {
        double v;
        if (i > 0) {
          v = XPA * E[i - 1][j][t];
          if (t > 0) v += o2p * E[i - 1][j][t - 1];
          if (t + 1 <= i + j - 1) v += double(t + 1) * E[i - 1][j][t + 1];
        } else {
          v = XPB * E[i][j - 1][t];
          if (t > 0) v += o2p * E[i][j - 1][t - 1];
          if (t + 1 <= i + j - 1) v += double(t + 1) * E[i][j - 1][t + 1];
        }
        E[i][j][t] = v;
      }
    }
}

__device__ __forceinline__ double rad_norm_dev(double a, int l) {
  const double tap = 2.0 * a / 3.14159265358979323846;
  double v = sqrt(sqrt(tap * tap * tap));
  const double fa = 4.0 * a;
  if (l == 1) v *= sqrt(fa);
  else if (l == 2) v *= fa;
  return v;
}

__device__ __forceinline__ double ang_dev(int l, int c) {
  return (l == 2 && (c == 0 || c == 3 || c == 5)) ? 0.57735026918962576451 : 1.0;
}

}  // namespace

__global__ void __launch_bounds__(128) one_electron_kernel(OneEArgs a) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.n_shells * a.n_shells) return;
  const int sa = idx / a.n_shells, sb = idx % a.n_shells;
  const int la = a.l[sa], lb = a.l[sb];
  const int na = ncart(la), nb = ncart(lb);
  const double A[3] = {a.center[3 * sa], a.center[3 * sa + 1], a.center[3 * sa + 2]};
  const double B[3] = {a.center[3 * sb], a.center[3 * sb + 1], a.center[3 * sb + 2]};
  double s[36], t[36], v[36];
  for (int i = 0; i < 36; ++i) s[i] = t[i] = v[i] = 0.0;
  double E[3][3][kE][kT];
  for (int ip = 0; ip < a.nprim[sa]; ++ip) {
    const double ea = a.exps[a.pstart[sa] + ip];
    const double ca = a.coefs[a.pstart[sa] + ip] * rad_norm_dev(ea, la);
    for (int jp = 0; jp < a.nprim[sb]; ++jp) {
      const double eb = a.exps[a.pstart[sb] + jp];
      const double cb = a.coefs[a.pstart[sb] + jp] * rad_norm_dev(eb, lb);
      const double p = ea + eb;
      for (int d = 0; d < 3; ++d) hermite_e<3>(ea, eb, A[d] - B[d], la, lb + 2, E[d]);
      const double sp = sqrt(3.14159265358979323846 / p);
      const double cc = ca * cb;
      double P[3];
      for (int d = 0; d < 3; ++d) P[d] = (ea * A[d] + eb * B[d]) / p;
      // overlap and kinetic
      for (int ia = 0; ia < na; ++ia)
        for (int ib = 0; ib < nb; ++ib) {
          double s1[3], t1[3];
          for (int d = 0; d < 3; ++d) {
            const int i = cart_pow(la, ia, d), j = cart_pow(lb, ib, d);
            s1[d] = E[d][i][j][0] * sp;
            double k = -2.0 * eb * double(2 * j + 1) * E[d][i][j][0] + 4.0 * eb * eb * E[d][i][j + 2][0];
            if (j >= 2) k += double(j * (j - 1)) * E[d][i][j - 2][0];
            t1[d] = -0.5 * k * sp;
          }
          s[ia * nb + ib] += cc * s1[0] * s1[1] * s1[2];
          t[ia * nb + ib] += cc * (t1[0] * s1[1] * s1[2] + s1[0] * t1[1] * s1[2] + s1[0] * s1[1] * t1[2]);
        }
      if (!a.V) continue;
      // nuclear attraction: R_tuv via Boys F_n(p |PC|^2), n <= la + lb <= 4
      const int N = la + lb;
      for (int c = 0; c < a.n_atoms; ++c) {
        const double PC[3] = {P[0] - a.atom_xyz[3 * c], P[1] - a.atom_xyz[3 * c + 1],
                              P[2] - a.atom_xyz[3 * c + 2]};
        double F[8];
        boys_all_dev(N, p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]), F);
        // R^n_{tuv}, t+u+v <= N - n, stored for n = 0 only at the end
        double R[5][5][5][5];
        double fac = 1.0;
        for (int n = 0; n <= N; ++n) {
          R[n][0][0][0] = fac * F[n];
          fac *= -2.0 * p;
        }
        for (int n = N - 1; n >= 0; --n) {
          const int lim = N - n;
          for (int tt = 0; tt <= lim; ++tt)
            for (int uu = 0; uu <= lim - tt; ++uu)
              for (int vv = 0; vv <= lim - tt - uu; ++vv) {
                if (tt + uu + vv == 0) continue;
                double val;
                if (tt > 0) {
                  val = PC[0] * R[n + 1][tt - 1][uu][vv];
                  if (tt > 1) val += double(tt - 1) * R[n + 1][tt - 2][uu][vv];
                } else if (uu > 0) {
                  val = PC[1] * R[n + 1][tt][uu - 1][vv];
                  if (uu > 1) val += double(uu - 1) * R[n + 1][tt][uu - 2][vv];
                } else {
                  val = PC[2] * R[n + 1][tt][uu][vv - 1];
                  if (vv > 1) val += double(vv - 1) * R[n + 1][tt][uu][vv - 2];
                }
                R[n][tt][uu][vv] = val;
              }
        }
        const double pre = -double(a.z[c]) * 2.0 * 3.14159265358979323846 / p * cc;
        for (int ia = 0; ia < na; ++ia)
          for (int ib = 0; ib < nb; ++ib) {
            const int ix = cart_pow(la, ia, 0), jx = cart_pow(lb, ib, 0);
            const int iy = cart_pow(la, ia, 1), jy = cart_pow(lb, ib, 1);
            const int iz = cart_pow(la, ia, 2), jz = cart_pow(lb, ib, 2);
            double acc = 0.0;
            for (int tt = 0; tt <= ix + jx; ++tt)
              for (int uu = 0; uu <= iy + jy; ++uu)
                for (int vv = 0; vv <= iz + jz; ++vv)
                  acc += E[0][ix][jx][tt] * E[1][iy][jy][uu] * E[2][iz][jz][vv] * R[0][tt][uu][vv];
            v[ia * nb + ib] += pre * acc;
          }
      }
    }
  }
  const int oa = a.off[sa], ob = a.off[sb];
  for (int ia = 0; ia < na; ++ia)
    for (int ib = 0; ib < nb; ++ib) {
      const double g = ang_dev(la, ia) * ang_dev(lb, ib);
      const long long o = (long long)(oa + ia) * a.nbf + ob + ib;
      if (a.S) a.S[o] = g * s[ia * nb + ib];
      if (a.T) a.T[o] = g * t[ia * nb + ib];
      if (a.V) a.V[o] = g * v[ia * nb + ib];
    }
}

// ---------------------------------------------------------------------------
// Nuclear gradient of the one-electron energy plus the nuclear repulsion
// gradient (the non-ERI terms of rhf_gradient, scf/gradient.rs:900-990, from
// overlap_derivative_matrix / hcore_derivative_matrix, gradient.rs:188,355):
//   g_A += 2 sum_{mu on A, nu} [D_mn d(T+V)_mn/dA - W_mn dS_mn/dA]   (bra derivative;
//          the ket term is equal by symmetry of D and W)
//   g_C += sum_mn D_mn dV^C_mn/dC                                      (operator term)
//   g_A -= sum_{B != A} Z_A Z_B (A - B) / |A - B|^3
// The derivative of a Cartesian Gaussian w.r.t. its centre raises and lowers
// the power: d/dA_x x^i e^{-a x^2} = 2a x^{i+1} e^{..} - i x^{i-1} e^{..}.
// One thread per (shell a, shell b) block; per-block gradient in shared memory.
__global__ void __launch_bounds__(128) one_electron_grad_kernel(OneEArgs a) {
  extern __shared__ double gacc[];
  if (a.gsmem) {
    for (int i = threadIdx.x; i < 3 * a.n_atoms; i += blockDim.x) gacc[i] = 0.0;
    __syncthreads();
  }
  double* gout = a.gsmem ? gacc : a.grad;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  // nuclear repulsion: threads 0 .. n_atoms-1 of block 0 (n_atoms <= 128 per
  // thread pass; larger molecules loop)
  if (blockIdx.x == 0) {
    for (int i = threadIdx.x; i < a.n_atoms; i += blockDim.x) {
      double g[3] = {0, 0, 0};
      for (int j = 0; j < a.n_atoms; ++j) {
        if (j == i) continue;
        double r[3], r2 = 0.0;
        for (int d = 0; d < 3; ++d) {
          r[d] = a.atom_xyz[3 * i + d] - a.atom_xyz[3 * j + d];
          r2 += r[d] * r[d];
        }
        const double rr = sqrt(r2);
        const double f = double(a.z[i] * a.z[j]) / (rr * rr * rr);
        for (int d = 0; d < 3; ++d) g[d] -= f * r[d];
      }
      for (int d = 0; d < 3; ++d) atomicAdd(gout + 3 * i + d, g[d]);
    }
  }
  if (idx < a.n_shells * a.n_shells) {
    const int sa = idx / a.n_shells, sb = idx % a.n_shells;
    const int la = a.l[sa], lb = a.l[sb];
    const int na = ncart(la), nb = ncart(lb);
    const int oa = a.off[sa], ob = a.off[sb];
    const double A[3] = {a.center[3 * sa], a.center[3 * sa + 1], a.center[3 * sa + 2]};
    const double B[3] = {a.center[3 * sb], a.center[3 * sb + 1], a.center[3 * sb + 2]};
    // D and W of the block with the angular factors of both components
    double dm[36], wm[36];
    for (int ia = 0; ia < na; ++ia)
      for (int ib = 0; ib < nb; ++ib) {
        const double g = ang_dev(la, ia) * ang_dev(lb, ib);
        const long long o = (long long)(oa + ia) * a.nbf + ob + ib;
        dm[ia * nb + ib] = g * a.D[o];
        wm[ia * nb + ib] = g * a.W[o];
      }
    double gA[3] = {0, 0, 0};
    double E[3][4][kE][kT];  // bra powers up to la + 1
    const int N = la + lb + 1;
    for (int ip = 0; ip < a.nprim[sa]; ++ip) {
      const double ea = a.exps[a.pstart[sa] + ip];
      const double ca = a.coefs[a.pstart[sa] + ip] * rad_norm_dev(ea, la);
      for (int jp = 0; jp < a.nprim[sb]; ++jp) {
        const double eb = a.exps[a.pstart[sb] + jp];
        const double cb = a.coefs[a.pstart[sb] + jp] * rad_norm_dev(eb, lb);
        const double p = ea + eb;
        for (int d = 0; d < 3; ++d) hermite_e<4>(ea, eb, A[d] - B[d], la + 1, lb + 2, E[d]);
        const double sp = sqrt(3.14159265358979323846 / p);
        const double cc = ca * cb;
        // 1D overlap / kinetic factors s(i, j), t(i, j) per direction
        auto s1 = [&](int d, int i, int j) { return E[d][i][j][0] * sp; };
        auto t1 = [&](int d, int i, int j) {
          double k = -2.0 * eb * double(2 * j + 1) * E[d][i][j][0] + 4.0 * eb * eb * E[d][i][j + 2][0];
          if (j >= 2) k += double(j * (j - 1)) * E[d][i][j - 2][0];
          return -0.5 * k * sp;
        };
        for (int ia = 0; ia < na; ++ia)
          for (int ib = 0; ib < nb; ++ib) {
            const double dmn = dm[ia * nb + ib], wmn = wm[ia * nb + ib];
            int pi[3], pj[3];
            for (int d = 0; d < 3; ++d) {
              pi[d] = cart_pow(la, ia, d);
              pj[d] = cart_pow(lb, ib, d);
            }
            double s[3], t[3], ds[3], dt[3];
            for (int d = 0; d < 3; ++d) {
              s[d] = s1(d, pi[d], pj[d]);
              t[d] = t1(d, pi[d], pj[d]);
              ds[d] = 2.0 * ea * s1(d, pi[d] + 1, pj[d]) - (pi[d] > 0 ? pi[d] * s1(d, pi[d] - 1, pj[d]) : 0.0);
              dt[d] = 2.0 * ea * t1(d, pi[d] + 1, pj[d]) - (pi[d] > 0 ? pi[d] * t1(d, pi[d] - 1, pj[d]) : 0.0);
            }
            for (int d = 0; d < 3; ++d) {
              const int e1 = (d + 1) % 3, e2 = (d + 2) % 3;
              const double dS = ds[d] * s[e1] * s[e2];
              const double dT = dt[d] * s[e1] * s[e2] + ds[d] * (t[e1] * s[e2] + s[e1] * t[e2]);
              gA[d] += 2.0 * cc * (dmn * dT - wmn * dS);
            }
          }
        double P[3];
        for (int d = 0; d < 3; ++d) P[d] = (ea * A[d] + eb * B[d]) / p;
        for (int c = 0; c < a.n_atoms; ++c) {
          const double PC[3] = {P[0] - a.atom_xyz[3 * c], P[1] - a.atom_xyz[3 * c + 1],
                                P[2] - a.atom_xyz[3 * c + 2]};
          double F[8];
          boys_all_dev(N, p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]), F);
          // R^0_{tuv}, t+u+v <= N <= 5, by the downward recurrence in n with
          // two levels kept (Rn: level n + 1, R: level n)
          double R[6][6][6], Rn[6][6][6];
          double fac = 1.0;
          for (int n = 0; n < N; ++n) fac *= -2.0 * p;
          Rn[0][0][0] = fac * F[N];
          for (int n = N - 1; n >= 0; --n) {
            fac /= -2.0 * p;
            const int lim = N - n;
            for (int tt = 0; tt <= lim; ++tt)
              for (int uu = 0; uu <= lim - tt; ++uu)
                for (int vv = 0; vv <= lim - tt - uu; ++vv) {
                  double val;
                  if (tt + uu + vv == 0) {
                    val = fac * F[n];
                  } else if (tt > 0) {
                    val = PC[0] * Rn[tt - 1][uu][vv];
                    if (tt > 1) val += double(tt - 1) * Rn[tt - 2][uu][vv];
                  } else if (uu > 0) {
                    val = PC[1] * Rn[tt][uu - 1][vv];
                    if (uu > 1) val += double(uu - 1) * Rn[tt][uu - 2][vv];
                  } else {
                    val = PC[2] * Rn[tt][uu][vv - 1];
                    if (vv > 1) val += double(vv - 1) * Rn[tt][uu][vv - 2];
                  }
                  R[tt][uu][vv] = val;
                }
            for (int tt = 0; tt <= lim; ++tt)
              for (int uu = 0; uu <= lim - tt; ++uu)
                for (int vv = 0; vv <= lim - tt - uu; ++vv) Rn[tt][uu][vv] = R[tt][uu][vv];
          }
          const double zc = double(a.z[c]) * 2.0 * 3.14159265358979323846 / p * cc;
          double gC[3] = {0, 0, 0};
          for (int ia = 0; ia < na; ++ia)
            for (int ib = 0; ib < nb; ++ib) {
              const double dmn = dm[ia * nb + ib];
              int pi[3], pj[3];
              for (int d = 0; d < 3; ++d) {
                pi[d] = cart_pow(la, ia, d);
                pj[d] = cart_pow(lb, ib, d);
              }
              // Hermite sum with the bra power of direction dd shifted by sh,
              // and one more R index in direction hf (operator term; -1: none)
              auto hsum = [&](int dd, int sh, int hf) {
                int q[3] = {pi[0], pi[1], pi[2]};
                if (dd >= 0) q[dd] += sh;
                double acc = 0.0;
                for (int tt = 0; tt <= q[0] + pj[0]; ++tt)
                  for (int uu = 0; uu <= q[1] + pj[1]; ++uu)
                    for (int vv = 0; vv <= q[2] + pj[2]; ++vv)
                      acc += E[0][q[0]][pj[0]][tt] * E[1][q[1]][pj[1]][uu] * E[2][q[2]][pj[2]][vv] *
                             R[tt + (hf == 0)][uu + (hf == 1)][vv + (hf == 2)];
                return acc;
              };
              for (int d = 0; d < 3; ++d) {
                // basis-function derivative of V^c (bra): V = -Z 2pi/p sum E R
                double dv = 2.0 * ea * hsum(d, 1, -1);
                if (pi[d] > 0) dv -= double(pi[d]) * hsum(d, -1, -1);
                gA[d] += 2.0 * dmn * (-zc) * dv;
                // operator derivative: dV^c/dC_d = +Z 2pi/p sum E R_{+1 in d}
                gC[d] += dmn * zc * hsum(-1, 0, d);
              }
            }
          for (int d = 0; d < 3; ++d)
            if (gC[d] != 0.0) atomicAdd(gout + 3 * c + d, gC[d]);
        }
      }
    }
    const int at = a.atom[sa];
    for (int d = 0; d < 3; ++d) atomicAdd(gout + 3 * at + d, gA[d]);
  }
  if (a.gsmem) {
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * a.n_atoms; i += blockDim.x)
      if (gacc[i] != 0.0) atomicAdd(a.grad + i, gacc[i]);
  }
}

cudaError_t launch_one_electron_grad(const OneEArgs& a, cudaStream_t st) {
  const int n = a.n_shells * a.n_shells;
  const int blocks = (n + 127) / 128 > 0 ? (n + 127) / 128 : 1;
  const size_t smem = a.gsmem ? sizeof(double) * 3 * a.n_atoms : 0;
  if (smem > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(one_electron_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem);
    if (e != cudaSuccess) return e;
  }
  one_electron_grad_kernel<<<blocks, 128, smem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_one_electron(const OneEArgs& a, cudaStream_t st) {
  const int n = a.n_shells * a.n_shells;
  one_electron_kernel<<<(n + 127) / 128, 128, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace iqcp
