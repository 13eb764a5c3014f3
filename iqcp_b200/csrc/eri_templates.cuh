// ERI engine kernels for sm_100a: Rys-quadrature shell quartets digested
// directly into J/K (Fock build) or contracted with D x D weights (gradient).
//
// Numerics follow the reference's shell_eri (integrals/eri/mod.rs:458-854):
// per surviving primitive quartet (K_ij >= thr, K_ij*K_kl >= thr, eri/mod.rs:603,611)
// the pair data of gaussian_product_2e.rs:260-340, per root the coefficients
// of rys_coefficients.rs:94-180 (t^2 -> t^2/(1-t^2)), the 2D VRR of
// vrr_2d.rs:143-205 anchored on A and C, and horizontal transfer to B and D
// (htr_4d.rs).  Differences in arrangement, none in the mathematics:
//   * shells are reordered inside a pair so that la >= lb (the block is the
//     same up to index order);
//   * the angular factor 1/sqrt((2i-1)!!(2j-1)!!(2k-1)!!) of every component
//     (overlap.rs:343) is taken out of the quartet and applied to D before and
//     to J/K after the build (it factorises per basis function), the radial
//     factor (2a/pi)^{3/4}(4a)^{L/2} and the contraction coefficient are folded
//     into the primitive pair;
//   * the quadrature weight and prefactor are folded into the z-axis VRR seed.
// Digestion uses the 8-fold permutational symmetry with degeneracy factors, so
// every unique quartet (pair(ij) >= pair(kl)) is evaluated once.
#pragma once
#include <cuda_runtime.h>

#include "engine.cuh"
#include "rys_device.cuh"

namespace iqcp {

constexpr double kTwoPi52 = 34.986836655249725;  // 2 pi^{5/2}

__host__ __device__ constexpr double ang_factor(int l, int c) {
  // 1/sqrt((2i-1)!!(2j-1)!!(2k-1)!!): only d components xx, yy, zz differ from 1
  return (l == 2 && (c == 0 || c == 3 || c == 5)) ? 0.57735026918962576451 : 1.0;
}

// ---------------------------------------------------------------------------
// 1D integrals of one axis for one root: VRR table g[n][m] (n <= NB, m <= NK)
// then transfer to I[a][b][c][d] with a <= IA, b <= IB, c <= IC, d <= ID.
// For energies IA..ID = LA..LD; for gradients the table is extended by one on
// each index that gets differentiated.
template <typename R, int NB, int NK, int IA, int IB, int IC, int ID>
__device__ __forceinline__ void axis_table(R c00, R c0p, R b00, R b10, R b01, R ab, R cd, R g00,
                                           R* __restrict__ I) {
  R g[NB + 1][NK + 1];
  g[0][0] = g00;
  if (NB > 0) {
    g[1 < NB + 1 ? 1 : 0][0] = c00 * g00;
#pragma unroll
    for (int n = 1; n < NB; ++n) g[n + 1][0] = c00 * g[n][0] + R(n) * b10 * g[n - 1][0];
  }
#pragma unroll
  for (int m = 0; m < NK; ++m) {
    g[0][m + 1] = (m > 0) ? c0p * g[0][m] + R(m) * b01 * g[0][m > 0 ? m - 1 : 0] : c0p * g[0][m];
#pragma unroll
    for (int n = 1; n <= NB; ++n) {
      R v = c0p * g[n][m] + R(n) * b00 * g[n - 1][m];
      if (m > 0) v += R(m) * b01 * g[n][m > 0 ? m - 1 : 0];
      g[n][m + 1] = v;
    }
  }
  // bra transfer: h[a][b][m] = h[a+1][b-1][m] + AB h[a][b-1][m]
  R h[NB + 1][IB + 1][NK + 1];
#pragma unroll
  for (int a = 0; a <= NB; ++a)
#pragma unroll
    for (int m = 0; m <= NK; ++m) h[a][0][m] = g[a][m];
#pragma unroll
  for (int b = 1; b <= IB; ++b)
#pragma unroll
    for (int a = 0; a + b <= NB; ++a)
#pragma unroll
      for (int m = 0; m <= NK; ++m) h[a][b][m] = h[a + 1][b - 1][m] + ab * h[a][b - 1][m];
  // ket transfer for every needed (a, b)
#pragma unroll
  for (int a = 0; a <= IA; ++a)
#pragma unroll
    for (int b = 0; b <= IB; ++b) {
      if (a + b > NB) continue;
      R k[NK + 1][ID + 1];
#pragma unroll
      for (int c = 0; c <= NK; ++c) k[c][0] = h[a][b][c];
#pragma unroll
      for (int d = 1; d <= ID; ++d)
#pragma unroll
        for (int c = 0; c + d <= NK; ++c) k[c][d] = k[c + 1][d - 1] + cd * k[c][d - 1];
#pragma unroll
      for (int c = 0; c <= IC; ++c)
#pragma unroll
        for (int d = 0; d <= ID; ++d)
          if (c + d <= NK) I[((a * (IB + 1) + b) * (IC + 1) + c) * (ID + 1) + d] = k[c][d];
    }
}

// Row a = A of axis_table's output, I[A][b][c][d] for every b, c, d, with the
// same recurrences in the same order (so the entries are bitwise those of
// axis_table): the VRR up to row min(A + IB, NB), the bra transfer only for
// the rows A..A+IB it feeds, the ket transfer for row A.  Lets several lanes
// share one table with a fraction of the registers.
template <typename R, int NB, int NK, int IA, int IB, int IC, int ID, int A>
__device__ __forceinline__ void axis_slice(R c00, R c0p, R b00, R b10, R b01, R ab, R cd, R g00,
                                           R* __restrict__ I) {
  constexpr int NT = (A + IB < NB) ? A + IB : NB;  // highest VRR row needed
  R g[NT + 1][NK + 1];
  g[0][0] = g00;
  if (NT > 0) {
    g[1 < NT + 1 ? 1 : 0][0] = c00 * g00;
#pragma unroll
    for (int n = 1; n < NT; ++n) g[n + 1][0] = c00 * g[n][0] + R(n) * b10 * g[n - 1][0];
  }
#pragma unroll
  for (int m = 0; m < NK; ++m) {
    g[0][m + 1] = (m > 0) ? c0p * g[0][m] + R(m) * b01 * g[0][m > 0 ? m - 1 : 0] : c0p * g[0][m];
#pragma unroll
    for (int n = 1; n <= NT; ++n) {
      R v = c0p * g[n][m] + R(n) * b00 * g[n - 1][m];
      if (m > 0) v += R(m) * b01 * g[n][m > 0 ? m - 1 : 0];
      g[n][m + 1] = v;
    }
  }
  R h[NT + 1][IB + 1][NK + 1];
#pragma unroll
  for (int a = A; a <= NT; ++a)
#pragma unroll
    for (int m = 0; m <= NK; ++m) h[a][0][m] = g[a][m];
#pragma unroll
  for (int b = 1; b <= IB; ++b)
#pragma unroll
    for (int a = A; a + b <= NT; ++a)
#pragma unroll
      for (int m = 0; m <= NK; ++m) h[a][b][m] = h[a + 1][b - 1][m] + ab * h[a][b - 1][m];
#pragma unroll
  for (int b = 0; b <= IB; ++b) {
    if (A + b > NB) continue;
    R k[NK + 1][ID + 1];
#pragma unroll
    for (int c = 0; c <= NK; ++c) k[c][0] = h[A][b][c];
#pragma unroll
    for (int d = 1; d <= ID; ++d)
#pragma unroll
      for (int c = 0; c + d <= NK; ++c) k[c][d] = k[c + 1][d - 1] + cd * k[c][d - 1];
#pragma unroll
    for (int c = 0; c <= IC; ++c)
#pragma unroll
      for (int d = 0; d <= ID; ++d)
        if (c + d <= NK) I[((A * (IB + 1) + b) * (IC + 1) + c) * (ID + 1) + d] = k[c][d];
  }
}

template <int LA, int LB, int LC, int LD>
struct Cls {
  static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  static constexpr int NCOMP = NA * NB * NC * ND;
  static constexpr int NBRA = LA + LB, NKET = LC + LD;
  static constexpr int NR = (LA + LB + LC + LD) / 2 + 1;
  static constexpr int TSZ = (LA + 1) * (LB + 1) * (LC + 1) * (LD + 1);
  __host__ __device__ static constexpr int tidx(int a, int b, int c, int d) {
    return ((a * (LB + 1) + b) * (LC + 1) + c) * (LD + 1) + d;
  }
};

__device__ __forceinline__ PrimPair load_pp(const PrimPair* __restrict__ p) {
  PrimPair r;
  const double2* s = reinterpret_cast<const double2*>(p);
  const double2 v0 = __ldg(s), v1 = __ldg(s + 1), v2 = __ldg(s + 2), v3 = __ldg(s + 3);
  r.p = v0.x; r.P[0] = v0.y; r.P[1] = v1.x; r.P[2] = v1.y;
  r.K = v2.x; r.cK = v2.y; r.aa = v3.x; r.inv_p = v3.y;
  return r;
}

// Contracted (radially normalised) quartet (ab|cd) into acc[NCOMP].
// Primitive quartets are visited as items it = i * np_ket + j, starting at
// `first` with step `stride`, so that `stride` lanes can share one quartet.
// R is the quadrature type: double, or float for the FP32 share of the mixed
// form, where the roots, weights and recurrence coefficients are formed in
// FP64 and rounded once, and each primitive quartet's FP32 block is added to
// the FP64 accumulators.
template <typename R, int LA, int LB, int LC, int LD>
__device__ __forceinline__ void quartet(const ShellPair& bp, const ShellPair& kp, const PrimPair* __restrict__ pp,
                                        double thr, double* __restrict__ acc, int first = 0, int stride = 1,
                                        const double* rtab = nullptr) {
  using C = Cls<LA, LB, LC, LD>;
  constexpr bool F32 = sizeof(R) == 4;
#pragma unroll
  for (int i = 0; i < C::NCOMP; ++i) acc[i] = 0.0;
  const double AB[3] = {bp.A[0] - bp.B[0], bp.A[1] - bp.B[1], bp.A[2] - bp.B[2]};
  const double CD[3] = {kp.A[0] - kp.B[0], kp.A[1] - kp.B[1], kp.A[2] - kp.B[2]};
  // ket-major order: the bra primitive is the same on every lane of the warp
  // (one broadcast line per load); each lane's own ket primitive, scattered
  // across lanes, is loaded once per j
  const int nitems = bp.np * kp.np;
  int jl = -1;
  PrimPair k;
  for (int it = first; it < nitems; it += stride) {
    const int j = it / bp.np, i = it - j * bp.np;
    if (j != jl) {
      k = load_pp(pp + kp.pstart + j);
      jl = j;
    }
    const PrimPair b = load_pp(pp + bp.pstart + i);
    if (b.K * k.K < thr) continue;
    const double p = b.p, q = k.p, s = p + q;
    const double PQ[3] = {b.P[0] - k.P[0], b.P[1] - k.P[1], b.P[2] - k.P[2]};
    const double rs = rsqrt(s), inv_s = rs * rs;  // 1/(p+q), 1/sqrt(p+q): one rsqrt
    const double rho = p * q * inv_s;
    const double T = rho * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
    const double pref = kTwoPi52 * b.cK * k.cK * b.inv_p * k.inv_p * rs;
    double rt[C::NR], wt[C::NR];
    if (rtab) rys_rule_tab<C::NR>(T, rtab, rt, wt);
    else rys_rule<C::NR>(T, rt, wt);
    const double PA[3] = {b.P[0] - bp.A[0], b.P[1] - bp.A[1], b.P[2] - bp.A[2]};
    const double QC[3] = {k.P[0] - kp.A[0], k.P[1] - kp.A[1], k.P[2] - kp.A[2]};
    R part[F32 ? C::NCOMP : 1];
    if constexpr (F32) {
#pragma unroll
      for (int o = 0; o < C::NCOMP; ++o) part[o] = R(0);
    }
#pragma unroll
    for (int r = 0; r < C::NR; ++r) {
      const double t2 = rt[r];
      // rys_coefficients.rs:94-180 with u2 (p+q) + pq = pq / (1 - t^2):
      // tmp5 = t^2 / (2(p+q)), tmp4 q = (1 - t^2) / (2p), tmp4 p = (1 - t^2) / (2q)
      const double b00 = 0.5 * t2 * inv_s, h = 0.5 - 0.5 * t2;
      const double b10 = fma(h, b.inv_p, b00), b01 = fma(h, k.inv_p, b00);
      const double f2 = t2 * q * inv_s, f3 = t2 * p * inv_s;
      R Ix[C::TSZ], Iy[C::TSZ], Iz[C::TSZ];
      axis_table<R, C::NBRA, C::NKET, LA, LB, LC, LD>(R(PA[0] - f2 * PQ[0]), R(QC[0] + f3 * PQ[0]), R(b00), R(b10),
                                                      R(b01), R(AB[0]), R(CD[0]), R(1), Ix);
      axis_table<R, C::NBRA, C::NKET, LA, LB, LC, LD>(R(PA[1] - f2 * PQ[1]), R(QC[1] + f3 * PQ[1]), R(b00), R(b10),
                                                      R(b01), R(AB[1]), R(CD[1]), R(1), Iy);
      axis_table<R, C::NBRA, C::NKET, LA, LB, LC, LD>(R(PA[2] - f2 * PQ[2]), R(QC[2] + f3 * PQ[2]), R(b00), R(b10),
                                                      R(b01), R(AB[2]), R(CD[2]), R(wt[r] * pref), Iz);
#pragma unroll
      for (int a = 0; a < C::NA; ++a)
#pragma unroll
        for (int bb = 0; bb < C::NB; ++bb)
#pragma unroll
          for (int c = 0; c < C::NC; ++c)
#pragma unroll
            for (int d = 0; d < C::ND; ++d) {
              const int ix = C::tidx(cart_pow(LA, a, 0), cart_pow(LB, bb, 0), cart_pow(LC, c, 0),
                                     cart_pow(LD, d, 0));
              const int iy = C::tidx(cart_pow(LA, a, 1), cart_pow(LB, bb, 1), cart_pow(LC, c, 1),
                                     cart_pow(LD, d, 1));
              const int iz = C::tidx(cart_pow(LA, a, 2), cart_pow(LB, bb, 2), cart_pow(LC, c, 2),
                                     cart_pow(LD, d, 2));
              const int o = ((a * C::NB + bb) * C::NC + c) * C::ND + d;
              if constexpr (F32) part[o] = fmaf(Ix[ix] * Iy[iy], Iz[iz], part[o]);
              else acc[o] = fma(Ix[ix] * Iy[iy], Iz[iz], acc[o]);
            }
    }
    if constexpr (F32) {
#pragma unroll
      for (int o = 0; o < C::NCOMP; ++o) acc[o] += double(part[o]);
    }
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Quartet kernel with G lanes per contracted quartet (G = 1, 8 or 32): the 32/G
// groups of a warp take consecutive kets of the task; the G lanes of a group
// split the quartet's primitive quartets and combine their partial blocks with
// a segmented shuffle reduction; lane 0 of each group digests the block.
template <int G>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename R, int LA, int LB, int LC, int LD, int G, bool DO_K>
__global__ void __launch_bounds__(128) jk_kernel(JKArgs args) {
  using C = Cls<LA, LB, LC, LD>;
  constexpr int NG = 32 / G;
  extern __shared__ double rtab[];
  rys_stage_table<C::NR>(rtab);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (int warp = next_task(args.next_task, lane); warp < args.ntasks; warp = next_task(args.next_task, lane)) {
  const QuartetTask task = args.tasks[warp];
  const ShellPair bp = args.pairs[task.bra];
  if (task_inactive(args.mol_active, bp.mol)) continue;
  const int grp = lane / G, sub = lane - grp * G;
  // this task's molecule block (bra and ket pairs always share a molecule)
  const int n = args.mol_n[bp.mol];
  const long long mb = args.mol_base[bp.mol];
  const double* __restrict__ D = args.D + mb;
  // kets of this pass, compacted so that no group idles on the other pass's kets
  const unsigned sel = task_sel(args.mx, warp, task.nket);
  const int nsel = __popc(sel);
  if (sizeof(R) == 4 && lane == 0 && args.mx.fp32_count && nsel) atomicAdd(args.mx.fp32_count, (unsigned long long)nsel);
  for (int kbase = 0; kbase < nsel; kbase += NG) {
    const int kk = kbase + grp;
    const bool active = kk < nsel;
    double acc[C::NCOMP];
    double f = 0.0;
    ShellPair kp = bp;
    if (active) {
      const int kpos = task.ket0 + (args.mx.pass ? nth_set_bit(sel, kk) : kk);
      kp = args.pairs[__ldg(args.ket_list + kpos)];
      quartet<R, LA, LB, LC, LD>(bp, kp, args.pp, args.prim_thr, acc, sub, G, rtab);
      f = 1.0;
      if (bp.sa == bp.sb) f *= 0.5;
      if (kp.sa == kp.sb) f *= 0.5;
      if (task.diag && kpos == task.bra_pos) f *= 0.5;
    } else {
#pragma unroll
      for (int i = 0; i < C::NCOMP; ++i) acc[i] = 0.0;
    }
    if (G > 1) {
#pragma unroll
      for (int i = 0; i < C::NCOMP; ++i) acc[i] = group_sum<G>(acc[i]);
    }
    const bool digest = active && sub == 0;
    // every density of the call (nset > 1: response densities) is digested
    // with the same integrals
    for (int s = 0; s < args.nset; ++s) {
      const double* __restrict__ Dm = D + s * args.set_stride;
      double* Jm = args.J + mb + s * args.set_stride;
      double* Km = DO_K ? args.K + mb + s * args.set_stride : nullptr;
      // J~_ab += 2f sum_cd (ab|cd) D_cd  -- same bra on every group: warp reduction
#pragma unroll
      for (int a = 0; a < C::NA; ++a)
#pragma unroll
        for (int b = 0; b < C::NB; ++b) {
          double v = 0.0;
          if (digest) {
#pragma unroll
            for (int c = 0; c < C::NC; ++c)
#pragma unroll
              for (int d = 0; d < C::ND; ++d)
                v = fma(acc[((a * C::NB + b) * C::NC + c) * C::ND + d], __ldg(Dm + (kp.oa + c) * n + kp.ob + d), v);
            v *= 2.0 * f;
          }
          v = warp_sum(v);
          if (lane == 0) atomicAdd(Jm + (bp.oa + a) * n + bp.ob + b, v);
        }
      if (digest) {
      // J~_cd += 2f sum_ab (ab|cd) D_ab
      {
        double dab[C::NA * C::NB];
#pragma unroll
        for (int a = 0; a < C::NA; ++a)
#pragma unroll
          for (int b = 0; b < C::NB; ++b) dab[a * C::NB + b] = __ldg(Dm + (bp.oa + a) * n + bp.ob + b);
#pragma unroll
        for (int c = 0; c < C::NC; ++c)
#pragma unroll
          for (int d = 0; d < C::ND; ++d) {
            double v = 0.0;
#pragma unroll
            for (int ab = 0; ab < C::NA * C::NB; ++ab) v = fma(acc[(ab * C::NC + c) * C::ND + d], dab[ab], v);
            atomicAdd(Jm + (kp.oa + c) * n + kp.ob + d, 2.0 * f * v);
          }
      }
      if constexpr (DO_K) {
      // K~_ac += f sum_bd I D_bd ; K~_bc += f sum_ad I D_ad ; K~_ad += f sum_bc I D_bc ; K~_bd += f sum_ac I D_ac
#pragma unroll
      for (int a = 0; a < C::NA; ++a)
#pragma unroll
        for (int c = 0; c < C::NC; ++c) {
          double v = 0.0;
#pragma unroll
          for (int b = 0; b < C::NB; ++b)
#pragma unroll
            for (int d = 0; d < C::ND; ++d)
              v = fma(acc[((a * C::NB + b) * C::NC + c) * C::ND + d], __ldg(Dm + (bp.ob + b) * n + kp.ob + d), v);
          atomicAdd(Km + (bp.oa + a) * n + kp.oa + c, f * v);
        }
#pragma unroll
      for (int b = 0; b < C::NB; ++b)
#pragma unroll
        for (int c = 0; c < C::NC; ++c) {
          double v = 0.0;
#pragma unroll
          for (int a = 0; a < C::NA; ++a)
#pragma unroll
            for (int d = 0; d < C::ND; ++d)
              v = fma(acc[((a * C::NB + b) * C::NC + c) * C::ND + d], __ldg(Dm + (bp.oa + a) * n + kp.ob + d), v);
          atomicAdd(Km + (bp.ob + b) * n + kp.oa + c, f * v);
        }
#pragma unroll
      for (int a = 0; a < C::NA; ++a)
#pragma unroll
        for (int d = 0; d < C::ND; ++d) {
          double v = 0.0;
#pragma unroll
          for (int b = 0; b < C::NB; ++b)
#pragma unroll
            for (int c = 0; c < C::NC; ++c)
              v = fma(acc[((a * C::NB + b) * C::NC + c) * C::ND + d], __ldg(Dm + (bp.ob + b) * n + kp.oa + c), v);
          atomicAdd(Km + (bp.oa + a) * n + kp.ob + d, f * v);
        }
#pragma unroll
      for (int b = 0; b < C::NB; ++b)
#pragma unroll
        for (int d = 0; d < C::ND; ++d) {
          double v = 0.0;
#pragma unroll
          for (int a = 0; a < C::NA; ++a)
#pragma unroll
            for (int c = 0; c < C::NC; ++c)
              v = fma(acc[((a * C::NB + b) * C::NC + c) * C::ND + d], __ldg(Dm + (bp.oa + a) * n + kp.oa + c), v);
          atomicAdd(Km + (bp.ob + b) * n + kp.ob + d, f * v);
        }
      }
    }
    }
  }
  }  // task loop
}

// ---------------------------------------------------------------------------
// Schwarz bounds: Q = sqrt(max |(ab|ab)|) over the block with the angular
// factors applied (compute_schwarz_bounds, eri/mod.rs:1263-1290).
template <int LA, int LB>
__global__ void __launch_bounds__(128) schwarz_kernel(ShellPair* pairs, const PrimPair* pp,
                                                      const int* list, int n, double thr) {
  using C = Cls<LA, LB, LA, LB>;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int pid = list[t];
  const ShellPair bp = pairs[pid];
  double acc[C::NCOMP];
  quartet<double, LA, LB, LA, LB>(bp, bp, pp, thr, acc);
  double mx = 0.0;
#pragma unroll
  for (int a = 0; a < C::NA; ++a)
#pragma unroll
    for (int b = 0; b < C::NB; ++b)
#pragma unroll
      for (int c = 0; c < C::NC; ++c)
#pragma unroll
        for (int d = 0; d < C::ND; ++d) {
          const double v = acc[((a * C::NB + b) * C::NC + c) * C::ND + d] * ang_factor(LA, a) *
                           ang_factor(LB, b) * ang_factor(LA, c) * ang_factor(LB, d);
          mx = fmax(mx, fabs(v));
        }
  pairs[pid].Q = sqrt(mx);
}

// ---------------------------------------------------------------------------
// 8-fold compressed ERI store (eri_compressed layout, eri/mod.rs:946-1070).
__device__ __forceinline__ long long pair_index(long long i, long long j) {
  return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i;
}

template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(128) store_kernel(StoreArgs args) {
  using C = Cls<LA, LB, LC, LD>;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= args.ntasks) return;
  const QuartetTask task = args.tasks[warp];
  if (lane >= task.nket) return;
  const ShellPair bp = args.pairs[task.bra];
  const ShellPair kp = args.pairs[args.ket_list[task.ket0 + lane]];
  double acc[C::NCOMP];
  quartet<double, LA, LB, LC, LD>(bp, kp, args.pp, args.prim_thr, acc);
#pragma unroll
  for (int a = 0; a < C::NA; ++a)
#pragma unroll
    for (int b = 0; b < C::NB; ++b)
#pragma unroll
      for (int c = 0; c < C::NC; ++c)
#pragma unroll
        for (int d = 0; d < C::ND; ++d) {
          const double v = acc[((a * C::NB + b) * C::NC + c) * C::ND + d] * ang_factor(LA, a) *
                           ang_factor(LB, b) * ang_factor(LC, c) * ang_factor(LD, d);
          long long P = pair_index(bp.oa + a, bp.ob + b), Q = pair_index(kp.oa + c, kp.ob + d);
          if (P < Q) { const long long t = P; P = Q; Q = t; }
          args.out[P * (P + 1) / 2 + Q] = v;
        }
}

// ---------------------------------------------------------------------------
// Two-electron gradient (eri_gradient_fused, scf/gradient.rs:1430-1640).
// WSH: the D x D weights of each lane's quartet live in shared memory (one
// column of NCOMP per thread, read back one component at a time) instead of
// NCOMP registers, which leaves the registers to the extended tables of the
// mid-size classes (G = 1 only).
template <int LA, int LB, int LC, int LD>
__host__ __device__ constexpr int grad_wsh_doubles() {
  return 128 * ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD);
}
template <int LA, int LB, int LC, int LD, bool WSH>
__host__ __device__ constexpr bool grad_stages_rys() {
  return !(WSH && ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD) > 60);
}

// Resident blocks asked of the compiler: 4 for L <= 1 (for (ps|ss) the
// 128-register cap spills 76 bytes per thread, and is still faster than 3
// blocks without spill: 4.2 against 4.4 ms on the 40-atom step); 1 above.
template <typename R, int LA, int LB, int LC, int LD, int G, bool WSH = false>
__global__ void __launch_bounds__(128, (LA + LB + LC + LD <= 1) ? 4 : 1) grad_kernel(GradArgs args) {
  using C = Cls<LA, LB, LC, LD>;
  // tables extended by one on A and C; the B derivative takes I(a, b+1) from
  // the horizontal recurrence, I(a+1, b) + AB I(a, b), and the D derivative
  // follows from translational invariance
  constexpr int EA = LA + 1, EB = LB, EC = LC + 1, ED = LD;
  constexpr int ESZ = (EA + 1) * (EB + 1) * (EC + 1) * (ED + 1);
  auto eidx = [](int a, int b, int c, int d) { return ((a * (EB + 1) + b) * (EC + 1) + c) * (ED + 1) + d; };
  constexpr int NR = grad_nroots(LA + LB + LC + LD);
  constexpr int NG = 32 / G;
  constexpr bool F32 = sizeof(R) == 4;
  static_assert(!WSH || G == 1, "shared weights are per thread");
  // large shared weight arrays (more than 60 components) leave no room for a
  // second block beside the staged Rys table: those kernels read the table
  // through L1 instead
  constexpr bool STAGE = grad_stages_rys<LA, LB, LC, LD, WSH>();
  extern __shared__ double rtab[];
  if constexpr (STAGE) rys_stage_table<NR>(rtab);
  constexpr int TABD = STAGE ? rys_tab_doubles<NR>() : 0;
  // weights of this thread's quartet: Wsh[c * 128] (WSH), as R
  R* Wsh = reinterpret_cast<R*>(rtab + TABD) + threadIdx.x;
  const volatile R* Wv = Wsh;
  // per-block gradient accumulator: many quartets hit the same few atoms, so
  // global atomics would serialise; one flush per block at the end instead
  double* gacc = rtab + TABD + (WSH ? grad_wsh_doubles<LA, LB, LC, LD>() * sizeof(R) / 8 : 0);
  if (args.gsmem)
    for (int i = threadIdx.x; i < 3 * args.natoms; i += blockDim.x) gacc[i] = 0.0;
  __syncthreads();
  double* gout = args.gsmem ? gacc : args.grad;
  const int lane = threadIdx.x & 31;
  for (int warp = next_task(args.next_task, lane); warp < args.ntasks; warp = next_task(args.next_task, lane)) {
  const QuartetTask task = args.tasks[warp];
  const ShellPair bp = args.pairs[task.bra];
  const int grp = lane / G, sub = lane - grp * G;
  // this task's molecule block (bra and ket pairs always share a molecule)
  const int n = args.mol_n[bp.mol];
  const long long mb = args.mol_base[bp.mol];
  const double* __restrict__ D = args.D + mb;
  const double xs = args.xscale;
  const bool ij_same = bp.sa == bp.sb;
  const double AB[3] = {bp.A[0] - bp.B[0], bp.A[1] - bp.B[1], bp.A[2] - bp.B[2]};
  double gA[3] = {0, 0, 0}, gB[3] = {0, 0, 0};
  const unsigned sel = task_sel(args.mx, warp, task.nket);
  const int nsel = __popc(sel);
  if (F32 && lane == 0 && args.mx.fp32_count && nsel) atomicAdd(args.mx.fp32_count, (unsigned long long)nsel);
  for (int kbase = 0; kbase < nsel; kbase += NG) {
    const int kk = kbase + grp;
    bool active = kk < nsel;
    ShellPair kp = bp;
    int kpos = 0;
    if (active) {
      kpos = task.ket0 + (args.mx.pass ? nth_set_bit(sel, kk) : kk);
      kp = args.pairs[__ldg(args.ket_list + kpos)];
      // the reference skips when the Schwarz bound of its bra pair (the larger
      // composite index) is below threshold (gradient.rs:1457-1460)
      const double qref = bp.comp >= kp.comp ? bp.Q : kp.Q;
      if (qref < args.schwarz_thr) active = false;
    }
    double gC[3] = {0, 0, 0}, gBq[3] = {0, 0, 0}, gAq[3] = {0, 0, 0};
    if (active) {
      const bool kl_same = kp.sa == kp.sb;
      const bool bk_same = task.diag && kpos == task.bra_pos;
      R W[WSH ? 1 : C::NCOMP];
#pragma unroll
      for (int a = 0; a < C::NA; ++a)
#pragma unroll
        for (int b = 0; b < C::NB; ++b)
#pragma unroll
          for (int c = 0; c < C::NC; ++c)
#pragma unroll
            for (int d = 0; d < C::ND; ++d) {
              const int i = bp.oa + a, j = bp.ob + b, k = kp.oa + c, l = kp.ob + d;
              const double dij = __ldg(D + i * n + j), dkl = __ldg(D + k * n + l);
              const double dik = __ldg(D + i * n + k), djl = __ldg(D + j * n + l);
              const double dil = __ldg(D + i * n + l), djk = __ldg(D + j * n + k);
              // compute_symmetry_weight (gradient.rs:1570-1640) with D symmetric
              double t = 0.5 * dij * dkl - xs * dik * djl;
              if (!ij_same) t += 0.5 * dij * dkl - xs * djk * dil;
              if (!kl_same) t += 0.5 * dij * dkl - xs * dil * djk;
              if (!ij_same && !kl_same) t += 0.5 * dij * dkl - xs * djl * dik;
              if (!bk_same) {
                t += 0.5 * dkl * dij - xs * dik * djl;
                if (!kl_same) t += 0.5 * dkl * dij - xs * dil * djk;
                if (!ij_same) t += 0.5 * dkl * dij - xs * djk * dil;
                if (!ij_same && !kl_same) t += 0.5 * dkl * dij - xs * djl * dik;
              }
              // D is angular-scaled: t = w_ref * (ang_a ang_b ang_c ang_d); the
              // |w| < 1e-15 skip applies to the reference weight w_ref
              const double angp = ang_factor(LA, a) * ang_factor(LB, b) * ang_factor(LC, c) * ang_factor(LD, d);
              const R wt = R((fabs(t / angp) < 1e-15) ? 0.0 : t);
              const int o = ((a * C::NB + b) * C::NC + c) * C::ND + d;
              if constexpr (WSH) Wsh[o * 128] = wt;
              else W[o] = wt;
            }
      const double CD[3] = {kp.A[0] - kp.B[0], kp.A[1] - kp.B[1], kp.A[2] - kp.B[2]};
      const int nitems = bp.np * kp.np;
      int jl = -1;
      PrimPair k;
      for (int it = sub; it < nitems; it += G) {
        // ket-major order (see quartet)
        const int pj = it / bp.np, pi = it - pj * bp.np;
        if (pj != jl) {
          k = load_pp(args.pp + kp.pstart + pj);
          jl = pj;
        }
        const PrimPair b = load_pp(args.pp + bp.pstart + pi);
        if (b.K * k.K < args.prim_thr) continue;
        const double p = b.p, q = k.p, s = p + q;
        const double PQ[3] = {b.P[0] - k.P[0], b.P[1] - k.P[1], b.P[2] - k.P[2]};
        const double rs = rsqrt(s), inv_s = rs * rs;  // 1/(p+q), 1/sqrt(p+q): one rsqrt
        const double rho = p * q * inv_s;
        const double T = rho * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
        const double pref = kTwoPi52 * b.cK * k.cK * b.inv_p * k.inv_p * rs;
        double rt[NR], wt[NR];
        if constexpr (STAGE) rys_rule_tab<NR>(T, rtab, rt, wt);
        else rys_rule<NR>(T, rt, wt);
        const double PA[3] = {b.P[0] - bp.A[0], b.P[1] - bp.A[1], b.P[2] - bp.A[2]};
        const double QC[3] = {k.P[0] - kp.A[0], k.P[1] - kp.A[1], k.P[2] - kp.A[2]};
        const R a2 = R(2.0 * b.aa), b2 = R(2.0 * (b.p - b.aa)), c2 = R(2.0 * k.aa);
        // FP32 share: this primitive quartet's derivatives in R, then added to the FP64 sums
        R pA[3] = {0, 0, 0}, pB[3] = {0, 0, 0}, pC[3] = {0, 0, 0};
        // WSH (mid-size classes): one root's tables live at a time
#pragma unroll (WSH ? 1 : NR)
        for (int r = 0; r < NR; ++r) {
          const double t2 = rt[r];
          // rys_coefficients.rs:94-180 with u2 (p+q) + pq = pq / (1 - t^2):
          // tmp5 = t^2 / (2(p+q)), tmp4 q = (1 - t^2) / (2p), tmp4 p = (1 - t^2) / (2q)
          const double b00 = 0.5 * t2 * inv_s, h = 0.5 - 0.5 * t2;
          const double b10 = fma(h, b.inv_p, b00), b01 = fma(h, k.inv_p, b00);
          const double f2 = t2 * q * inv_s, f3 = t2 * p * inv_s;
          R E[3][ESZ];
#pragma unroll
          for (int ax = 0; ax < 3; ++ax)
            axis_table<R, LA + LB + 1, LC + LD + 1, EA, EB, EC, ED>(
                R(PA[ax] - f2 * PQ[ax]), R(QC[ax] + f3 * PQ[ax]), R(b00), R(b10), R(b01), R(AB[ax]), R(CD[ax]),
                R(ax == 2 ? wt[r] * pref : 1.0), E[ax]);
#pragma unroll
          for (int a = 0; a < C::NA; ++a)
#pragma unroll
            for (int bb = 0; bb < C::NB; ++bb)
#pragma unroll
              for (int c = 0; c < C::NC; ++c)
#pragma unroll
                for (int d = 0; d < C::ND; ++d) {
                  const int wo = ((a * C::NB + bb) * C::NC + c) * C::ND + d;
                  const R w = WSH ? Wv[wo * 128] : W[WSH ? 0 : wo];
                  R reg[3], dA[3], dB[3], dC[3];
#pragma unroll
                  for (int ax = 0; ax < 3; ++ax) {
                    const int ia = cart_pow(LA, a, ax), ib = cart_pow(LB, bb, ax), ic = cart_pow(LC, c, ax),
                              id = cart_pow(LD, d, ax);
                    reg[ax] = E[ax][eidx(ia, ib, ic, id)];
                    dA[ax] = a2 * E[ax][eidx(ia + 1, ib, ic, id)] -
                             (ia > 0 ? R(ia) * E[ax][eidx(ia > 0 ? ia - 1 : 0, ib, ic, id)] : R(0));
                    dB[ax] = b2 * (E[ax][eidx(ia + 1, ib, ic, id)] + R(AB[ax]) * E[ax][eidx(ia, ib, ic, id)]) -
                             (ib > 0 ? R(ib) * E[ax][eidx(ia, ib > 0 ? ib - 1 : 0, ic, id)] : R(0));
                    dC[ax] = c2 * E[ax][eidx(ia, ib, ic + 1, id)] -
                             (ic > 0 ? R(ic) * E[ax][eidx(ia, ib, ic > 0 ? ic - 1 : 0, id)] : R(0));
                  }
                  const R wyz = w * reg[1] * reg[2], wxz = w * reg[0] * reg[2], wxy = w * reg[0] * reg[1];
                  if constexpr (F32) {
                    pA[0] = fmaf(wyz, dA[0], pA[0]); pA[1] = fmaf(wxz, dA[1], pA[1]); pA[2] = fmaf(wxy, dA[2], pA[2]);
                    pB[0] = fmaf(wyz, dB[0], pB[0]); pB[1] = fmaf(wxz, dB[1], pB[1]); pB[2] = fmaf(wxy, dB[2], pB[2]);
                    pC[0] = fmaf(wyz, dC[0], pC[0]); pC[1] = fmaf(wxz, dC[1], pC[1]); pC[2] = fmaf(wxy, dC[2], pC[2]);
                  } else {
                    gAq[0] = fma(wyz, dA[0], gAq[0]); gAq[1] = fma(wxz, dA[1], gAq[1]); gAq[2] = fma(wxy, dA[2], gAq[2]);
                    gBq[0] = fma(wyz, dB[0], gBq[0]); gBq[1] = fma(wxz, dB[1], gBq[1]); gBq[2] = fma(wxy, dB[2], gBq[2]);
                    gC[0] = fma(wyz, dC[0], gC[0]); gC[1] = fma(wxz, dC[1], gC[1]); gC[2] = fma(wxy, dC[2], gC[2]);
                  }
                }
        }
        if constexpr (F32) {
#pragma unroll
          for (int x = 0; x < 3; ++x) {
            gAq[x] += double(pA[x]);
            gBq[x] += double(pB[x]);
            gC[x] += double(pC[x]);
          }
        }
      }
    }
    // ket atoms differ per group: segmented reduction, lane 0 of the group adds
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      const double c = group_sum<G>(gC[x]);
      const double dsum = group_sum<G>(gAq[x] + gBq[x] + gC[x]);
      if (active && sub == 0) {
        atomicAdd(gout + 3 * kp.atom_a + x, c);
        atomicAdd(gout + 3 * kp.atom_b + x, -dsum);  // translational invariance
      }
      gA[x] += gAq[x];
      gB[x] += gBq[x];
    }
  }
  // bra atoms are shared by the whole warp: one reduction per task
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    const double sa = warp_sum(gA[x]);
    const double sb = warp_sum(gB[x]);
    if (lane == 0) {
      atomicAdd(gout + 3 * bp.atom_a + x, sa);
      atomicAdd(gout + 3 * bp.atom_b + x, sb);
    }
  }
  }  // task loop
  if (args.gsmem) {
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * args.natoms; i += blockDim.x)
      if (gacc[i] != 0.0) atomicAdd(args.grad + i, gacc[i]);
  }
}

}  // namespace iqcp
