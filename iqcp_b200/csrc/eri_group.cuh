// Grouped gradient quartet kernel: G lanes (8 or 32) per contracted quartet.
//
// Same numerics as grad_kernel (eri_templates.cuh): per surviving primitive
// quartet and Rys root the extended 1D tables of the three axes, the nine
// A/B/C derivatives per component, D by translational invariance.  Two
// differences in arrangement keep it out of local memory:
//   * the D x D weights of the group's quartet (compute_symmetry_weight,
//     scf/gradient.rs:1570-1640) live in shared memory, formed by the G lanes
//     together and read by all of them (one address per group), instead of
//     NCOMP registers per lane;
//   * the G lanes split (primitive quartet, root) items rather than primitive
//     quartets, so one lane holds one root's tables at a time and short
//     contractions still fill the group.
#pragma once
#include "eri_team.cuh"

namespace iqcp {

template <typename R, int LA, int LB, int LC, int LD, int G>
struct GroupGrad {
  using C = Cls<LA, LB, LC, LD>;
  static constexpr int NG = 32 / G;                                   // groups per warp
  static constexpr int NR = grad_nroots(LA + LB + LC + LD);
  static constexpr int WDOUBLES = (4 * NG * C::NCOMP * (int)sizeof(R) + 15) / 16 * 2;  // 4 warps per block
};

// Weight of component comp (a, b, c, d) of quartet (bp, kp): sum over the
// distinct permutations of 1/2 D_ij D_kl - xs D_ik D_jl on the angular-scaled
// density, zero where the reference weight is below 1e-15 (gradient.rs:1585-1640).
template <int LA, int LB, int LC, int LD>
__device__ __forceinline__ double grad_weight(const double* __restrict__ D, int n, const ShellPair& bp,
                                              const ShellPair& kp, int comp, bool ij_same, bool kl_same,
                                              bool bk_same, double xs) {
  using C = Cls<LA, LB, LC, LD>;
  const int d = comp % C::ND, c = (comp / C::ND) % C::NC, b = (comp / (C::ND * C::NC)) % C::NB,
            a = comp / (C::ND * C::NC * C::NB);
  const int i = bp.oa + a, j = bp.ob + b, k = kp.oa + c, l = kp.ob + d;
  const double dij = __ldg(D + i * n + j), dkl = __ldg(D + k * n + l);
  const double dik = __ldg(D + i * n + k), djl = __ldg(D + j * n + l);
  const double dil = __ldg(D + i * n + l), djk = __ldg(D + j * n + k);
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
  const double angp = ang_factor(LA, a) * ang_factor(LB, b) * ang_factor(LC, c) * ang_factor(LD, d);
  return (fabs(t / angp) < 1e-15) ? 0.0 : t;
}

template <typename R, int LA, int LB, int LC, int LD, int G>
__global__ void __launch_bounds__(128) grad_group_kernel(GradArgs args) {
  using C = Cls<LA, LB, LC, LD>;
  using GG = GroupGrad<R, LA, LB, LC, LD, G>;
  constexpr int EA = LA + 1, EB = LB, EC = LC + 1, ED = LD;
  constexpr int ESZ = (EA + 1) * (EB + 1) * (EC + 1) * (ED + 1);
  constexpr int NR = GG::NR, NG = GG::NG;
  auto eidx = [](int a, int b, int c, int d) { return ((a * (EB + 1) + b) * (EC + 1) + c) * (ED + 1) + d; };
  extern __shared__ __align__(16) double smem[];
  double* rtab = smem;
  rys_stage_table<NR>(rtab);
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // weights of the warp's groups, interleaved: W[comp * NG + group]; read
  // through a volatile view so that they stay in shared memory instead of
  // being hoisted into registers across the item loop
  R* W = reinterpret_cast<R*>(smem + rys_tab_doubles<NR>()) + wib * NG * C::NCOMP;
  const volatile R* Wv = W;
  double* gacc = smem + rys_tab_doubles<NR>() + GG::WDOUBLES;
  if (args.gsmem)
    for (int i = threadIdx.x; i < 3 * args.natoms; i += blockDim.x) gacc[i] = 0.0;
  __syncthreads();
  double* gout = args.gsmem ? gacc : args.grad;
  const int grp = lane / G, sub = lane - grp * G;
  for (int warp = next_task(args.next_task, lane); warp < args.ntasks; warp = next_task(args.next_task, lane)) {
  const QuartetTask task = args.tasks[warp];
  const ShellPair bp = args.pairs[task.bra];
  const int n = args.mol_n[bp.mol];
  const long long mb = args.mol_base[bp.mol];
  const double* __restrict__ D = args.D + mb;
  const double xs = args.xscale;
  const bool ij_same = bp.sa == bp.sb;
  const double AB[3] = {bp.A[0] - bp.B[0], bp.A[1] - bp.B[1], bp.A[2] - bp.B[2]};
  double gA[3] = {0, 0, 0}, gB[3] = {0, 0, 0};
  const unsigned sel = task_sel(args.mx, warp, task.nket);
  const int nsel = __popc(sel);
  if (sizeof(R) == 4 && lane == 0 && args.mx.fp32_count && nsel)
    atomicAdd(args.mx.fp32_count, (unsigned long long)nsel);
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
    __syncwarp();  // the previous quartet's weights are no longer read
    if (active) {
      const bool kl_same = kp.sa == kp.sb, bk_same = task.diag && kpos == task.bra_pos;
      for (int c = sub; c < C::NCOMP; c += G)
        W[c * NG + grp] = R(grad_weight<LA, LB, LC, LD>(D, n, bp, kp, c, ij_same, kl_same, bk_same, xs));
    }
    __syncwarp();
    double gC[3] = {0, 0, 0}, gBq[3] = {0, 0, 0}, gAq[3] = {0, 0, 0};
    if (active) {
      const double CD[3] = {kp.A[0] - kp.B[0], kp.A[1] - kp.B[1], kp.A[2] - kp.B[2]};
      const int nitems = bp.np * kp.np * NR;
      for (int it = sub; it < nitems; it += G) {
        // ket-major order of primitive quartets (see quartet), roots innermost
        const int pq = it / NR, r = it - pq * NR;
        const int pj = pq / bp.np, pi = pq - pj * bp.np;
        const PrimPair k = load_pp(args.pp + kp.pstart + pj);
        const PrimPair b = load_pp(args.pp + bp.pstart + pi);
        if (b.K * k.K < args.prim_thr) continue;
        const double p = b.p, q = k.p, s = p + q;
        const double PQ[3] = {b.P[0] - k.P[0], b.P[1] - k.P[1], b.P[2] - k.P[2]};
        const double rs = rsqrt(s), inv_s = rs * rs;  // 1/(p+q), 1/sqrt(p+q): one rsqrt
        const double rho = p * q * inv_s;
        const double T = rho * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
        const double pref = kTwoPi52 * b.cK * k.cK * b.inv_p * k.inv_p * rs;
        double t2, wr;
        rys_rule_one<NR>(T, r, rtab, &t2, &wr);
        // rys_coefficients.rs:94-180 with u2 (p+q) + pq = pq / (1 - t^2)
        const double b00 = 0.5 * t2 * inv_s, h = 0.5 - 0.5 * t2;
        const double b10 = fma(h, b.inv_p, b00), b01 = fma(h, k.inv_p, b00);
        const double f2 = t2 * q * inv_s, f3 = t2 * p * inv_s;
        const R a2 = R(2.0 * b.aa), b2 = R(2.0 * (b.p - b.aa)), c2 = R(2.0 * k.aa);
        R E[3][ESZ];
#pragma unroll
        for (int ax = 0; ax < 3; ++ax)
          axis_table<R, LA + LB + 1, LC + LD + 1, EA, EB, EC, ED>(
              R(b.P[ax] - bp.A[ax] - f2 * PQ[ax]), R(k.P[ax] - kp.A[ax] + f3 * PQ[ax]), R(b00), R(b10), R(b01),
              R(AB[ax]), R(CD[ax]), R(ax == 2 ? wr * pref : 1.0), E[ax]);
        R pA[3] = {0, 0, 0}, pB[3] = {0, 0, 0}, pC[3] = {0, 0, 0};
#pragma unroll
        for (int a = 0; a < C::NA; ++a)
#pragma unroll
          for (int bb = 0; bb < C::NB; ++bb)
#pragma unroll
            for (int c = 0; c < C::NC; ++c)
#pragma unroll
              for (int d = 0; d < C::ND; ++d) {
                const R w = Wv[(((a * C::NB + bb) * C::NC + c) * C::ND + d) * NG + grp];
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
                pA[0] = fma(wyz, dA[0], pA[0]); pA[1] = fma(wxz, dA[1], pA[1]); pA[2] = fma(wxy, dA[2], pA[2]);
                pB[0] = fma(wyz, dB[0], pB[0]); pB[1] = fma(wxz, dB[1], pB[1]); pB[2] = fma(wxy, dB[2], pB[2]);
                pC[0] = fma(wyz, dC[0], pC[0]); pC[1] = fma(wxz, dC[1], pC[1]); pC[2] = fma(wxy, dC[2], pC[2]);
              }
#pragma unroll
        for (int x = 0; x < 3; ++x) {
          gAq[x] += double(pA[x]);
          gBq[x] += double(pB[x]);
          gC[x] += double(pC[x]);
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
