// Warp-cooperative quartet kernels for the larger angular-momentum classes.
//
// One warp evaluates one contracted shell quartet at a time (the 32 kets of its
// task one after another).  Per surviving primitive quartet:
//   phase A  lanes 0 .. 3*NR-1 each take one (root, axis): the Rys root from
//            the tables, the recurrence coefficients (rys_coefficients.rs:94),
//            the 2D VRR (vrr_2d.rs:143) and the horizontal transfer to B and D
//            (htr_4d.rs), written as one 1D table to shared memory;
//   phase B  every lane accumulates its own components c = lane + 32 m of the
//            block, sum over roots of Ix * Iy * Iz, from packed per-component
//            table offsets held in registers.
// The contracted block is then staged in shared memory and digested into J/K
// (8-fold symmetry, degeneracy factors) with one atomic per output element, or
// for gradients contracted with the D x D weights per primitive quartet.
// Numerics are those of the thread-per-quartet kernels (eri_templates.cuh).
#pragma once
#include "eri_templates.cuh"

namespace iqcp {

// Component ax (runtime) of a 3-vector without indexing it: an indexed
// access would place the vector -- and the ShellPair / PrimPair it belongs to --
// in local memory.
__device__ __forceinline__ double pick3(int ax, double x, double y, double z) {
  return ax == 0 ? x : (ax == 1 ? y : z);
}

// Rule for one root r of an N-point rule (phase A lanes each need one root).
// (table staged in shared memory at s)
template <int N>
__device__ __forceinline__ void rys_rule_one(double T, int r, const double* s, double* t2, double* w) {
  constexpr int NI = rys_nint(N);
  if (T >= double(NI)) {
    const int base = (N * (N - 1)) / 2;
    *t2 = __ldg(kRysAsymRoot + base + r) / T;
    *w = __ldg(kRysAsymWeight + base + r) / sqrt(T);
    return;
  }
  const int k = int(T);
  const double x2 = 2.0 * (2.0 * (T - double(k)) - 1.0);
  const double* c = s + k * rys_tab_stride<N>();
  *t2 = cheb_clenshaw_s(c + r * (RYS_TAB_DEG + 1), x2);
  *w = cheb_clenshaw_s(c + (N + r) * (RYS_TAB_DEG + 1), x2);
}

// Shared-memory footprint (doubles) of one warp of the J/K team kernel
template <int LA, int LB, int LC, int LD>
struct TeamJK {
  using C = Cls<LA, LB, LC, LD>;
  // (root, axis) tables TSP = TSZ | 1 entries apart, so that the lanes of
  // phase A, writing the same entry of consecutive tables, spread over the banks
  static constexpr int TSP = C::TSZ | 1;
  static constexpr int TAB = C::NR * 3 * TSP;
  static constexpr int BLK = C::NCOMP;
  static constexpr int WORK = TAB > BLK ? TAB : BLK;
  static constexpr int DB = C::NA * C::NB + C::NC * C::ND + C::NB * C::ND + C::NA * C::ND + C::NB * C::NC +
                            C::NA * C::NC;
  static constexpr int PER_WARP = WORK + DB;
  static constexpr int CPL = (C::NCOMP + 31) / 32;
  // resident 128-thread blocks asked of the compiler: 4 (128 registers, 16
  // warps per SM) where shared memory admits them and the tables are small
  // enough not to spill (<= 36 entries: ptxas 0-52 bytes); 1 otherwise (the
  // 54- and 81-entry tables spill 250+ bytes at 128 registers)
  static constexpr int SMEM_BLOCKS =
      (228 * 1024) / (int(sizeof(double)) * (4 * PER_WARP + rys_tab_doubles<C::NR>()) + 1024);
  static constexpr int MINB = C::TSZ <= 36 ? (SMEM_BLOCKS < 4 ? (SMEM_BLOCKS > 0 ? SMEM_BLOCKS : 1) : 4) : 1;
};

// One contracted quartet: phases A and B over all surviving primitive
// quartets, accumulating this lane's components into acc (FP64).  R is the
// quadrature type: double, or float for the mixed form (roots, weights and
// recurrence coefficients are formed in FP64 and rounded once).
template <typename R, int LA, int LB, int LC, int LD>
__device__ __forceinline__ void team_prim_loop(const JKArgs& args, const ShellPair& bp, const ShellPair& kp,
                                               const double* AB, const double* CD, const int* offs, double* acc,
                                               R* tab, int lane, const double* rtab) {
  using C = Cls<LA, LB, LC, LD>;
  constexpr int NR = C::NR, TSZ = TeamJK<LA, LB, LC, LD>::TSP, CPL = TeamJK<LA, LB, LC, LD>::CPL;
  for (int i = 0; i < bp.np; ++i) {
    const PrimPair pb = load_pp(args.pp + bp.pstart + i);
    for (int j = 0; j < kp.np; ++j) {
      const PrimPair pk = load_pp(args.pp + kp.pstart + j);
      if (pb.K * pk.K < args.prim_thr) continue;
      if (lane < 3 * NR) {
        const int r = lane / 3, ax = lane - 3 * r;
        const double p = pb.p, q = pk.p, s = p + q;
        const double PQ[3] = {pb.P[0] - pk.P[0], pb.P[1] - pk.P[1], pb.P[2] - pk.P[2]};
        const double rs = rsqrt(s), inv_s = rs * rs;  // 1/(p+q), 1/sqrt(p+q): one rsqrt
        const double rho = p * q * inv_s;
        const double T = rho * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
        double t2, wr;
        rys_rule_one<NR>(T, r, rtab, &t2, &wr);
        const double b00 = 0.5 * t2 * inv_s, h = 0.5 - 0.5 * t2;
        const double b10 = fma(h, pb.inv_p, b00), b01 = fma(h, pk.inv_p, b00);
        const double pa = pick3(ax, pb.P[0] - bp.A[0], pb.P[1] - bp.A[1], pb.P[2] - bp.A[2]);
        const double qc = pick3(ax, pk.P[0] - kp.A[0], pk.P[1] - kp.A[1], pk.P[2] - kp.A[2]);
        const double pq = pick3(ax, PQ[0], PQ[1], PQ[2]);
        const double g00 = ax == 2 ? wr * kTwoPi52 * pb.cK * pk.cK * pb.inv_p * pk.inv_p * rs : 1.0;
        axis_table<R, C::NBRA, C::NKET, LA, LB, LC, LD>(
            R(pa - t2 * q * inv_s * pq), R(qc + t2 * p * inv_s * pq), R(b00), R(b10), R(b01),
            R(pick3(ax, AB[0], AB[1], AB[2])), R(pick3(ax, CD[0], CD[1], CD[2])), R(g00), tab + (r * 3 + ax) * TSZ);
      }
      __syncwarp();
#pragma unroll
      for (int m = 0; m < CPL; ++m) {
        const int o = offs[m];
        const int ox = o & 0xff, oy = (o >> 8) & 0xff, oz = (o >> 16) & 0xff;
        R sum = R(0);
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          const R* t = tab + r * 3 * TSZ;
          sum = fma(t[ox] * t[oy], t[oz], sum);
        }
        acc[m] += double(sum);
      }
      __syncwarp();
    }
  }
}

template <typename R, int LA, int LB, int LC, int LD, bool DO_K>
__global__ void __launch_bounds__(128, TeamJK<LA, LB, LC, LD>::MINB) jk_team_kernel(JKArgs args) {
  using C = Cls<LA, LB, LC, LD>;
  using TM = TeamJK<LA, LB, LC, LD>;
  constexpr int NR = C::NR, TSZ = TM::TSP, CPL = TM::CPL;  // table stride
  extern __shared__ double smem[];
  double* rtab = smem;
  rys_stage_table<NR>(rtab);
  __syncthreads();
  const int wib = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  double* work = smem + rys_tab_doubles<NR>() + wib * TM::PER_WARP;
  double* Dab = work + TM::WORK;
  double* Dcd = Dab + C::NA * C::NB;
  double* Dbd = Dcd + C::NC * C::ND;
  double* Dad = Dbd + C::NB * C::ND;
  double* Dbc = Dad + C::NA * C::ND;
  double* Dac = Dbc + C::NB * C::NC;

  // packed table offsets of this lane's components: x | y << 8 | z << 16
  int offs[CPL];
#pragma unroll
  for (int m = 0; m < CPL; ++m) {
    int comp = lane + 32 * m;
    if (comp >= C::NCOMP) comp = 0;
    const int d = comp % C::ND, c = (comp / C::ND) % C::NC, b = (comp / (C::ND * C::NC)) % C::NB,
              a = comp / (C::ND * C::NC * C::NB);
    int o = 0;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax)
      o |= (ax * TSZ + C::tidx(cart_pow(LA, a, ax), cart_pow(LB, b, ax), cart_pow(LC, c, ax),
                               cart_pow(LD, d, ax))) << (8 * ax);
    offs[m] = o;
  }

  const int S = args.ket_split;  // work items per task (slices of its kets)
  for (int item = next_task(args.next_task, lane); item < args.ntasks * S; item = next_task(args.next_task, lane)) {
  const int warp = item / S;     // the task
  const QuartetTask task = args.tasks[warp];
  const ShellPair bp = args.pairs[task.bra];
  if (task_inactive(args.mol_active, bp.mol)) continue;
  const int kper = (task.nket + S - 1) / S, k_lo = (item - warp * S) * kper;
  const int k_hi = task.nket < k_lo + kper ? task.nket : k_lo + kper;
  // this task's molecule block (bra and ket pairs always share a molecule)
  const int n = args.mol_n[bp.mol];
  const long long mb = args.mol_base[bp.mol];
  const double* __restrict__ D = args.D + mb;
  const double AB[3] = {bp.A[0] - bp.B[0], bp.A[1] - bp.B[1], bp.A[2] - bp.B[2]};
  __syncwarp();
  for (int i = lane; i < C::NA * C::NB; i += 32)
    Dab[i] = __ldg(D + (bp.oa + i / C::NB) * n + bp.ob + i % C::NB);

  int nf32 = 0;
  const unsigned sel = task_sel(args.mx, warp, task.nket);
  for (int kk = k_lo; kk < k_hi; ++kk) {
    if (!((sel >> kk) & 1u)) continue;  // another pass's ket (the same on every lane)
    const int kpos = task.ket0 + kk;
    const ShellPair kp = args.pairs[__ldg(args.ket_list + kpos)];
    const double CD[3] = {kp.A[0] - kp.B[0], kp.A[1] - kp.B[1], kp.A[2] - kp.B[2]};
    double acc[CPL];
#pragma unroll
    for (int m = 0; m < CPL; ++m) acc[m] = 0.0;
    team_prim_loop<R, LA, LB, LC, LD>(args, bp, kp, AB, CD, offs, acc, reinterpret_cast<R*>(work), lane, rtab);
    ++nf32;
    // ---- digestion ----
    double f = 1.0;
    if (bp.sa == bp.sb) f *= 0.5;
    if (kp.sa == kp.sb) f *= 0.5;
    if (task.diag && kpos == task.bra_pos) f *= 0.5;
#pragma unroll
    for (int m = 0; m < CPL; ++m) {
      const int comp = lane + 32 * m;
      if (comp < C::NCOMP) work[comp] = f * acc[m];
    }
    // every density of the call (nset > 1: response densities) is digested
    // with the same integrals
    for (int s = 0; s < args.nset; ++s) {
      const double* __restrict__ Dm = D + s * args.set_stride;
      double* Jm = args.J + mb + s * args.set_stride;
      double* Km = DO_K ? args.K + mb + s * args.set_stride : nullptr;
      if (s > 0) {  // the bra block of this density (set 0's was staged per task)
        __syncwarp();
        for (int i = lane; i < C::NA * C::NB; i += 32)
          Dab[i] = __ldg(Dm + (bp.oa + i / C::NB) * n + bp.ob + i % C::NB);
      }
      for (int i = lane; i < C::NC * C::ND; i += 32) Dcd[i] = __ldg(Dm + (kp.oa + i / C::ND) * n + kp.ob + i % C::ND);
      if (DO_K) {
        for (int i = lane; i < C::NB * C::ND; i += 32) Dbd[i] = __ldg(Dm + (bp.ob + i / C::ND) * n + kp.ob + i % C::ND);
        for (int i = lane; i < C::NA * C::ND; i += 32) Dad[i] = __ldg(Dm + (bp.oa + i / C::ND) * n + kp.ob + i % C::ND);
        for (int i = lane; i < C::NB * C::NC; i += 32) Dbc[i] = __ldg(Dm + (bp.ob + i / C::NC) * n + kp.oa + i % C::NC);
        for (int i = lane; i < C::NA * C::NC; i += 32) Dac[i] = __ldg(Dm + (bp.oa + i / C::NC) * n + kp.oa + i % C::NC);
      }
      __syncwarp();
      // J~_ab += 2 sum_cd I D_cd
      for (int ab = lane; ab < C::NA * C::NB; ab += 32) {
        double v = 0.0;
#pragma unroll
        for (int cd = 0; cd < C::NC * C::ND; ++cd) v = fma(work[ab * C::NC * C::ND + cd], Dcd[cd], v);
        atomicAdd(Jm + (bp.oa + ab / C::NB) * n + bp.ob + ab % C::NB, 2.0 * v);
      }
      // J~_cd += 2 sum_ab I D_ab
      for (int cd = lane; cd < C::NC * C::ND; cd += 32) {
        double v = 0.0;
#pragma unroll
        for (int ab = 0; ab < C::NA * C::NB; ++ab) v = fma(work[ab * C::NC * C::ND + cd], Dab[ab], v);
        atomicAdd(Jm + (kp.oa + cd / C::ND) * n + kp.ob + cd % C::ND, 2.0 * v);
      }
      if (DO_K) {
        // K~_ac += sum_bd I D_bd
        for (int x = lane; x < C::NA * C::NC; x += 32) {
          const int a = x / C::NC, c = x % C::NC;
          double v = 0.0;
#pragma unroll
          for (int b = 0; b < C::NB; ++b)
#pragma unroll
            for (int d = 0; d < C::ND; ++d)
              v = fma(work[((a * C::NB + b) * C::NC + c) * C::ND + d], Dbd[b * C::ND + d], v);
          atomicAdd(Km + (bp.oa + a) * n + kp.oa + c, v);
        }
        // K~_bc += sum_ad I D_ad
        for (int x = lane; x < C::NB * C::NC; x += 32) {
          const int b = x / C::NC, c = x % C::NC;
          double v = 0.0;
#pragma unroll
          for (int a = 0; a < C::NA; ++a)
#pragma unroll
            for (int d = 0; d < C::ND; ++d)
              v = fma(work[((a * C::NB + b) * C::NC + c) * C::ND + d], Dad[a * C::ND + d], v);
          atomicAdd(Km + (bp.ob + b) * n + kp.oa + c, v);
        }
        // K~_ad += sum_bc I D_bc
        for (int x = lane; x < C::NA * C::ND; x += 32) {
          const int a = x / C::ND, d = x % C::ND;
          double v = 0.0;
#pragma unroll
          for (int b = 0; b < C::NB; ++b)
#pragma unroll
            for (int c = 0; c < C::NC; ++c)
              v = fma(work[((a * C::NB + b) * C::NC + c) * C::ND + d], Dbc[b * C::NC + c], v);
          atomicAdd(Km + (bp.oa + a) * n + kp.ob + d, v);
        }
        // K~_bd += sum_ac I D_ac
        for (int x = lane; x < C::NB * C::ND; x += 32) {
          const int b = x / C::ND, d = x % C::ND;
          double v = 0.0;
#pragma unroll
          for (int a = 0; a < C::NA; ++a)
#pragma unroll
            for (int c = 0; c < C::NC; ++c)
              v = fma(work[((a * C::NB + b) * C::NC + c) * C::ND + d], Dac[a * C::NC + c], v);
          atomicAdd(Km + (bp.ob + b) * n + kp.ob + d, v);
        }
      }
      __syncwarp();
    }
    if (args.nset > 1) {  // restore set 0's bra block for the next ket
      for (int i = lane; i < C::NA * C::NB; i += 32)
        Dab[i] = __ldg(D + (bp.oa + i / C::NB) * n + bp.ob + i % C::NB);
    }
    __syncwarp();
  }
  if (sizeof(R) == 4 && lane == 0 && args.mx.fp32_count && nf32) atomicAdd(args.mx.fp32_count, (unsigned long long)nf32);
  }  // task loop
}

// ---------------------------------------------------------------------------
// Gradient team kernel with per-root derivative tables.
//
// Tables are extended by one on A and C (the B derivative takes I(a, b+1) =
// I(a+1, b) + AB I(a, b) from the horizontal recurrence, the D derivative
// follows from translational invariance, dD = -(dA + dB + dC)), with the
// roots of total angular momentum L + 1 (grad_nroots).  Per surviving
// primitive quartet:
//   phase A   fused (tables of <= kTeamFusedMaxTab entries): a lane per
//             (root, axis) builds the whole extended table in registers and
//             writes the four derivative planes below itself; otherwise the
//             lanes build the tables E in shared memory, one row a of a table
//             per lane (axis_slice), and
//   phase A2  all 32 lanes turn them into, for every unextended index
//             (ia, ib, ic, id), the four values I, dI/dA, dI/dB, dI/dC
//             (d/dA: 2a E(ia+1) - ia E(ia-1), likewise B, C), stored as two
//             planes of pairs (I, dA) and (dB, dC);
//   phase B   each lane accumulates its components c = lane + 32 m: per root
//             two vector loads per axis and 15 flops for the nine A/B/C
//             derivatives (instead of ~21 scattered loads when each lane
//             forms the derivatives from E itself).
// The Rys coefficients are read through L1 (the 3*NR lanes of a warp read one
// T interval), so no table is staged per block, and the warps per block are
// chosen so that the per-warp tables fit.
template <int N>
__device__ __forceinline__ void rys_rule_one_g(double T, int r, double* t2, double* w) {
  constexpr int NI = rys_nint(N);
  if (T >= double(NI)) {
    const int base = (N * (N - 1)) / 2;
    *t2 = __ldg(kRysAsymRoot + base + r) / T;
    *w = __ldg(kRysAsymWeight + base + r) / sqrt(T);
    return;
  }
  const int k = int(T);
  const double x2 = 2.0 * (2.0 * (T - double(k)) - 1.0);
  const double* c = kRysCheb + kRysOffset[N] + k * (2 * N * (RYS_TAB_DEG + 1));
  *t2 = cheb_clenshaw(c + r * (RYS_TAB_DEG + 1), x2);
  *w = cheb_clenshaw(c + (N + r) * (RYS_TAB_DEG + 1), x2);
}

// Warps per block for a per-warp shared footprint of `per_warp` doubles: the
// choice of 4, 2, 1 with the most warps resident per SM (228 KB shared memory,
// 1 KB reserved per block; at most 16 counted, beyond which registers limit
// anyway), ties to the larger block.
__host__ __device__ constexpr int team_resident(int w, int per_warp) {
  return w * ((228 * 1024) / (w * per_warp * 8 + 1024)) < 16 ? w * ((228 * 1024) / (w * per_warp * 8 + 1024)) : 16;
}
__host__ __device__ constexpr int team_warps_per_block(int per_warp) {
  return (team_resident(4, per_warp) >= team_resident(2, per_warp) &&
          team_resident(4, per_warp) >= team_resident(1, per_warp) && team_resident(4, per_warp) > 0)
             ? 4
             : (team_resident(2, per_warp) >= team_resident(1, per_warp) && team_resident(2, per_warp) > 0 ? 2 : 1);
}

// Per-warp shared-memory budget (doubles) of the gradient team kernel; 20 KB
// leaves room for about eleven resident warps per SM.
constexpr int kTeamGradBudget = 2560;
// Largest extended table (entries) that one lane builds whole in registers
// (the fused phase A); up to 96 the spill is a few hundred bytes, which costs
// less than the shared table it replaces.
constexpr int kTeamFusedMaxTab = 96;
// Register budget per thread of the gradient team kernel (sets its minimum
// resident blocks): 128, i.e. 16 warps per SM where shared memory allows,
// except for extended tables above 72 entries, whose register-resident fused
// phase A then spills more than the extra warps gain ((dd|dp): 2.55 ms at 168
// registers, 2.66 ms at 128; (dp|pp) 6.83 -> 6.67 ms, (dp|ds) 5.49 -> 5.01 ms)
constexpr int team_grad_regs(int tsz) { return tsz <= 72 ? 128 : 168; }

template <int LA, int LB, int LC, int LD>
struct TeamGrad2 {
  using C = Cls<LA, LB, LC, LD>;
  static constexpr int EA = LA + 1, EB = LB, EC = LC + 1, ED = LD;  // B derivative via I(a+1,b) + AB I(a,b)
  static constexpr int NR = grad_nroots(LA + LB + LC + LD);
  static constexpr int TSZ = (EA + 1) * (EB + 1) * (EC + 1) * (ED + 1);
  // extended tables TSP = TSZ | 1 entries apart: the lanes of phase A write the
  // same entry of consecutive tables, which an even stride (48, 64, 72 ...)
  // puts in one or two banks
  static constexpr int TSP = TSZ | 1;
  // fused phase A: one lane per (root, axis) builds its whole table in
  // registers and writes the derivative planes itself (no shared E table)
  static constexpr bool FUSED = TSZ <= kTeamFusedMaxTab;
  static constexpr int SA = (EB + 1) * (EC + 1) * (ED + 1), SB = (EC + 1) * (ED + 1), SC = ED + 1;
  static constexpr int RSZ = (LA + 1) * (LB + 1) * (LC + 1) * (LD + 1);
  // derivative tables: one row per bra index pair (ia, ib) of KQ = (LC+1)(LD+1)
  // ket entries, rows KQP = KQ | 1 entries apart (an odd pitch spreads the rows
  // that the lanes of a warp read over the shared-memory banks)
  static constexpr int KQ = (LC + 1) * (LD + 1);
  static constexpr int KQP = KQ | 1;
  static constexpr int RSZP = (LA + 1) * (LB + 1) * KQP;
  __host__ __device__ static constexpr int qpos(int e) { return (e / KQ) * KQP + e % KQ; }
  // pair (I, dA) / (dB, dC) index of entry position pos in plane pl of table t:
  // planes RSZP + 1 pairs apart and tables 2 RSZP + 1, so the lanes of the
  // fused phase A (one table each) store to different banks
  static constexpr int PSTR = RSZP + 1, TSTR = 2 * RSZP + 1;
  __host__ __device__ static constexpr int pair(int t, int pl, int pos) { return t * TSTR + pl * PSTR + pos; }
  // RBATCH: the Rys rules of JCH ket primitives come from one pass of the
  // warp (a lane per (primitive, root)) ahead of their primitive quartets;
  // otherwise NR lanes compute each quartet's rule.  Measured per class on
  // the 40-atom 6-31G* step: batching gains 3-6% with pp and dd kets and
  // loses 15-40% with ds kets and for (dd|dp)
  static constexpr bool RBATCH = (LC == 1 && LD == 1) || (LC == 2 && LD == 2);
  // at most 6 primitives: with 8, (dp|pp)'s four blocks of four warps (and
  // the per-block gradient accumulator) exceed the SM's shared memory by 1.5 KB
  static constexpr int JCH = RBATCH ? (32 / NR < 6 ? 32 / NR : 6) : 1;
  static constexpr int DBLK = C::NA * C::NB + C::NC * C::ND + C::NA * C::NC + C::NB * C::ND + C::NA * C::ND +
                              C::NB * C::NC;
  // shared footprint (doubles) with the tables of rch roots at a time
  static constexpr int footprint(int rch) {
    return (FUSED ? 0 : ((3 * rch * TSP + 3) / 4) * 4) + ((3 * rch * TSTR * 2 + 3) / 4) * 4 + ((DBLK + 3) / 4) * 4 +
           ((C::NCOMP + 1) / 2) * 2 + 2 * NR * JCH;
  }
  static constexpr int pick_rch(int rch) {
    return (rch <= 1 || footprint(rch) <= kTeamGradBudget) ? rch : pick_rch(rch - 1);
  }
  // roots per pass of phases A, A2 and B: all of them, or as many as keep the
  // per-warp tables within the budget (the (dd|..) and (dp|dp) classes)
  static constexpr int RCH = pick_rch(NR);
  static constexpr int NT = 3 * RCH;                      // (root, axis) tables of one pass
  static constexpr int TAB = FUSED ? 0 : ((NT * TSP + 3) / 4) * 4;  // extended tables (doubles, padded)
  static constexpr int QT = ((NT * TSTR * 2 + 3) / 4) * 4;  // I, dA, dB, dC per unextended entry
  static constexpr int WOFF = TAB + QT + ((DBLK + 3) / 4) * 4;  // D x D weights of the quartet (NCOMP)
  static constexpr int ROFF = WOFF + ((C::NCOMP + 1) / 2) * 2;  // Rys roots and weights of JCH ket primitives
  static constexpr int PER_WARP = ROFF + 2 * NR * JCH;
  // phase B items: (root, bra component pair) looping over the ket components,
  // or for kets of more than 9 components (root, bra pair, c) looping over d
  static constexpr bool BYC = C::NC * C::ND > 9;
  static constexpr int NITEM = RCH * C::NA * C::NB * (BYC ? C::NC : 1);  // per pass (whole chunk)
  static constexpr int CPL = (C::NCOMP + 31) / 32;
  static constexpr int WPB = team_warps_per_block(PER_WARP);
  // resident blocks per SM asked of the compiler: what shared memory allows,
  // but no more than leaves TREG registers per thread (65536 / (MINB * 32 * WPB))
  static constexpr int TREG = team_grad_regs(TSZ);
  static constexpr int SMB = team_resident(WPB, PER_WARP) / WPB;
  static constexpr int RGB = 65536 / (TREG * 32 * WPB);
  static constexpr int MINB = (SMB < RGB ? SMB : RGB) > 0 ? (SMB < RGB ? SMB : RGB) : 1;
  __host__ __device__ static constexpr int eidx(int a, int b, int c, int d) {
    return ((a * (EB + 1) + b) * (EC + 1) + c) * (ED + 1) + d;
  }
  __host__ __device__ static constexpr int ridx(int a, int b, int c, int d) {
    return ((a * (LB + 1) + b) * (LC + 1) + c) * (LD + 1) + d;
  }
};

template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

template <typename R, int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(32 * TeamGrad2<LA, LB, LC, LD>::WPB, TeamGrad2<LA, LB, LC, LD>::MINB)
grad_team2_kernel(GradArgs args) {
  using C = Cls<LA, LB, LC, LD>;
  using TG = TeamGrad2<LA, LB, LC, LD>;
  using V2 = typename Vec2<R>::type;
  constexpr int NR = TG::NR, RSZ = TG::RSZ, CPL = TG::CPL;
  extern __shared__ __align__(16) double smem[];
  const int wib = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  double* wbase = smem + wib * TG::PER_WARP;
  R* tab = reinterpret_cast<R*>(wbase);
  R* qt = reinterpret_cast<R*>(wbase + TG::TAB);
  double* gacc = smem + TG::WPB * TG::PER_WARP;
  if (args.gsmem)
    for (int i = threadIdx.x; i < 3 * args.natoms; i += blockDim.x) gacc[i] = 0.0;
  __syncthreads();
  double* gout = args.gsmem ? gacc : args.grad;
  double* Dab = wbase + TG::TAB + TG::QT;
  double* Dcd = Dab + C::NA * C::NB;
  double* Dac = Dcd + C::NC * C::ND;
  double* Dbd = Dac + C::NA * C::NC;
  double* Dad = Dbd + C::NB * C::ND;
  double* Dbc = Dad + C::NA * C::ND;

  R* Wsh = reinterpret_cast<R*>(wbase + TG::WOFF);   // weights of the current quartet
  double* rts_all = wbase + TG::ROFF;                // t^2 and weight of each (ket primitive, root)

  const int S = args.ket_split;  // work items per task (slices of its kets)
  for (int item = next_task(args.next_task, lane); item < args.ntasks * S; item = next_task(args.next_task, lane)) {
  const int warp = item / S;     // the task
  const QuartetTask task = args.tasks[warp];
  const ShellPair bp = args.pairs[task.bra];
  const int kper = (task.nket + S - 1) / S, k_lo = (item - warp * S) * kper;
  const int k_hi = task.nket < k_lo + kper ? task.nket : k_lo + kper;
  // this task's molecule block (bra and ket pairs always share a molecule)
  const int n = args.mol_n[bp.mol];
  const long long mb = args.mol_base[bp.mol];
  const double* __restrict__ D = args.D + mb;
  const double AB[3] = {bp.A[0] - bp.B[0], bp.A[1] - bp.B[1], bp.A[2] - bp.B[2]};
  __syncwarp();
  for (int i = lane; i < C::NA * C::NB; i += 32)
    Dab[i] = __ldg(D + (bp.oa + i / C::NB) * n + bp.ob + i % C::NB);
  const bool ij_same = bp.sa == bp.sb;
  const double xs = args.xscale;
  int nsel = 0;
  const unsigned sel = task_sel(args.mx, warp, task.nket);

  for (int kk = k_lo; kk < k_hi; ++kk) {
    if (!((sel >> kk) & 1u)) continue;  // another pass's ket (the same on every lane)
    const int kpos = task.ket0 + kk;
    const ShellPair kp = args.pairs[__ldg(args.ket_list + kpos)];
    // the reference skips when the Schwarz bound of its bra pair (the larger
    // composite index) is below threshold (gradient.rs:1457-1460)
    const double qref = bp.comp >= kp.comp ? bp.Q : kp.Q;
    if (qref < args.schwarz_thr) continue;
    ++nsel;
    const bool kl_same = kp.sa == kp.sb;
    const bool bk_same = task.diag && kpos == task.bra_pos;
    for (int i = lane; i < C::NC * C::ND; i += 32) Dcd[i] = __ldg(D + (kp.oa + i / C::ND) * n + kp.ob + i % C::ND);
    for (int i = lane; i < C::NA * C::NC; i += 32) Dac[i] = __ldg(D + (bp.oa + i / C::NC) * n + kp.oa + i % C::NC);
    for (int i = lane; i < C::NB * C::ND; i += 32) Dbd[i] = __ldg(D + (bp.ob + i / C::ND) * n + kp.ob + i % C::ND);
    for (int i = lane; i < C::NA * C::ND; i += 32) Dad[i] = __ldg(D + (bp.oa + i / C::ND) * n + kp.ob + i % C::ND);
    for (int i = lane; i < C::NB * C::NC; i += 32) Dbc[i] = __ldg(D + (bp.ob + i / C::NC) * n + kp.oa + i % C::NC);
    __syncwarp();
    // D x D weights of the quartet's components into shared memory
    // (compute_symmetry_weight, gradient.rs:1570-1640)
    for (int comp = lane; comp < C::NCOMP; comp += 32) {
      const int d = comp % C::ND, c = (comp / C::ND) % C::NC, b = (comp / (C::ND * C::NC)) % C::NB,
                a = comp / (C::ND * C::NC * C::NB);
      const double dab = Dab[a * C::NB + b], dcd = Dcd[c * C::ND + d];
      const double dac = Dac[a * C::NC + c], dbd = Dbd[b * C::ND + d];
      const double dad = Dad[a * C::ND + d], dbc = Dbc[b * C::NC + c];
      // w(p,q,r,s) = 1/2 D_pq D_rs - xs D_pr D_qs over the distinct permutations
      double t = 0.5 * dab * dcd - xs * dac * dbd;
      if (!ij_same) t += 0.5 * dab * dcd - xs * dbc * dad;
      if (!kl_same) t += 0.5 * dab * dcd - xs * dad * dbc;
      if (!ij_same && !kl_same) t += 0.5 * dab * dcd - xs * dbd * dac;
      if (!bk_same) {
        t += 0.5 * dcd * dab - xs * dac * dbd;
        if (!kl_same) t += 0.5 * dcd * dab - xs * dad * dbc;
        if (!ij_same) t += 0.5 * dcd * dab - xs * dbc * dad;
        if (!ij_same && !kl_same) t += 0.5 * dcd * dab - xs * dbd * dac;
      }
      const double angp = ang_factor(LA, a) * ang_factor(LB, b) * ang_factor(LC, c) * ang_factor(LD, d);
      Wsh[comp] = R(fabs(t / angp) < 1e-15 ? 0.0 : t);  // |w| < 1e-15 skip on the reference weight
    }
    double g[9];
#pragma unroll
    for (int x = 0; x < 9; ++x) g[x] = 0.0;
    const double CD[3] = {kp.A[0] - kp.B[0], kp.A[1] - kp.B[1], kp.A[2] - kp.B[2]};
    for (int i = 0; i < bp.np; ++i) {
      const PrimPair pb = load_pp(args.pp + bp.pstart + i);
      for (int j = 0; j < kp.np; ++j) {
        const PrimPair pk = load_pp(args.pp + kp.pstart + j);
        const int jj = TG::RBATCH ? j % TG::JCH : 0;
        if constexpr (TG::RBATCH) {
          // the rules of ket primitives j .. j + JCH - 1, one lane per
          // (primitive, root); screened pairs are computed too and never read
          if (jj == 0) {
            __syncwarp();
            const int jl = lane / NR, r = lane - jl * NR;
            if (jl < TG::JCH && j + jl < kp.np) {
              const PrimPair pl = load_pp(args.pp + kp.pstart + j + jl);
              const double PQ[3] = {pb.P[0] - pl.P[0], pb.P[1] - pl.P[1], pb.P[2] - pl.P[2]};
              const double rs = rsqrt(pb.p + pl.p);
              const double T = pb.p * pl.p * (rs * rs) * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
              double t2, wr;
              rys_rule_one_g<NR>(T, r, &t2, &wr);
              rts_all[2 * lane] = t2;
              rts_all[2 * lane + 1] = wr;
            }
          }
        }
        if (pb.K * pk.K < args.prim_thr) continue;
        const double p = pb.p, q = pk.p, s = p + q;
        const double PQ[3] = {pb.P[0] - pk.P[0], pb.P[1] - pk.P[1], pb.P[2] - pk.P[2]};
        const double rs = rsqrt(s), inv_s = rs * rs;  // 1/(p+q), 1/sqrt(p+q): one rsqrt
        if constexpr (!TG::RBATCH) {
          __syncwarp();
          if (lane < NR) {  // the Rys rule, one root per lane
            const double T = p * q * inv_s * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
            double t2, wr;
            rys_rule_one_g<NR>(T, lane, &t2, &wr);
            rts_all[2 * lane] = t2;
            rts_all[2 * lane + 1] = wr;
          }
        }
        const double* rts = rts_all + 2 * NR * jj;
        R gl[9];
#pragma unroll
        for (int x = 0; x < 9; ++x) gl[x] = R(0);
        for (int r0 = 0; r0 < NR; r0 += TG::RCH) {  // roots in passes of RCH
        const int nr = NR - r0 < TG::RCH ? NR - r0 : TG::RCH;
        __syncwarp();
        if constexpr (TG::FUSED) {
          // phase A, fused: a lane per (root, axis) builds the whole extended
          // table in registers and writes I, dI/dA, dI/dB, dI/dC of every
          // unextended entry as two planes of pairs
          const R e2a = R(2.0 * pb.aa), e2b = R(2.0 * (pb.p - pb.aa)), e2c = R(2.0 * pk.aa);
          for (int t = lane; t < 3 * nr; t += 32) {
            const int r = r0 + t / 3, ax = t % 3;
            const double t2 = rts[2 * r], wr = rts[2 * r + 1];
            const double b00 = 0.5 * t2 * inv_s, h = 0.5 - 0.5 * t2;
            const double b10 = fma(h, pb.inv_p, b00), b01 = fma(h, pk.inv_p, b00);
            const double pa = pick3(ax, pb.P[0] - bp.A[0], pb.P[1] - bp.A[1], pb.P[2] - bp.A[2]);
            const double qc = pick3(ax, pk.P[0] - kp.A[0], pk.P[1] - kp.A[1], pk.P[2] - kp.A[2]);
            const double pq = pick3(ax, PQ[0], PQ[1], PQ[2]);
            const double g00 = ax == 2 ? wr * kTwoPi52 * pb.cK * pk.cK * pb.inv_p * pk.inv_p * rs : 1.0;
            const R abx = R(pick3(ax, AB[0], AB[1], AB[2])), cdx = R(pick3(ax, CD[0], CD[1], CD[2]));
            R E[TG::TSZ];
            axis_table<R, TG::EA + TG::EB, TG::EC + TG::ED, TG::EA, TG::EB, TG::EC, TG::ED>(
                R(pa - t2 * q * inv_s * pq), R(qc + t2 * p * inv_s * pq), R(b00), R(b10), R(b01), abx, cdx, R(g00),
                E);
            V2* q0 = reinterpret_cast<V2*>(qt + TG::pair(t, 0, 0) * 2);
            V2* q1 = reinterpret_cast<V2*>(qt + TG::pair(t, 1, 0) * 2);
#pragma unroll
            for (int e = 0; e < RSZ; ++e) {
              const int d = e % (LD + 1), c = (e / (LD + 1)) % (LC + 1), b = (e / ((LD + 1) * (LC + 1))) % (LB + 1),
                        a = e / ((LD + 1) * (LC + 1) * (LB + 1));
              const int x = TG::eidx(a, b, c, d);
              const R ex = E[x], ea = E[x + TG::SA];
              V2 v0, v1;
              v0.x = ex;
              v0.y = a ? e2a * ea - R(a) * E[a ? x - TG::SA : x] : e2a * ea;
              v1.x = b ? e2b * (ea + abx * ex) - R(b) * E[b ? x - TG::SB : x] : e2b * (ea + abx * ex);
              v1.y = c ? e2c * E[x + TG::SC] - R(c) * E[c ? x - TG::SC : x] : e2c * E[x + TG::SC];
              q0[TG::qpos(e)] = v0;
              q1[TG::qpos(e)] = v1;
            }
          }
        } else {
        // phase A: (root, axis, row a) slices of the extended tables, one per lane
        for (int task = lane; task < 3 * nr * (TG::EA + 1); task += 32) {
          const int a = task / (3 * nr), t = task - a * (3 * nr);
          const int r = r0 + t / 3, ax = t % 3;
          const double t2 = rts[2 * r], wr = rts[2 * r + 1];
          const double b00 = 0.5 * t2 * inv_s, h = 0.5 - 0.5 * t2;
          const double b10 = fma(h, pb.inv_p, b00), b01 = fma(h, pk.inv_p, b00);
          const double pa = pick3(ax, pb.P[0] - bp.A[0], pb.P[1] - bp.A[1], pb.P[2] - bp.A[2]);
          const double qc = pick3(ax, pk.P[0] - kp.A[0], pk.P[1] - kp.A[1], pk.P[2] - kp.A[2]);
          const double pq = pick3(ax, PQ[0], PQ[1], PQ[2]);
          const double g00 = ax == 2 ? wr * kTwoPi52 * pb.cK * pk.cK * pb.inv_p * pk.inv_p * rs : 1.0;
          const R c00 = R(pa - t2 * q * inv_s * pq), c0p = R(qc + t2 * p * inv_s * pq);
          const R abx = R(pick3(ax, AB[0], AB[1], AB[2])), cdx = R(pick3(ax, CD[0], CD[1], CD[2]));
          R* dst = tab + t * TG::TSP;
#define IQCP_SLICE(AV)                                                                                  \
  axis_slice<R, LA + LB + 1, LC + LD + 1, TG::EA, TG::EB, TG::EC, TG::ED, AV>(                          \
      c00, c0p, R(b00), R(b10), R(b01), abx, cdx, R(g00), dst)
          if (a == 0) IQCP_SLICE(0);
          else if (a == 1) IQCP_SLICE(1);
          else if constexpr (TG::EA >= 2) {
            if (a == 2) IQCP_SLICE((TG::EA >= 2 ? 2 : 0));
            else if constexpr (TG::EA >= 3) IQCP_SLICE((TG::EA >= 3 ? 3 : 0));
          }
#undef IQCP_SLICE
        }
        __syncwarp();
        // phase A2: I, dI/dA, dI/dB, dI/dC on the unextended indices
        {
          const R e2a = R(2.0 * pb.aa), e2b = R(2.0 * (pb.p - pb.aa)), e2c = R(2.0 * pk.aa);
          for (int it = lane; it < 3 * nr * RSZ; it += 32) {
            const int t = it / RSZ, e = it - t * RSZ;
            const R abx = R(pick3(t % 3, AB[0], AB[1], AB[2]));
            const int d = e % (LD + 1), c = (e / (LD + 1)) % (LC + 1), b = (e / ((LD + 1) * (LC + 1))) % (LB + 1),
                      a = e / ((LD + 1) * (LC + 1) * (LB + 1));
            const R* E = tab + t * TG::TSP;
            const int x = TG::eidx(a, b, c, d);
            // two planes of pairs per table, (I, dA) and (dB, dC), 2 * sizeof(R) apart
            // per entry, so that lanes reading different entries spread over the banks
            V2* q0 = reinterpret_cast<V2*>(qt + TG::pair(t, 0, TG::qpos(e)) * 2);
            V2* q1 = reinterpret_cast<V2*>(qt + TG::pair(t, 1, TG::qpos(e)) * 2);
            // power 0 has no lowered term; the index is clamped so no load leaves the table
            const R ex = E[x], ea = E[x + TG::SA];
            V2 v0, v1;
            v0.x = ex;
            v0.y = e2a * ea - R(a) * E[a ? x - TG::SA : x];
            v1.x = e2b * (ea + abx * ex) - R(b) * E[b ? x - TG::SB : x];  // I(a, b+1) by the HRR
            v1.y = e2c * E[x + TG::SC] - R(c) * E[c ? x - TG::SC : x];
            *q0 = v0;  // one paired store per plane
            *q1 = v1;
          }
        }
        }  // phase A
        __syncwarp();
        // phase B: items (root, a, b[, c]); a lane loads each (I, dA, dB, dC) pair
        // of its table rows once and reuses it over the ket components of the item
        const int nitem = nr * (TG::NITEM / TG::RCH);
        for (int item = lane; item < nitem; item += 32) {
          int rest = item;
          int c0 = 0;
          if constexpr (TG::BYC) {
            c0 = rest % C::NC;
            rest /= C::NC;
          }
          const int ab = rest % (C::NA * C::NB), r = rest / (C::NA * C::NB);
          const int a = ab / C::NB, b = ab - a * C::NB;
          // this item's rows: QI (I, dA) and (dB, dC) pairs per axis, loaded once
          constexpr int QI = TG::BYC ? LD + 1 : TG::KQ;
          V2 q0[3][QI], q1[3][QI];
#pragma unroll
          for (int ax = 0; ax < 3; ++ax) {
            const int t = r * 3 + ax;
            const int row = cart_pow(LA, a, ax) * (LB + 1) + cart_pow(LB, b, ax);
            const int pos = row * TG::KQP + (TG::BYC ? cart_pow(LC, c0, ax) * (LD + 1) : 0);
            const V2* p0 = reinterpret_cast<const V2*>(qt + TG::pair(t, 0, pos) * 2);
            const V2* p1 = reinterpret_cast<const V2*>(qt + TG::pair(t, 1, pos) * 2);
#pragma unroll
            for (int j = 0; j < QI; ++j) {
              q0[ax][j] = p0[j];  // I, dI/dA
              q1[ax][j] = p1[j];  // dI/dB, dI/dC
            }
          }
          const R* wrow = Wsh + ab * (C::NC * C::ND) + c0 * C::ND;
#pragma unroll
          for (int cc = 0; cc < (TG::BYC ? 1 : C::NC); ++cc)
#pragma unroll
            for (int d = 0; d < C::ND; ++d) {
              const R w = wrow[cc * C::ND + d];
              V2 v0[3], v1[3];
#pragma unroll
              for (int ax = 0; ax < 3; ++ax) {
                const int j = (TG::BYC ? 0 : cart_pow(LC, cc, ax) * (LD + 1)) + cart_pow(LD, d, ax);
                v0[ax] = q0[ax][j];
                v1[ax] = q1[ax][j];
              }
              const R wyz = w * v0[1].x * v0[2].x, wxz = w * v0[0].x * v0[2].x, wxy = w * v0[0].x * v0[1].x;
              gl[0] = fma(wyz, v0[0].y, gl[0]); gl[1] = fma(wxz, v0[1].y, gl[1]); gl[2] = fma(wxy, v0[2].y, gl[2]);
              gl[3] = fma(wyz, v1[0].x, gl[3]); gl[4] = fma(wxz, v1[1].x, gl[4]); gl[5] = fma(wxy, v1[2].x, gl[5]);
              gl[6] = fma(wyz, v1[0].y, gl[6]); gl[7] = fma(wxz, v1[1].y, gl[7]); gl[8] = fma(wxy, v1[2].y, gl[8]);
            }
        }
        }  // root passes
#pragma unroll
        for (int x = 0; x < 9; ++x) g[x] += double(gl[x]);
      }
    }
    // warp reduction of the nine derivatives, then atomics (D by invariance)
#pragma unroll
    for (int x = 0; x < 9; ++x) g[x] = warp_sum(g[x]);
    if (lane == 0) {
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        atomicAdd(gout + 3 * bp.atom_a + ax, g[ax]);
        atomicAdd(gout + 3 * bp.atom_b + ax, g[3 + ax]);
        atomicAdd(gout + 3 * kp.atom_a + ax, g[6 + ax]);
        atomicAdd(gout + 3 * kp.atom_b + ax, -(g[ax] + g[3 + ax] + g[6 + ax]));
      }
    }
    __syncwarp();
  }
  if (sizeof(R) == 4 && lane == 0 && args.mx.fp32_count && nsel) atomicAdd(args.mx.fp32_count, (unsigned long long)nsel);
  }  // task loop
  if (args.gsmem) {
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * args.natoms; i += blockDim.x)
      if (gacc[i] != 0.0) atomicAdd(args.grad + i, gacc[i]);
  }
}

}  // namespace iqcp
