// Shared device/host definitions of the ERI engine: shell-pair tables in HBM,
// quartet tasks, Cartesian component tables.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace iqcp {

constexpr int kNumModes = 4;  // quartet-kernel variants per class

// Default variant before autotuning: warp-cooperative for component-rich
// classes, one quartet per thread for the rest.
__host__ __device__ constexpr int default_mode(int X, int Y, int kind) {
  return ((X == 5 || (X == 4 && Y >= 2)) && !(kind == 1 && X == 4 && Y == 3)) ? 1 : 0;
}

// Angular-momentum classes of a shell pair with la >= lb:
// 0 ss, 1 ps, 2 pp, 3 ds, 4 dp, 5 dd  (index la*(la+1)/2 + lb)
constexpr int kNumPairClasses = 6;
constexpr int kMaxL = 2;

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
// Rys roots of the first-derivative integrals.  Every product the gradient
// contracts has one index raised by one, total angular momentum L + 1, i.e. a
// polynomial of degree L + 1 in t^2, which an n-point rule integrates exactly
// once 2n - 1 >= L + 1.  (The reference takes L/2 + 2 for even L,
// integrals/eri/mod.rs:2146-2147, one root more than exactness needs; the
// results agree to rounding.)
__host__ __device__ constexpr int grad_nroots(int L) { return (L + 1) / 2 + 1; }
__host__ __device__ constexpr int pair_class(int la, int lb) { return la * (la + 1) / 2 + lb; }
__host__ __device__ constexpr int class_la(int c) { return c == 0 ? 0 : (c <= 2 ? 1 : 2); }
__host__ __device__ constexpr int class_lb(int c) { return c - class_la(c) * (class_la(c) + 1) / 2; }

// Cartesian powers, reference order (integrals/cartesian.rs:113-136):
// x exponent descending, then y exponent descending.
__host__ __device__ constexpr int cart_pow(int l, int c, int axis) {
  // l = 0: (000); l = 1: x y z; l = 2: xx xy xz yy yz zz
  return l == 0 ? 0
       : l == 1 ? (c == axis ? 1 : 0)
       : (axis == 0 ? (c == 0 ? 2 : (c <= 2 ? 1 : 0))
          : axis == 1 ? (c == 1 ? 1 : (c == 3 ? 2 : (c == 4 ? 1 : 0)))
                      : (c == 2 ? 1 : (c == 4 ? 1 : (c == 5 ? 2 : 0))));
}

// One primitive pair of a shell pair (A first, la >= lb), 64 bytes.
struct __align__(16) PrimPair {
  double p;       // alpha_a + alpha_b
  double P[3];    // Gaussian product centre
  double K;       // exp(-alpha_a alpha_b / p |AB|^2)  (screening value)
  double cK;      // K * c_a * c_b * Nrad(alpha_a, la) * Nrad(alpha_b, lb)
  double aa;      // alpha_a (alpha_b = p - alpha_a)
  double inv_p;   // 1 / p
};

// One shell pair (la >= lb after the swap), 64 bytes.
struct __align__(16) ShellPair {
  double A[3];
  double B[3];
  double Q;       // Schwarz bound sqrt(max |(ab|ab)|)
  int pstart;     // first PrimPair
  int np;         // number of PrimPairs (K >= prim threshold)
  int oa, ob;     // first basis function of shell a / b
  int sa, sb;     // shell indices (for same-shell degeneracy)
  int atom_a, atom_b;
  int comp;       // reference composite index si(si+1)/2+sj, si>=sj
  int mol;        // molecule of a batched context (0 for a single geometry)
};

// Unit of work for one warp: one bra pair against up to 32 consecutive ket
// pairs of a class list.
struct QuartetTask {
  int bra;        // ShellPair index
  int ket0;       // first position in the ket class list
  int nket;       // 1..32
  int diag;       // 1 when bra and ket lists are the same class (position ket0+i == bra_pos => pair with itself)
  int bra_pos;    // position of the bra in its class list
  int flags;      // reserved (0)
};

// Dynamic task distribution of the persistent quartet kernels: lane 0 of a
// warp takes the next task index from the launch's counter.
__device__ __forceinline__ int next_task(int* counter, int lane) {
  int t = 0;
  if (lane == 0) t = atomicAdd(counter, 1);
  return __shfl_sync(0xffffffffu, t, 0);
}

// Mixed precision.  A mixed call runs a class either wholly in FP64 or twice
// over the same task list: pass 1 takes the quartets whose bound
// Q_ij Q_kl Dmax is at or above the cutoff (FP64 quadrature), pass 2 the rest
// (FP32 quadrature, FP64 roots, weights and accumulation).  Dmax is the
// largest |D| over the six shell blocks the quartet digests with (J/K) or its
// square (gradient, whose weights are products of two density elements).
// Pass 0 takes every quartet.  The split is fixed once per call as a bit mask
// per task (precision_mask_kernel).
struct Mixed {
  const double* dmax;       // per molecule: max |D| per shell block, ns x ns at dbase[m]
  const long long* dbase;
  const int* shell0;        // per molecule: first global shell
  const int* ns;            // per molecule: shell count
  double cutoff;
  int pass;                 // 0 all, 1 FP64 share, 2 FP32 share
  unsigned long long* fp32_count;  // quartets evaluated in pass 2 (may be null)
  const unsigned* mask;     // per task of the launch: bit k set = ket k runs in FP32 (passes 1, 2)
};

__device__ __forceinline__ double mixed_dbound(const Mixed& mx, const ShellPair& bp, const ShellPair& kp) {
  const int m = bp.mol, s0 = mx.shell0[m], ns = mx.ns[m];
  const double* dm = mx.dmax + mx.dbase[m];
  const int i = bp.sa - s0, j = bp.sb - s0, k = kp.sa - s0, l = kp.sb - s0;
  return fmax(fmax(dm[i * ns + j], dm[k * ns + l]),
              fmax(fmax(dm[i * ns + k], dm[i * ns + l]), fmax(dm[j * ns + k], dm[j * ns + l])));
}

// Bit mask of a task's kets in this launch's pass.
__device__ __forceinline__ unsigned task_sel(const Mixed& mx, int task, int nket) {
  const unsigned all = nket >= 32 ? 0xffffffffu : ((1u << nket) - 1u);
  if (mx.pass == 0) return all;
  const unsigned f32 = __ldg(mx.mask + task);
  return mx.pass == 2 ? (f32 & all) : (all & ~f32);
}

// Position of the (k+1)-th set bit of mask (k < popc(mask)).
__device__ __forceinline__ int nth_set_bit(unsigned mask, int k) {
  for (int i = 0; i < k; ++i) mask &= mask - 1;
  return __ffs(mask) - 1;
}

// Kernel argument blocks (passed by value).
struct JKArgs {
  const ShellPair* pairs;
  const PrimPair* pp;
  const int* ket_list;
  const QuartetTask* tasks;
  int ntasks;
  const double* D;   // angular-scaled density
  int nbf;
  double* J;         // unsymmetrised accumulators (nbf x nbf)
  double* K;         // may be null
  double prim_thr;
  int mode;          // kernel variant: 0 thread per quartet, 1 warp-cooperative, 2/3: 8/32 lanes per quartet
  Mixed mx;
  int* next_task;             // work counter (zeroed before the launch)
  int ket_split = 1;          // team kernels: warps per task, each taking a slice of its kets
  const long long* mol_base;  // per molecule: offset of its nbf x nbf block in D, J, K
  const int* mol_n;           // per molecule: nbf (row stride of its block)
  int nset;                   // densities digested per quartet (1, or several response densities)
  long long set_stride;       // elements between consecutive densities in D, J and K
  const int* mol_active;      // per molecule: 0 = skip its tasks (a converged geometry of a batched SCF); may be null
};

// Tasks of molecules flagged inactive are skipped (the same on every lane).
__device__ __forceinline__ bool task_inactive(const int* mol_active, int mol) {
  return mol_active != nullptr && __ldg(mol_active + mol) == 0;
}

struct StoreArgs {
  const ShellPair* pairs;
  const PrimPair* pp;
  const int* ket_list;
  const QuartetTask* tasks;
  int ntasks;
  double* out;
  double prim_thr;
};

struct GradArgs {
  const ShellPair* pairs;
  const PrimPair* pp;
  const int* ket_list;
  const QuartetTask* tasks;
  int ntasks;
  const double* D;   // angular-scaled density
  int nbf;
  double xscale;     // 0.25 * hf_frac
  double* grad;      // natoms x 3
  double prim_thr;
  double schwarz_thr;
  int mode;          // kernel variant: 0 thread per quartet, 1 warp-cooperative, 2/3: 8/32 lanes per quartet
  int natoms;        // gradient rows; accumulated per block in shared memory when gsmem
  int gsmem;
  Mixed mx;
  int* next_task;    // work counter (zeroed before the launch)
  int ket_split = 1;  // team kernel: warps per task, each taking a slice of its kets
  const long long* mol_base;  // per molecule: offset of its block in D
  const int* mol_n;           // per molecule: nbf
};

struct OneEArgs {
  int n_shells, n_atoms, nbf;
  const int* l;
  const int* nprim;
  const int* pstart;
  const int* off;
  const double* center;
  const double* exps;
  const double* coefs;
  const double* atom_xyz;
  const int* z;
  double* S;  // may be null
  double* T;  // may be null
  double* V;  // may be null
  // nuclear gradient of the one-electron energy (one_electron_grad_kernel)
  const int* atom;     // per shell: atom index
  const double* D;     // density, nbf x nbf
  const double* W;     // energy-weighted density (factor 2 convention), nbf x nbf
  double* grad;        // n_atoms x 3, added to
  int gsmem;           // accumulate per block in shared memory (3 * n_atoms doubles)
};

// Host launchers (eri_aux.cu, onee.cu)
cudaError_t launch_jk(int X, int Y, const JKArgs& a, cudaStream_t st);
cudaError_t launch_store(int X, int Y, const StoreArgs& a, cudaStream_t st);
cudaError_t launch_grad(int X, int Y, const GradArgs& a, cudaStream_t st);
cudaError_t launch_schwarz(int X, ShellPair* pairs, const PrimPair* pp, const int* list, int n,
                           double thr, cudaStream_t st);
// Packed per-molecule matrices: molecule m owns elements [base[m], base[m+1])
// as an n[m] x n[m] row-major block; its basis functions start at bf0[m] in
// the global angular-factor array.
struct Packing {
  const long long* base;  // nmol + 1 offsets (device)
  const int* n;           // nmol (device)
  const int* bf0;         // nmol (device)
  int nmol;
  long long total;
};
cudaError_t launch_scale_density(const double* D, const double* ang, const Packing& P, double* Ds, cudaStream_t st);
cudaError_t launch_symmetrize(const double* X, const double* ang, const Packing& P, double* out, cudaStream_t st);
cudaError_t launch_fock(const double* H, const double* Jt, const double* Kt, const double* ang, const Packing& P,
                        double kscale, double* F, cudaStream_t st);
cudaError_t launch_boys_batch(int m, int n, const double* T, double* F, cudaStream_t st);
cudaError_t launch_rys_batch(int nr, int n, const double* T, double* R, double* W, cudaStream_t st);
cudaError_t launch_one_electron(const OneEArgs& a, cudaStream_t st);
cudaError_t launch_one_electron_grad(const OneEArgs& a, cudaStream_t st);
// max |D| per shell block of every molecule (layout of Mixed::dmax); D packed
cudaError_t launch_shell_dmax(const double* D, const Packing& P, const int* shell_off, const int* shell_l,
                              const Mixed& mx, long long total, double* dmax, cudaStream_t st);
// FP32 masks of the mixed form for every task (GRAD: density bound squared)
cudaError_t launch_precision_masks(const ShellPair* pairs, const int* ket_list, const QuartetTask* tasks,
                                   int ntasks, const Mixed& mx, bool grad, unsigned* mask, cudaStream_t st);
cudaError_t launch_count_prim_quartets(const ShellPair* pairs, const PrimPair* pp, const int* ket_list,
                                       const QuartetTask* tasks, int ntasks, double thr,
                                       unsigned long long* out, cudaStream_t st);
// FMA-throughput probe: which = 0 FP64, 1 FP32; returns flops done and device ms
cudaError_t launch_fma_peak(int which, double* flops, float* ms);

}  // namespace iqcp
