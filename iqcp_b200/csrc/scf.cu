// Batched restricted Hartree-Fock on the device, one CUDA graph per iteration.
//
// The caller side of the Fock build for many geometries at once: the reference
// runs rhf_scf (crates/qc-core/src/scf/mod.rs:1363-1586) once per geometry
// inside its optimiser and scan loops (optimizer/mod.rs:274-320).  Here every
// geometry of a (batched) context iterates together, and one iteration is one
// replay of a captured CUDA graph:
//
//   1. F = H + J - K/2 of every geometry: iqcp_fock_device on the packed batch;
//   2. E = 1/2 Tr D (H + F) + E_nuc (scf/mod.rs:898);
//   3. Pulay DIIS (scf/mod.rs:1116-1327) on the AO commutator F D S - S D F
//      (scf/mod.rs:990), with a ring buffer of diis_size Fock matrices whose
//      slot and fill count live on the device;
//   4. the new density without an eigensolver: canonical purification
//      (Palser and Manolopoulos, Phys. Rev. B 58, 12704 (1998)) of
//      F' = X^T F X, D = 2 X P X^T.  For a closed shell with a HOMO-LUMO gap, P
//      converges to the projector on the n_occ lowest eigenvectors of F' -- the
//      aufbau density the reference takes from sorted_eigen (scf/mod.rs:743)
//      and D = 2 C_occ C_occ^T (:780).
//
// Every dense step is a batched FP64 matrix product over the packed n_m x n_m
// blocks (gemm_packed_kernel), so nothing in the iteration needs the host; the
// host reads back the per-geometry energy change, density change and DIIS
// error after each replay to test convergence (scf/mod.rs:1508-1520).  Set-up:
// X = S^-1/2 (scf/mod.rs:709) by the coupled Newton-Schulz iteration (matrix
// products only), and the core-Hamiltonian guess (:1379-1389) by purifying
// X^T H X.  At convergence W = 1/2 D F D equals the energy-weighted density
// 2 sum_occ e_i C_i C_i^T (scf/gradient.rs:101-130), so the nuclear gradient
// of every geometry follows from iqcp_one_electron_grad_device and
// iqcp_eri_grad_device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/iqcp.h"
#include "internal.h"

namespace iqcp {
namespace {

constexpr int kMaxDiis = 16;

// ---------------------------------------------------------------------------
// Batched FP64 matrix product over packed blocks:
//   C_m = alpha op(A_m) op(B_m) + beta C_m   for every molecule m,
// op(X) = X or X^T; 64 x 64 output tile per block, 4 x 4 per thread, k in
// chunks of 16 staged in shared memory.
constexpr int GT = 64, GK = 16;

// Molecules whose flag in `active` is 0 (converged geometries of the batched
// SCF) are skipped by every per-molecule kernel below; active may be null.
__device__ __forceinline__ bool frozen(const int* __restrict__ active, int m) {
  return active != nullptr && active[m] == 0;
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(256) gemm_packed_kernel(const long long* __restrict__ base,
                                                          const int* __restrict__ nm, const int* __restrict__ active,
                                                          const double* __restrict__ A,
                                                          const double* __restrict__ B, double* __restrict__ C,
                                                          double alpha, double beta) {
  const int m = blockIdx.z;
  const int n = nm[m];
  const int r0 = blockIdx.y * GT, c0 = blockIdx.x * GT;
  if (r0 >= n || c0 >= n || frozen(active, m)) return;
  const long long o = base[m];
  const double* Am = A + o;
  const double* Bm = B + o;
  double* Cm = C + o;
  __shared__ double As[GK][GT + 1];  // As[k][i] = op(A)(r0 + i, k0 + k)
  __shared__ double Bs[GK][GT + 1];  // Bs[k][j] = op(B)(k0 + k, c0 + j)
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4];
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) acc[u][v] = 0.0;
  for (int k0 = 0; k0 < n; k0 += GK) {
    for (int e = threadIdx.x; e < GT * GK; e += 256) {
      // consecutive threads read consecutive addresses of the row-major blocks
      const int i = TA ? e % GT : e / GK, ka = TA ? e / GT : e % GK;
      const int r = r0 + i, kk = k0 + ka;
      As[ka][i] = (r < n && kk < n) ? (TA ? Am[(long long)kk * n + r] : Am[(long long)r * n + kk]) : 0.0;
      const int j = TB ? e / GK : e % GT, kb = TB ? e % GK : e / GT;
      const int c = c0 + j, kr = k0 + kb;
      Bs[kb][j] = (c < n && kr < n) ? (TB ? Bm[(long long)c * n + kr] : Bm[(long long)kr * n + c]) : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < GK; ++k) {
      double a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        a[u] = As[k][ty + 16 * u];
        b[u] = Bs[k][tx + 16 * u];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = fma(a[u], b[v], acc[u][v]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int r = r0 + ty + 16 * u, c = c0 + tx + 16 * v;
      if (r < n && c < n) {
        const long long idx = (long long)r * n + c;
        Cm[idx] = beta == 0.0 ? alpha * acc[u][v] : fma(beta, Cm[idx], alpha * acc[u][v]);
      }
    }
}

// Block-wide sum of v (blockDim.x = 256); every thread gets the result.
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int w = 0; w < 8; ++w) t += sh[w];
  __syncthreads();
  return t;
}

__device__ __forceinline__ double block_max(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = sh[0];
#pragma unroll
  for (int w = 1; w < 8; ++w) t = fmax(t, sh[w]);
  __syncthreads();
  return t;
}

// E_m = 1/2 sum D (H + F) + E_nuc_m; dE_m = E_m - E_m(previous).  One block per molecule.
__global__ void energy_kernel(const long long* __restrict__ base, const int* __restrict__ active,
                              const double* __restrict__ D, const double* __restrict__ H,
                              const double* __restrict__ F, const double* __restrict__ enuc, double* __restrict__ E,
                              double* __restrict__ dE) {
  __shared__ double sh[8];
  const int m = blockIdx.x;
  if (frozen(active, m)) return;
  double s = 0.0;
  for (long long i = base[m] + threadIdx.x; i < base[m + 1]; i += blockDim.x) s += D[i] * (H[i] + F[i]);
  s = block_sum(s, sh);
  if (threadIdx.x == 0) {
    const double e = 0.5 * s + enuc[m];
    dE[m] = e - E[m];
    E[m] = e;
  }
}

// out = T - T^T per molecule block (grid: chunks x molecules)
__global__ void antisym_kernel(const long long* __restrict__ base, const int* __restrict__ nm,
                               const int* __restrict__ active, const double* __restrict__ T,
                               double* __restrict__ out) {
  const int m = blockIdx.y, n = nm[m];
  if (frozen(active, m)) return;
  const long long o = base[m], nn = (long long)n * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn; e += (long long)gridDim.x * blockDim.x) {
    const int i = int(e / n), j = int(e - (long long)i * n);
    out[o + e] = T[o + e] - T[o + (long long)j * n + i];
  }
}

// out_m = max |X| over molecule m's block
__global__ void maxabs_kernel(const long long* __restrict__ base, const double* __restrict__ X,
                              double* __restrict__ out) {
  __shared__ double sh[8];
  const int m = blockIdx.x;
  double v = 0.0;
  for (long long i = base[m] + threadIdx.x; i < base[m + 1]; i += blockDim.x) v = fmax(v, fabs(X[i]));
  v = block_max(v, sh);
  if (threadIdx.x == 0) out[m] = v;
}

// rms difference sqrt(sum (A - B)^2 / n^2) per molecule; then B = A
__global__ void rmsdiff_copy_kernel(const long long* __restrict__ base, const int* __restrict__ active,
                                    const double* __restrict__ A, double* __restrict__ B, double* __restrict__ out) {
  __shared__ double sh[8];
  const int m = blockIdx.x;
  if (frozen(active, m)) return;
  double s = 0.0;
  for (long long i = base[m] + threadIdx.x; i < base[m + 1]; i += blockDim.x) {
    const double d = A[i] - B[i];
    s += d * d;
    B[i] = A[i];
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) out[m] = sqrt(s / double(base[m + 1] - base[m]));
}

// DIIS ring buffer: store F and the error of this iteration at the current slot
__global__ void diis_store_kernel(long long total, const int* __restrict__ slot, const double* __restrict__ F,
                                  const double* __restrict__ err, double* __restrict__ Fbuf,
                                  double* __restrict__ Ebuf) {
  const long long off = (long long)(*slot) * total;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    Fbuf[off + i] = F[i];
    Ebuf[off + i] = err[i];
  }
}

// Bm[m][slot][l] = Bm[m][l][slot] = <e_slot, e_l> (grid: molecules x K)
__global__ void diis_overlap_kernel(const long long* __restrict__ base, long long total, int K,
                                    const int* __restrict__ slot, const double* __restrict__ Ebuf,
                                    double* __restrict__ Bm) {
  __shared__ double sh[8];
  const int m = blockIdx.x, l = blockIdx.y, s0 = *slot;
  const double* es = Ebuf + (long long)s0 * total;
  const double* el = Ebuf + (long long)l * total;
  double v = 0.0;
  for (long long i = base[m] + threadIdx.x; i < base[m + 1]; i += blockDim.x) v += es[i] * el[i];
  v = block_sum(v, sh);
  if (threadIdx.x == 0) {
    Bm[((long long)m * K + s0) * K + l] = v;
    Bm[((long long)m * K + l) * K + s0] = v;
  }
}

// Coefficients c (sum 1) minimising |sum c_k e_k|^2 over the filled slots:
// c proportional to B^-1 1 on the filled block (the Lagrange form of
// scf/mod.rs:1116-1327), B scaled by its largest diagonal, unfilled slots
// decoupled, 1e-14 on the diagonal.  One thread per molecule, Gaussian
// elimination.  Also advances nothing: the ring position is updated by
// diis_advance_kernel after the extrapolation.
__global__ void diis_solve_kernel(int nmol, int K, const int* __restrict__ count, const double* __restrict__ Bm,
                                  double* __restrict__ coef) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nmol) return;
  const int filled = min(*count + 1, K);
  double A[kMaxDiis][kMaxDiis], x[kMaxDiis];
  const double* B = Bm + (long long)m * K * K;
  double scale = 1e-300;
  for (int k = 0; k < filled; ++k) scale = fmax(scale, B[k * K + k]);
  for (int k = 0; k < K; ++k) {
    for (int l = 0; l < K; ++l) A[k][l] = (k < filled && l < filled) ? B[k * K + l] / scale : 0.0;
    if (k >= filled) A[k][k] = 1.0;
    A[k][k] += 1e-14;
    x[k] = k < filled ? 1.0 : 0.0;
  }
  for (int k = 0; k < K; ++k) {
    const double piv = A[k][k];
    for (int i = k + 1; i < K; ++i) {
      const double f = A[i][k] / piv;
      for (int j = k; j < K; ++j) A[i][j] -= f * A[k][j];
      x[i] -= f * x[k];
    }
  }
  for (int k = K - 1; k >= 0; --k) {
    double s = x[k];
    for (int j = k + 1; j < K; ++j) s -= A[k][j] * x[j];
    x[k] = s / A[k][k];
  }
  double sum = 0.0;
  for (int k = 0; k < K; ++k) sum += x[k];
  for (int k = 0; k < K; ++k) coef[(long long)m * K + k] = x[k] / sum;
}

// Fx = sum_k c_k Fbuf[k] per molecule block (grid: chunks x molecules)
__global__ void diis_extrapolate_kernel(const long long* __restrict__ base, const int* __restrict__ active,
                                        long long total, int K, const double* __restrict__ coef,
                                        const double* __restrict__ Fbuf, double* __restrict__ Fx) {
  const int m = blockIdx.y;
  if (frozen(active, m)) return;
  const long long o = base[m], nn = base[m + 1] - o;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn; e += (long long)gridDim.x * blockDim.x) {
    double v = 0.0;
    for (int k = 0; k < K; ++k) v = fma(coef[(long long)m * K + k], Fbuf[(long long)k * total + o + e], v);
    Fx[o + e] = v;
  }
}

__global__ void diis_advance_kernel(int K, int* slot, int* count) {
  *slot = (*slot + 1) % K;
  *count = min(*count + 1, K);
}

// Canonical purification, start: per molecule the Gershgorin bounds of F',
// mu = Tr F' / n, lambda = min(ne / (emax - mu), (n - ne) / (mu - emin));
// P0 = lambda/n (mu I - F') + ne/n I.  One block per molecule.
__global__ void purify_start_kernel(const long long* __restrict__ base, const int* __restrict__ nm,
                                    const int* __restrict__ active, const int* __restrict__ nocc,
                                    const double* __restrict__ Fp, double* __restrict__ P) {
  __shared__ double sh[8];
  __shared__ double par[2];
  const int m = blockIdx.x, n = nm[m];
  if (frozen(active, m)) return;
  const double* F = Fp + base[m];
  double lo = 1e300, hi = -1e300, tr = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double r = 0.0;
    for (int j = 0; j < n; ++j) r += fabs(F[(long long)i * n + j]);
    const double d = F[(long long)i * n + i];
    r -= fabs(d);
    lo = fmin(lo, d - r);
    hi = fmax(hi, d + r);
    tr += d;
  }
  tr = block_sum(tr, sh);
  hi = block_max(hi, sh);
  lo = -block_max(-lo, sh);
  if (threadIdx.x == 0) {
    const double mu = tr / n, ne = nocc[m];
    const double lam = fmin(ne / fmax(hi - mu, 1e-30), (n - ne) / fmax(mu - lo, 1e-30));
    par[0] = lam / n;
    par[1] = mu;
  }
  __syncthreads();
  const double a = par[0], mu = par[1], b = double(nocc[m]) / n;
  for (long long e = threadIdx.x; e < (long long)n * n; e += blockDim.x) {
    const int i = int(e / n), j = int(e - (long long)i * n);
    P[base[m] + e] = a * ((i == j ? mu : 0.0) - F[e]) + (i == j ? b : 0.0);
  }
}

// Canonical purification, traces of one step: tr[2m] = Tr(P - P2),
// tr[2m+1] = Tr(P2 - P3).  One block per molecule.
__global__ void purify_trace_kernel(const long long* __restrict__ base, const int* __restrict__ nm,
                                    const int* __restrict__ active, const double* __restrict__ P,
                                    const double* __restrict__ P2, const double* __restrict__ P3,
                                    double* __restrict__ tr) {
  __shared__ double sh[8];
  const int m = blockIdx.x, n = nm[m];
  if (frozen(active, m)) return;
  const long long o = base[m];
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const long long d = o + (long long)i * n + i;
    a += P[d] - P2[d];
    b += P2[d] - P3[d];
  }
  a = block_sum(a, sh);
  b = block_sum(b, sh);
  if (threadIdx.x == 0) {
    tr[2 * m] = a;
    tr[2 * m + 1] = b;
  }
}

// Canonical purification, update: c = t2 / t1; P <- ((1 + c) P2 - P3) / c for
// c >= 1/2, else ((1 - 2c) P + (1 + c) P2 - P3) / (1 - c).  Once P is
// idempotent to rounding t1 vanishes and the McWeeny step (c = 1/2) is taken.
// Grid: chunks x molecules.
__global__ void purify_update_kernel(const long long* __restrict__ base, const int* __restrict__ active,
                                     const double* __restrict__ tr, double* __restrict__ P,
                                     const double* __restrict__ P2, const double* __restrict__ P3) {
  const int m = blockIdx.y;
  if (frozen(active, m)) return;
  const long long o = base[m], nn = base[m + 1] - o;
  const double t1 = tr[2 * m], t2 = tr[2 * m + 1];
  const double c = fabs(t1) < 1e-13 ? 0.5 : t2 / t1;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn; e += (long long)gridDim.x * blockDim.x) {
    const long long i = o + e;
    P[i] = c >= 0.5 ? ((1.0 + c) * P2[i] - P3[i]) / fmax(c, 1e-30)
                    : ((1.0 - 2.0 * c) * P[i] + (1.0 + c) * P2[i] - P3[i]) / fmax(1.0 - c, 1e-30);
  }
}

// 3 I - X per molecule (grid: chunks x molecules)
__global__ void three_minus_kernel(const long long* __restrict__ base, const int* __restrict__ nm,
                                   const double* __restrict__ X, double* __restrict__ out) {
  const int m = blockIdx.y, n = nm[m];
  const long long o = base[m], nn = (long long)n * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn; e += (long long)gridDim.x * blockDim.x) {
    const int i = int(e / n), j = int(e - (long long)i * n);
    out[o + e] = (i == j ? 3.0 : 0.0) - X[o + e];
  }
}

// Newton-Schulz start: s_m = largest absolute row sum of S (>= its largest
// eigenvalue); Y = S / s, Z = I; scale[m] = s.  One block per molecule.
__global__ void ns_start_kernel(const long long* __restrict__ base, const int* __restrict__ nm,
                                const double* __restrict__ S, double* __restrict__ Y, double* __restrict__ Z,
                                double* __restrict__ scale) {
  __shared__ double sh[8];
  const int m = blockIdx.x, n = nm[m];
  const long long o = base[m];
  double r = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double t = 0.0;
    for (int j = 0; j < n; ++j) t += fabs(S[o + (long long)i * n + j]);
    r = fmax(r, t);
  }
  const double s = block_max(r, sh);
  for (long long e = threadIdx.x; e < (long long)n * n; e += blockDim.x) {
    const int i = int(e / n), j = int(e - (long long)i * n);
    Y[o + e] = S[o + e] / s;
    Z[o + e] = i == j ? 1.0 : 0.0;
  }
  if (threadIdx.x == 0) scale[m] = s;
}

// X = Z / sqrt(s) per molecule; err_m = max |Z Y - I| (from ZY)
__global__ void ns_finish_kernel(const long long* __restrict__ base, const int* __restrict__ nm,
                                 const double* __restrict__ Z, const double* __restrict__ scale,
                                 double* __restrict__ X) {
  const int m = blockIdx.y, n = nm[m];
  const long long o = base[m], nn = (long long)n * n;
  const double f = 1.0 / sqrt(scale[m]);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn; e += (long long)gridDim.x * blockDim.x)
    X[o + e] = Z[o + e] * f;
}

__global__ void identity_error_kernel(const long long* __restrict__ base, const int* __restrict__ nm,
                                      const double* __restrict__ A, double* __restrict__ out) {
  __shared__ double sh[8];
  const int m = blockIdx.x, n = nm[m];
  const long long o = base[m];
  double v = 0.0;
  for (long long e = threadIdx.x; e < (long long)n * n; e += blockDim.x) {
    const int i = int(e / n), j = int(e - (long long)i * n);
    v = fmax(v, fabs(A[o + e] - (i == j ? 1.0 : 0.0)));
  }
  v = block_max(v, sh);
  if (threadIdx.x == 0) out[m] = v;
}

}  // namespace
}  // namespace iqcp

// ---------------------------------------------------------------------------
// Host driver
namespace iqcp {
namespace {

struct ScfBuffers {
  std::vector<void*> owned;
  ~ScfBuffers() {
    for (void* p : owned) cudaFree(p);
  }
  template <typename T>
  cudaError_t get(T** p, long long n) {
    *p = nullptr;
    const cudaError_t e = cudaMalloc(p, sizeof(T) * (size_t)std::max(n, 1LL));
    if (e == cudaSuccess) owned.push_back(*p);
    return e;
  }
};

struct ScfRun {
  iqcp_ctx* ctx = nullptr;
  cudaStream_t st = nullptr;
  int nmol = 0, nmax = 0, K = 8, purify_iters = 64;
  long long total = 0;
  const long long* base = nullptr;  // device, n_mol + 1
  const int* nm = nullptr;          // device, n_mol
  double *S, *H, *X, *D, *F, *Fx, *P, *P2, *P3, *T1, *T2, *Dn, *Fbuf, *Ebuf;
  double *Bm, *coef, *enuc, *E, *dE, *dD, *err, *scale, *tr;
  int *nocc, *slot, *count;
  int* active = nullptr;  // per molecule: 1 while iterating (null during set-up and the final gradient)

  dim3 elem_grid() const {
    const long long nn = (long long)nmax * nmax;
    return dim3((unsigned)std::min<long long>((nn + 2047) / 2048, 256), (unsigned)nmol);
  }
  cudaError_t gemm(bool ta, bool tb, const double* A, const double* B, double* C, double alpha, double beta) const {
    const int t = (nmax + GT - 1) / GT;
    const dim3 grid(t, t, nmol);
    if (!ta && !tb) gemm_packed_kernel<false, false><<<grid, 256, 0, st>>>(base, nm, active, A, B, C, alpha, beta);
    else if (ta && !tb) gemm_packed_kernel<true, false><<<grid, 256, 0, st>>>(base, nm, active, A, B, C, alpha, beta);
    else if (!ta && tb) gemm_packed_kernel<false, true><<<grid, 256, 0, st>>>(base, nm, active, A, B, C, alpha, beta);
    else gemm_packed_kernel<true, true><<<grid, 256, 0, st>>>(base, nm, active, A, B, C, alpha, beta);
    return cudaGetLastError();
  }
  // Dout = 2 X P X^T with P the purified projector of Fp (Fp is left intact);
  // iters purification steps (default purify_iters)
  cudaError_t purify_density(const double* Fp, double* Dout, int iters = 0) const {
    if (iters <= 0) iters = purify_iters;
    purify_start_kernel<<<nmol, 256, 0, st>>>(base, nm, active, nocc, Fp, P);
    cudaError_t e = cudaGetLastError();
    for (int it = 0; it < iters && e == cudaSuccess; ++it) {
      if ((e = gemm(false, false, P, P, P2, 1.0, 0.0)) != cudaSuccess) break;
      if ((e = gemm(false, false, P2, P, P3, 1.0, 0.0)) != cudaSuccess) break;
      purify_trace_kernel<<<nmol, 256, 0, st>>>(base, nm, active, P, P2, P3, tr);
      purify_update_kernel<<<elem_grid(), 256, 0, st>>>(base, active, tr, P, P2, P3);
      e = cudaGetLastError();
    }
    if (e != cudaSuccess) return e;
    if ((e = gemm(false, false, X, P, T1, 1.0, 0.0)) != cudaSuccess) return e;
    return gemm(false, true, T1, X, Dout, 2.0, 0.0);
  }
  // One SCF iteration of every geometry, enqueued on st (capturable)
  int step() {
    int rc = iqcp_fock_device(ctx, H, D, 1.0, F);
    if (rc) return rc;
    energy_kernel<<<nmol, 256, 0, st>>>(base, active, D, H, F, enuc, E, dE);
    cudaError_t e = cudaGetLastError();
    // DIIS error: the AO commutator F D S - S D F (scf/mod.rs:990); (F D S)^T = S D F
    if (e == cudaSuccess) e = gemm(false, false, F, D, T1, 1.0, 0.0);
    if (e == cudaSuccess) e = gemm(false, false, T1, S, T2, 1.0, 0.0);
    if (e == cudaSuccess) {
      antisym_kernel<<<elem_grid(), 256, 0, st>>>(base, nm, active, T2, P2);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
      maxabs_kernel<<<nmol, 256, 0, st>>>(base, P2, err);
      diis_store_kernel<<<2048, 256, 0, st>>>(total, slot, F, P2, Fbuf, Ebuf);
      diis_overlap_kernel<<<dim3(nmol, K), 256, 0, st>>>(base, total, K, slot, Ebuf, Bm);
      diis_solve_kernel<<<(nmol + 63) / 64, 64, 0, st>>>(nmol, K, count, Bm, coef);
      diis_extrapolate_kernel<<<elem_grid(), 256, 0, st>>>(base, active, total, K, coef, Fbuf, Fx);
      diis_advance_kernel<<<1, 1, 0, st>>>(K, slot, count);
      e = cudaGetLastError();
    }
    // F' = X^T Fx X, purified into the new density
    if (e == cudaSuccess) e = gemm(true, false, X, Fx, T1, 1.0, 0.0);
    if (e == cudaSuccess) e = gemm(false, false, T1, X, T2, 1.0, 0.0);
    if (e == cudaSuccess) e = purify_density(T2, Dn);
    if (e == cudaSuccess) {
      rmsdiff_copy_kernel<<<nmol, 256, 0, st>>>(base, active, Dn, D, dD);
      e = cudaGetLastError();
    }
    if (e != cudaSuccess) return ctx_fail(ctx, IQCP_ERR_CUDA, cudaGetErrorString(e));
    return IQCP_OK;
  }
};

}  // namespace
}  // namespace iqcp

using namespace iqcp;

#define SCF_CK(call)                                                                             \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) {                                                                     \
      rc = ctx_fail(ctx, IQCP_ERR_CUDA, (std::string(#call) + ": " + cudaGetErrorString(e_)).c_str()); \
      goto done;                                                                                 \
    }                                                                                            \
  } while (0)

extern "C" {

void iqcp_scf_default_options(iqcp_scf_options* o) {
  o->e_tol = 1e-9;
  o->d_tol = 1e-7;
  o->err_tol = 1e-5;
  o->max_iter = 80;
  o->diis_size = 8;
  o->purify_iters = 64;
}

int iqcp_batch_scf(iqcp_ctx* ctx, const iqcp_scf_options* opts_in, const double* D0, double* energies,
                   int* converged, int* iterations, double* D_out, double* grad) {
  if (!ctx) return IQCP_ERR_ARG;
  iqcp_scf_options opts;
  if (opts_in) opts = *opts_in;
  else iqcp_scf_default_options(&opts);
  if (opts.diis_size < 1 || opts.diis_size > kMaxDiis || opts.max_iter < 0 || opts.purify_iters < 1)
    return ctx_fail(ctx, IQCP_ERR_ARG, "scf options out of range (diis_size 1..16, purify_iters >= 1)");
  const int nmol = ctx_n_mol(ctx);
  const std::vector<long long>& mb = ctx_mol_base(ctx);
  const std::vector<int>& mn = ctx_mol_nbf(ctx);
  const std::vector<int>& a0 = ctx_mol_atom0(ctx);
  const std::vector<int>& zs = ctx_atom_z(ctx);
  const std::vector<double>& xyz = ctx_atom_xyz(ctx);
  // closed shells, nuclear repulsion per molecule
  std::vector<int> h_nocc(nmol);
  std::vector<double> h_enuc(nmol, 0.0);
  for (int m = 0; m < nmol; ++m) {
    int ne = 0;
    for (int a = a0[m]; a < a0[m + 1]; ++a) {
      ne += zs[a];
      for (int b = a0[m]; b < a; ++b) {
        const double dx = xyz[3 * a] - xyz[3 * b], dy = xyz[3 * a + 1] - xyz[3 * b + 1],
                     dz = xyz[3 * a + 2] - xyz[3 * b + 2];
        h_enuc[m] += double(zs[a]) * zs[b] / std::sqrt(dx * dx + dy * dy + dz * dz);
      }
    }
    if (ne % 2) return ctx_fail(ctx, IQCP_ERR_ARG, "iqcp_batch_scf: open-shell molecule (odd electron count)");
    h_nocc[m] = ne / 2;
  }
  int rc = cudaSetDevice(ctx_device(ctx)) == cudaSuccess ? IQCP_OK : IQCP_ERR_CUDA;
  if (rc) return ctx_fail(ctx, rc, "cudaSetDevice");
  const cudaStream_t caller = ctx_stream(ctx);
  ScfBuffers buf;
  ScfRun r;
  cudaStream_t own = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<double> host(4 * (size_t)nmol);
  std::vector<double> hS, hH;
  const Packing& pk = ctx_packing(ctx);
  int it = 0;
  bool all_conv = false;
  std::vector<char> conv(nmol, 0);
  std::vector<int> h_active;
  r.ctx = ctx;
  r.nmol = nmol;
  r.K = opts.diis_size;
  r.purify_iters = opts.purify_iters;
  r.total = mb[nmol];
  r.nmax = *std::max_element(mn.begin(), mn.end());
  r.base = pk.base;
  r.nm = pk.n;
  // work on a private stream: capture needs one, and the caller's may be the legacy default stream
  SCF_CK(cudaStreamSynchronize(caller));
  SCF_CK(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
  r.st = own;
  iqcp_set_stream(ctx, own);
  for (double** p : {&r.S, &r.H, &r.X, &r.D, &r.F, &r.Fx, &r.P, &r.P2, &r.P3, &r.T1, &r.T2, &r.Dn})
    SCF_CK(buf.get(p, r.total));
  SCF_CK(buf.get(&r.Fbuf, r.total * r.K));
  SCF_CK(buf.get(&r.Ebuf, r.total * r.K));
  SCF_CK(buf.get(&r.Bm, (long long)nmol * r.K * r.K));
  SCF_CK(buf.get(&r.coef, (long long)nmol * r.K));
  for (double** p : {&r.enuc, &r.E, &r.dE, &r.dD, &r.err, &r.scale}) SCF_CK(buf.get(p, nmol));
  SCF_CK(buf.get(&r.tr, 2LL * nmol));
  SCF_CK(buf.get(&r.nocc, nmol));
  SCF_CK(buf.get(&r.slot, 1));
  SCF_CK(buf.get(&r.count, 1));
  int* d_active;
  SCF_CK(buf.get(&d_active, nmol));
  SCF_CK(cudaMemsetAsync(r.Ebuf, 0, sizeof(double) * r.total * r.K, own));
  SCF_CK(cudaMemsetAsync(r.Fbuf, 0, sizeof(double) * r.total * r.K, own));
  SCF_CK(cudaMemsetAsync(r.Bm, 0, sizeof(double) * nmol * r.K * r.K, own));
  SCF_CK(cudaMemsetAsync(r.E, 0, sizeof(double) * nmol, own));
  SCF_CK(cudaMemsetAsync(r.slot, 0, sizeof(int), own));
  SCF_CK(cudaMemsetAsync(r.count, 0, sizeof(int), own));
  SCF_CK(cudaMemcpyAsync(r.enuc, h_enuc.data(), sizeof(double) * nmol, cudaMemcpyHostToDevice, own));
  SCF_CK(cudaMemcpyAsync(r.nocc, h_nocc.data(), sizeof(int) * nmol, cudaMemcpyHostToDevice, own));
  // one-electron matrices (set-up, through the host)
  hS.resize(r.total);
  hH.resize(r.total);
  {
    std::vector<double> hT(r.total);
    rc = iqcp_one_electron(ctx, hS.data(), hT.data(), hH.data());
    if (rc) goto done;
    for (long long i = 0; i < r.total; ++i) hH[i] += hT[i];
  }
  SCF_CK(cudaMemcpyAsync(r.S, hS.data(), sizeof(double) * r.total, cudaMemcpyHostToDevice, own));
  SCF_CK(cudaMemcpyAsync(r.H, hH.data(), sizeof(double) * r.total, cudaMemcpyHostToDevice, own));
  // X = S^-1/2: coupled Newton-Schulz on Y = S/s, Z = I (Y -> (S/s)^1/2, Z -> (S/s)^-1/2)
  {
    double *Y = r.P, *Z = r.P2, *ZY = r.P3, *Tm = r.T1, *Yn = r.T2, *Zn = r.Dn;
    ns_start_kernel<<<nmol, 256, 0, own>>>(r.base, r.nm, r.S, Y, Z, r.scale);
    SCF_CK(cudaGetLastError());
    bool ok = false;
    for (int k = 0; k < 200 && !ok; ++k) {
      SCF_CK(r.gemm(false, false, Z, Y, ZY, 1.0, 0.0));
      if (k % 4 == 3) {
        identity_error_kernel<<<nmol, 256, 0, own>>>(r.base, r.nm, ZY, r.err);
        SCF_CK(cudaMemcpyAsync(host.data(), r.err, sizeof(double) * nmol, cudaMemcpyDeviceToHost, own));
        SCF_CK(cudaStreamSynchronize(own));
        ok = *std::max_element(host.begin(), host.begin() + nmol) < 1e-13;
        if (ok) break;
      }
      three_minus_kernel<<<r.elem_grid(), 256, 0, own>>>(r.base, r.nm, ZY, Tm);
      SCF_CK(cudaGetLastError());
      SCF_CK(r.gemm(false, false, Y, Tm, Yn, 0.5, 0.0));
      SCF_CK(r.gemm(false, false, Tm, Z, Zn, 0.5, 0.0));
      std::swap(Y, Yn);
      std::swap(Z, Zn);
    }
    if (!ok) {
      rc = ctx_fail(ctx, IQCP_ERR_NUMERIC, "iqcp_batch_scf: S^-1/2 did not converge (near-singular overlap)");
      goto done;
    }
    ns_finish_kernel<<<r.elem_grid(), 256, 0, own>>>(r.base, r.nm, Z, r.scale, r.X);
    SCF_CK(cudaGetLastError());
  }
  // starting density: the caller's, or the core-Hamiltonian guess (purified X^T H X)
  if (D0) {
    SCF_CK(cudaMemcpyAsync(r.D, D0, sizeof(double) * r.total, cudaMemcpyHostToDevice, own));
  } else {
    SCF_CK(r.gemm(true, false, r.X, r.H, r.T1, 1.0, 0.0));
    SCF_CK(r.gemm(false, false, r.T1, r.X, r.T2, 1.0, 0.0));
    // the core Hamiltonian's spectrum is wide next to its gap: more steps, once
    SCF_CK(r.purify_density(r.T2, r.D, 4 * opts.purify_iters));
  }
  // iterations: the first eagerly (sets kernel attributes), then graph replays.
  // A geometry that meets the thresholds stops iterating, as rhf_scf stops per
  // geometry: its flag turns 0 and every kernel of the iteration, the Fock
  // build's quartet kernels included, skips it from the next replay on.
  h_active.assign(nmol, 1);
  SCF_CK(cudaMemcpyAsync(d_active, h_active.data(), sizeof(int) * nmol, cudaMemcpyHostToDevice, own));
  r.active = d_active;
  ctx_set_mol_active(ctx, d_active);
  for (it = 1; it <= opts.max_iter; ++it) {
    if (it == 1) {
      rc = r.step();
      if (rc) goto done;
    } else {
      if (!exec) {
        SCF_CK(cudaStreamBeginCapture(own, cudaStreamCaptureModeThreadLocal));
        rc = r.step();
        cudaError_t ce = cudaStreamEndCapture(own, &graph);
        if (rc) goto done;
        SCF_CK(ce);
        SCF_CK(cudaGraphInstantiate(&exec, graph, 0));
      }
      SCF_CK(cudaGraphLaunch(exec, own));
    }
    SCF_CK(cudaMemcpyAsync(host.data(), r.dE, sizeof(double) * nmol, cudaMemcpyDeviceToHost, own));
    SCF_CK(cudaMemcpyAsync(host.data() + nmol, r.dD, sizeof(double) * nmol, cudaMemcpyDeviceToHost, own));
    SCF_CK(cudaMemcpyAsync(host.data() + 2 * nmol, r.err, sizeof(double) * nmol, cudaMemcpyDeviceToHost, own));
    SCF_CK(cudaStreamSynchronize(own));
    all_conv = true;
    bool frozen_now = false;
    for (int m = 0; m < nmol; ++m) {
      if (!h_active[m]) continue;  // converged earlier
      conv[m] = std::fabs(host[m]) < opts.e_tol && host[nmol + m] < opts.d_tol && host[2 * nmol + m] < opts.err_tol;
      all_conv = all_conv && conv[m];
      if (it > 2 && conv[m]) {
        h_active[m] = 0;
        frozen_now = true;
      }
    }
    if (it > 2 && all_conv) break;
    if (frozen_now)
      SCF_CK(cudaMemcpyAsync(d_active, h_active.data(), sizeof(int) * nmol, cudaMemcpyHostToDevice, own));
  }
  r.active = nullptr;
  ctx_set_mol_active(ctx, nullptr);
  if (it > opts.max_iter) it = opts.max_iter;
  if (iterations) *iterations = it;
  if (energies) SCF_CK(cudaMemcpyAsync(energies, r.E, sizeof(double) * nmol, cudaMemcpyDeviceToHost, own));
  if (D_out) SCF_CK(cudaMemcpyAsync(D_out, r.D, sizeof(double) * r.total, cudaMemcpyDeviceToHost, own));
  if (grad) {
    // W = 1/2 D F D at the final density, then the one- and two-electron parts
    double* g = nullptr;
    const int natoms = a0[nmol];
    SCF_CK(buf.get(&g, 3LL * natoms));
    rc = iqcp_fock_device(ctx, r.H, r.D, 1.0, r.F);
    if (rc) goto done;
    SCF_CK(r.gemm(false, false, r.D, r.F, r.T1, 1.0, 0.0));
    SCF_CK(r.gemm(false, false, r.T1, r.D, r.T2, 0.5, 0.0));
    SCF_CK(cudaMemsetAsync(g, 0, sizeof(double) * 3 * natoms, own));
    rc = iqcp_one_electron_grad_device(ctx, r.D, r.T2, g);
    if (rc) goto done;
    rc = iqcp_eri_grad_device(ctx, r.D, 1.0, g);
    if (rc) goto done;
    SCF_CK(cudaMemcpyAsync(grad, g, sizeof(double) * 3 * natoms, cudaMemcpyDeviceToHost, own));
  }
  SCF_CK(cudaStreamSynchronize(own));
  if (converged)
    for (int m = 0; m < nmol; ++m) converged[m] = opts.max_iter > 0 ? conv[m] : 0;
done:
  ctx_set_mol_active(ctx, nullptr);
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  if (own) cudaStreamSynchronize(own);
  iqcp_set_stream(ctx, caller);
  if (own) cudaStreamDestroy(own);
  return rc;
}

}  // extern "C"
