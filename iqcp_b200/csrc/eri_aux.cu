// Auxiliary kernels of the ERI engine: Schwarz bounds, density/J/K scaling
// and symmetrisation, Fock assembly, batched Boys/Rys evaluation, and the
// class dispatch of the quartet kernels (instantiated in eri_inst_*.cu).
#include "eri_templates.cuh"

namespace iqcp {

// ---------------------------------------------------------------------------
// Element-wise helpers
__global__ void scale_density_kernel(const double* __restrict__ D, const double* __restrict__ ang,
                                     int n, double* __restrict__ Ds) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)n * n) return;
  const int i = int(idx / n), j = int(idx % n);
  Ds[idx] = ang[i] * D[idx] * ang[j];
}

// out = ang_i ang_j (X_ij + X_ji)
__global__ void symmetrize_kernel(const double* __restrict__ X, const double* __restrict__ ang,
                                  int n, double* __restrict__ out) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)n * n) return;
  const int i = int(idx / n), j = int(idx % n);
  out[idx] = ang[i] * ang[j] * (X[idx] + X[(long long)j * n + i]);
}

// F = H + ang(Jt+Jt^T)ang - 0.5 k ang(Kt+Kt^T)ang
__global__ void fock_kernel(const double* __restrict__ H, const double* __restrict__ Jt,
                            const double* __restrict__ Kt, const double* __restrict__ ang, int n,
                            double kscale, double* __restrict__ F) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)n * n) return;
  const int i = int(idx / n), j = int(idx % n);
  const long long t = (long long)j * n + i;
  const double s = ang[i] * ang[j];
  double v = s * (Jt[idx] + Jt[t]);
  if (Kt) v -= 0.5 * kscale * s * (Kt[idx] + Kt[t]);
  F[idx] = H[idx] + v;
}

__global__ void boys_batch_kernel(int m, int n, const double* __restrict__ T, double* __restrict__ F) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double f[32];
  boys_all_dev(m, T[i], f);
  for (int k = 0; k <= m; ++k) F[(long long)i * (m + 1) + k] = f[k];
}

__global__ void rys_batch_kernel(int nr, int n, const double* __restrict__ T, double* __restrict__ R,
                                 double* __restrict__ W) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double r[RYS_TAB_MAXN], w[RYS_TAB_MAXN];
  rys_rule_n(nr, T[i], r, w);
  for (int k = 0; k < nr; ++k) {
    R[(long long)i * nr + k] = r[k];
    W[(long long)i * nr + k] = w[k];
  }
}

// ---------------------------------------------------------------------------
// Host launchers
cudaError_t launch_schwarz(int X, ShellPair* pairs, const PrimPair* pp, const int* list, int n,
                           double thr, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const int blocks = (n + 127) / 128;
  switch (X) {
    case 0: schwarz_kernel<0, 0><<<blocks, 128, 0, st>>>(pairs, pp, list, n, thr); break;
    case 1: schwarz_kernel<1, 0><<<blocks, 128, 0, st>>>(pairs, pp, list, n, thr); break;
    case 2: schwarz_kernel<1, 1><<<blocks, 128, 0, st>>>(pairs, pp, list, n, thr); break;
    case 3: schwarz_kernel<2, 0><<<blocks, 128, 0, st>>>(pairs, pp, list, n, thr); break;
    case 4: schwarz_kernel<2, 1><<<blocks, 128, 0, st>>>(pairs, pp, list, n, thr); break;
    case 5: schwarz_kernel<2, 2><<<blocks, 128, 0, st>>>(pairs, pp, list, n, thr); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

static inline int nblk(long long n, int b) { return int((n + b - 1) / b); }

cudaError_t launch_scale_density(const double* D, const double* ang, int n, double* Ds, cudaStream_t st) {
  scale_density_kernel<<<nblk((long long)n * n, 256), 256, 0, st>>>(D, ang, n, Ds);
  return cudaGetLastError();
}
cudaError_t launch_symmetrize(const double* X, const double* ang, int n, double* out, cudaStream_t st) {
  symmetrize_kernel<<<nblk((long long)n * n, 256), 256, 0, st>>>(X, ang, n, out);
  return cudaGetLastError();
}
cudaError_t launch_fock(const double* H, const double* Jt, const double* Kt, const double* ang, int n,
                        double kscale, double* F, cudaStream_t st) {
  fock_kernel<<<nblk((long long)n * n, 256), 256, 0, st>>>(H, Jt, Kt, ang, n, kscale, F);
  return cudaGetLastError();
}
cudaError_t launch_boys_batch(int m, int n, const double* T, double* F, cudaStream_t st) {
  boys_batch_kernel<<<nblk(n, 128), 128, 0, st>>>(m, n, T, F);
  return cudaGetLastError();
}
cudaError_t launch_rys_batch(int nr, int n, const double* T, double* R, double* W, cudaStream_t st) {
  rys_batch_kernel<<<nblk(n, 128), 128, 0, st>>>(nr, n, T, R, W);
  return cudaGetLastError();
}


#define IQCP_DECL_BRA(NAME, ARGS)                                                \
  extern template cudaError_t NAME<0, 0>(int, const ARGS&, cudaStream_t);        \
  extern template cudaError_t NAME<1, 0>(int, const ARGS&, cudaStream_t);        \
  extern template cudaError_t NAME<1, 1>(int, const ARGS&, cudaStream_t);        \
  extern template cudaError_t NAME<2, 0>(int, const ARGS&, cudaStream_t);        \
  extern template cudaError_t NAME<2, 1>(int, const ARGS&, cudaStream_t);        \
  extern template cudaError_t NAME<2, 2>(int, const ARGS&, cudaStream_t);
IQCP_DECL_BRA(launch_jk_bra, JKArgs)
IQCP_DECL_BRA(launch_store_bra, StoreArgs)
IQCP_DECL_BRA(launch_grad_bra, GradArgs)

#define IQCP_BRA_DISPATCH(NAME)                      \
  switch (X) {                                       \
    case 0: return NAME<0, 0>(Y, a, st);             \
    case 1: return NAME<1, 0>(Y, a, st);             \
    case 2: return NAME<1, 1>(Y, a, st);             \
    case 3: return NAME<2, 0>(Y, a, st);             \
    case 4: return NAME<2, 1>(Y, a, st);             \
    case 5: return NAME<2, 2>(Y, a, st);             \
    default: return cudaErrorInvalidValue;           \
  }

cudaError_t launch_jk(int X, int Y, const JKArgs& a, cudaStream_t st) {
  if (a.ntasks == 0) return cudaSuccess;
  if (Y > X) return cudaErrorInvalidValue;
  IQCP_BRA_DISPATCH(launch_jk_bra)
}
cudaError_t launch_store(int X, int Y, const StoreArgs& a, cudaStream_t st) {
  if (a.ntasks == 0) return cudaSuccess;
  if (Y > X) return cudaErrorInvalidValue;
  IQCP_BRA_DISPATCH(launch_store_bra)
}
cudaError_t launch_grad(int X, int Y, const GradArgs& a, cudaStream_t st) {
  if (a.ntasks == 0) return cudaSuccess;
  if (Y > X) return cudaErrorInvalidValue;
  IQCP_BRA_DISPATCH(launch_grad_bra)
}

}  // namespace iqcp
