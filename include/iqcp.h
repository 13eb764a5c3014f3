/*
 * iqcp.h -- C ABI of libiqcp_gpu.so, the B200 (sm_100a) direct Fock-build and
 * two-electron nuclear-gradient engine for Cartesian Gaussian basis sets.
 *
 * The entry points replace, one for one, the reference's (ExaPsi/IQCP,
 * crates/qc-core) Rust functions on this path; each declaration names the
 * function it stands in for.  Plain pointers and sizes only.
 *
 * Conventions
 *  - Matrices are nbf x nbf, row-major, FP64.  All matrices on this path are
 *    symmetric, so row- and column-major (the reference's nalgebra DMatrix is
 *    column-major) hold the same elements.
 *  - The density carries the RHF factor 2 (D = 2 C_occ C_occ^T), as in
 *    scf/mod.rs:780-794.
 *  - Basis functions are Cartesian, shell by shell in the order given, with
 *    components ordered xx,xy,xz,yy,yz,zz for d (integrals/cartesian.rs:113).
 *    Every primitive x component carries coef * N(alpha, i, j, k)
 *    (integrals/overlap.rs:343); the caller passes the raw tabulated
 *    contraction coefficients.
 *  - Every function returns IQCP_OK (0) or a negative status; the message of
 *    the last failure on a context is available from iqcp_last_error().
 *  - Calls on one context are synchronous with respect to the host and not
 *    thread-safe; use one context per host thread.
 */
#ifndef IQCP_H_
#define IQCP_H_

#ifdef __cplusplus
extern "C" {
#endif

enum iqcp_status {
  IQCP_OK = 0,
  IQCP_ERR_ARG = -1,        /* invalid argument (sizes, unsupported L, NULL) */
  IQCP_ERR_CUDA = -2,       /* a CUDA runtime call failed */
  IQCP_ERR_NOMEM = -3,      /* device or host allocation failed */
  IQCP_ERR_NUMERIC = -4,    /* non-finite input or result */
  IQCP_ERR_NODEVICE = -5,   /* no usable sm_100 device */
  IQCP_ERR_BASIS = -6       /* unknown basis name or element */
};

enum iqcp_precision {
  IQCP_FP64 = 0,            /* all quadrature in FP64 */
  IQCP_MIXED = 1            /* FP32 quadrature for weak quartets, FP64 roots and accumulation */
};

/* A basis as qc-core's BasisSet holds it (basis/mod.rs:113-130). */
typedef struct iqcp_basis_desc {
  int n_shells;
  int n_atoms;
  const int* l;               /* [n_shells] angular momentum, 0..2 */
  const int* nprim;           /* [n_shells] primitives per shell */
  const int* atom_of_shell;   /* [n_shells] */
  const double* center;       /* [3*n_shells] bohr */
  const double* exps;         /* [sum nprim] exponents, shell by shell */
  const double* coefs;        /* [sum nprim] raw contraction coefficients */
  const double* atom_xyz;     /* [3*n_atoms] bohr */
  const int* z;               /* [n_atoms] atomic numbers */
} iqcp_basis_desc;

typedef struct iqcp_options {
  double schwarz_threshold;   /* 1e-12: eri/mod.rs:1258 SCHWARZ_THRESHOLD */
  double prim_threshold;      /* 1e-15: K_ij and K_ij*K_kl screens, eri/mod.rs:603,611 */
  int precision;              /* enum iqcp_precision */
  double mixed_cutoff;        /* MIXED: quartets with Q_ij*Q_kl*max|D| below this use FP32 */
  int device;                 /* CUDA device ordinal */
} iqcp_options;

typedef struct iqcp_ctx iqcp_ctx;

/* Default options (thresholds of the reference, FP64). */
void iqcp_default_options(iqcp_options* opts);

/*
 * Build a basis for atoms (bohr) from the built-in tables.
 * Replaces BasisSet::build (basis/mod.rs:164) with get_element_basis
 * (basis/builtin.rs:97).  Call once with the array pointers NULL to get the
 * counts, then again with arrays of those sizes.  Returns IQCP_ERR_BASIS for an
 * unknown basis name or an element outside H..Ar.
 */
int iqcp_basis_build(const char* basis_name, int n_atoms, const int* z, const double* xyz,
                     int* n_shells, int* n_prims, int* nbf, int* l, int* nprim,
                     int* atom_of_shell, double* center, double* exps, double* coefs);

/*
 * Create a context for one basis (geometry): uploads the basis, builds the
 * class-sorted shell-pair data and the Schwarz bounds on the device and the
 * screened quartet lists.  Stands in for the set-up half of eri_compressed
 * (integrals/eri/mod.rs:992-1030, compute_schwarz_bounds :1263).
 */
int iqcp_create(const iqcp_basis_desc* basis, const iqcp_options* opts, iqcp_ctx** out);
void iqcp_destroy(iqcp_ctx* ctx);

/*
 * One context for many molecules (or geometries) of uneven size: every
 * J/K, Fock, gradient and one-electron call then covers all of them with one
 * launch per angular-momentum class.  Matrices are packed: molecule m owns the
 * nbf[m] x nbf[m] row-major block at offset mat_offset[m]; gradient rows of
 * molecule m are atoms [atom_offset[m], atom_offset[m+1]).  The quartet lists
 * never pair shells of different molecules.  iqcp_batch_layout fills
 * mat_offset[n_mol+1], nbf[n_mol], atom_offset[n_mol+1] (any may be NULL) and
 * returns n_mol.  No counterpart in the reference, which loops over geometries
 * (optimizer/mod.rs:274-320).  iqcp_eri_compressed, iqcp_jk_device_noalloc and
 * the mixed form are single-geometry only.
 */
int iqcp_create_batch(int n_mol, const iqcp_basis_desc* bases, const iqcp_options* opts, iqcp_ctx** out);
int iqcp_batch_layout(const iqcp_ctx* ctx, long long* mat_offset, int* nbf, int* atom_offset);
const char* iqcp_last_error(const iqcp_ctx* ctx);
int iqcp_nbf(const iqcp_ctx* ctx);

/*
 * Switch the context between the FP64 form and the mixed form (quartets with
 * Q_ij*Q_kl*max|D| below mixed_cutoff run their quadrature in FP32; Rys roots
 * and weights, recurrence coefficients and all accumulation stay FP64).  max|D|
 * is the largest density element over the six shell blocks the quartet
 * digests with; gradients use its square (D x D weights).  Applies to J/K,
 * Fock and ERI-gradient calls, single or batched contexts.
 */
int iqcp_set_precision(iqcp_ctx* ctx, int precision, double mixed_cutoff);

/*
 * Run the context's work on this CUDA stream (cudaStream_t); NULL = the
 * context's own stream, which is created non-blocking (it does not order with
 * the legacy default stream).  A caller working on the legacy default stream
 * passes cudaStreamLegacy, not NULL.  Inside a J/K build or gradient the
 * class kernels also run on three side streams of the context, forked from
 * this stream by an event and joined back to it before the call's last
 * operation, so work queued on this stream before the call precedes all of
 * them and work queued after it follows all of them (in stream capture too).
 */
int iqcp_set_stream(iqcp_ctx* ctx, void* stream);

/*
 * Coulomb and exchange matrices from a density, host buffers.
 * J_mn = sum_ls D_ls (mn|ls),  K_mn = sum_ls D_ls (ml|ns).
 * Replaces build_jk / build_coulomb / build_exchange (dft/ks_scf.rs:1306,1342,1369).
 * K may be NULL (Coulomb only).
 */
int iqcp_jk(iqcp_ctx* ctx, const double* D, double* J, double* K);

/*
 * Fock matrix F = H + J - 1/2 * k_scale * K, host buffers.  k_scale = 1 is RHF
 * (build_fock, scf/mod.rs:825-881); k_scale = hf_frac is the hybrid KS form
 * (dft/ks_scf.rs:1795-1843, 1953-1960).
 */
int iqcp_fock(iqcp_ctx* ctx, const double* H, const double* D, double k_scale, double* F);

/*
 * Device-pointer forms of iqcp_jk / iqcp_fock for data resident in HBM.  They
 * enqueue their kernels on the context stream (iqcp_set_stream) and may return
 * before the outputs are written: order with them on that stream, or
 * synchronise it, before reading the outputs from another stream.  They
 * (and iqcp_eri_grad_device, iqcp_one_electron_grad_device) may be captured
 * into a CUDA graph on the context stream (iqcp_set_stream to the capturing
 * stream): while the stream captures they only enqueue work, and
 * iqcp_last_stats / iqcp_launch_profile are not updated.  Call each once
 * before capturing (the first call sets kernel attributes).
 */
int iqcp_jk_device(iqcp_ctx* ctx, const double* d_D, double* d_J, double* d_K);
int iqcp_fock_device(iqcp_ctx* ctx, const double* d_H, const double* d_D, double k_scale,
                     double* d_F);

/*
 * iqcp_jk_device without any device allocation: same inputs, outputs and
 * results as iqcp_jk_device in either precision (FP64 or MIXED, as set on the
 * context), but its scratch (scaled density, J/K accumulators) lives in a
 * fixed file-scope device array instead of context buffers.  No counterpart
 * in the reference.  For callers whose Fock-build loop may not call cudaMalloc
 * (all of HBM handed to their own pool, or no implicit device synchronisation
 * allowed); the context is created beforehand by iqcp_create.
 * Limit: nbf <= 512 (3*512*512 doubles, 6 MiB held on every GPU that loads the
 * library); larger bases and batched contexts return IQCP_ERR_ARG.  The first
 * call on a device looks up the array's address (cudaGetSymbolAddress) --
 * make it before any stream capture.  The call enqueues its work on the
 * context stream and returns without waiting for the GPU; iqcp_last_stats
 * then reports quartets and launches but 0 for device time and FP32 count.
 * All calls share the array: calls that overlap on the GPU race, so
 * serialise them.
 */
int iqcp_jk_device_noalloc(iqcp_ctx* ctx, const double* d_D, double* d_J, double* d_K);

/*
 * J and K of nset densities at once, each quartet evaluated once and
 * digested into every density: J_s, K_s of D_s for s < nset.  The matrices
 * of density s start at element s * P, P = nbf*nbf (or the packed size of a
 * batched context, see iqcp_batch_layout); each D_s must be symmetric.  This
 * is the J/K of the CPHF response densities: gen_vind_rhf / gen_vind_rhf_vo
 * (scf/cphf.rs:828-990) form dm1 = dm + dm^T per trial vector and build J, K
 * from it one density at a time.  FP64 quadrature whatever the context's
 * precision.  K may be NULL.  Host buffers, or device pointers for the
 * _device form (enqueued on the context stream, like iqcp_jk_device).
 */
int iqcp_jk_multi(iqcp_ctx* ctx, int nset, const double* D, double* J, double* K);
int iqcp_jk_multi_device(iqcp_ctx* ctx, int nset, const double* d_D, double* d_J, double* d_K);

/*
 * J and K in the real spherical-harmonic basis (single-geometry contexts):
 * D, J, K are nsph x nsph, nsph = iqcp_nbf_spherical(ctx) = sum over shells of
 * 2l + 1, functions shell by shell with m = -l..l (d: d-2, d-1, d0, d+1, d+2).
 * The reference's spherical path transforms each Cartesian ERI block with
 * EriSphericalTransform (integrals/spherical.rs:390-470, coefficients
 * CART2SPH_D :71) and digests the transformed ERIs; here J_sph =
 * C^T J_cart[C D C^T] C with the same coefficients (C[cart][sph]), which is
 * the same sum.  K may be NULL.
 */
int iqcp_nbf_spherical(iqcp_ctx* ctx);
int iqcp_jk_spherical(iqcp_ctx* ctx, const double* D, double* J, double* K);

/*
 * The four matrices of compute_fock_decomposition (scf/fock.rs:104-179), host
 * buffers: J, K, G = J - 1/2 k_scale K and F = H + G (k_scale = 1 for RHF).
 * Any output may be NULL; H may be NULL when F is.
 */
int iqcp_fock_decomposition(iqcp_ctx* ctx, const double* H, const double* D, double k_scale, double* J, double* K,
                            double* G, double* F);

/*
 * Two-electron part of the nuclear gradient, host buffers:
 * grad[3*atom + dir] += sum over unique quartets of w * d(ij|kl)/dR with
 * w = sum_perm [1/2 D_ij D_kl - 1/4 hf_frac D_ik D_jl].
 * Replaces eri_gradient_fused (scf/gradient.rs:1430-1566) with
 * compute_symmetry_weight (:1570-1640) and shell_eri_with_derivatives
 * (integrals/eri/mod.rs:2035-2548).
 */
int iqcp_eri_grad(iqcp_ctx* ctx, const double* D, double hf_frac, double* grad);
int iqcp_eri_grad_device(iqcp_ctx* ctx, const double* d_D, double hf_frac, double* d_grad);

/*
 * Batched RHF to self-consistency on the device: every geometry of the
 * context (batched or single) iterates together, one CUDA graph replay per
 * iteration (Fock build, energy, DIIS on FDS - SDF, density by
 * canonical purification of X^T F X), with X = S^-1/2 from a Newton-Schulz
 * iteration and the core-Hamiltonian guess unless D0 is given.  Replaces the
 * per-geometry rhf_scf loop (scf/mod.rs:1363-1586) of the optimiser and scan
 * callers (optimizer/mod.rs:274-320).  Converged when |dE| < e_tol, rms dD <
 * d_tol and max |DIIS error| < err_tol (scf/mod.rs:1508-1520).  Host buffers,
 * packed per geometry as in iqcp_create_batch: D0 (NULL: core guess),
 * energies[n_mol], converged[n_mol] (0/1), iterations, D_out (packed, may be
 * NULL) and grad (n_atoms x 3, overwritten with the RHF gradient at the final
 * density; may be NULL).  max_iter = 0 returns the starting density only.
 * Closed shells only.  Device scratch is allocated for the call and freed.
 */
typedef struct iqcp_scf_options {
  double e_tol;       /* 1e-9 Ha */
  double d_tol;       /* 1e-7, rms density change */
  double err_tol;     /* 1e-5, largest DIIS error element */
  int max_iter;       /* 80 */
  int diis_size;      /* 8 (1..16) */
  int purify_iters;   /* 64 canonical-purification steps per iteration */
} iqcp_scf_options;
void iqcp_scf_default_options(iqcp_scf_options* opts);
int iqcp_batch_scf(iqcp_ctx* ctx, const iqcp_scf_options* opts, const double* D0, double* energies,
                   int* converged, int* iterations, double* D_out, double* grad);

/*
 * SAD initial density of one geometry (build_sad_density, scf/sad.rs:698-760):
 * per element, a spherically averaged atomic RHF with fractional subshell
 * occupations (PySCF AtomSphAverageRHF; sad.rs:207-640), the atomic blocks
 * placed on the diagonal, zero between atoms.  D: nbf x nbf row-major (the
 * matrix is symmetric).  The atomic integrals come from one-atom contexts on
 * opts->device (NULL: default options).  Pack the densities of a batch in the
 * iqcp_create_batch layout to start iqcp_batch_scf from them (D0).
 */
int iqcp_sad_density(const iqcp_basis_desc* basis, const iqcp_options* opts, double* D);

/*
 * All unique ERIs in the reference's 8-fold compressed layout,
 * idx = P(P+1)/2 + Q, P = pair(i,j) >= Q = pair(k,l), pair(i,j) = i(i+1)/2 + j.
 * Replaces eri_compressed (integrals/eri/mod.rs:992-1070); out holds
 * n_pairs(n_pairs+1)/2 doubles, n_pairs = nbf(nbf+1)/2.  Small bases only.
 */
int iqcp_eri_compressed(iqcp_ctx* ctx, double* out, long long out_len);

/*
 * One-electron matrices over the context's basis, host buffers (any may be
 * NULL): overlap S (integrals/overlap.rs:647 overlap_matrix), kinetic T and
 * nuclear attraction V with H = T + V (integrals/hcore.rs:103 hcore_matrix,
 * nuclear.rs:68-305).
 */
int iqcp_one_electron(iqcp_ctx* ctx, double* S, double* T, double* V);

/*
 * Non-ERI part of the RHF nuclear gradient, added into grad (n_atoms x 3):
 * nuclear repulsion + sum_mn D_mn dH_mn/dR - sum_mn W_mn dS_mn/dR, with the
 * Hellmann-Feynman term of the nuclear attraction operator.  W is the
 * energy-weighted density 2 sum_occ e_i C_mi C_ni (the factor-2 convention of
 * scf/gradient.rs:116).  Replaces the overlap_derivative_matrix /
 * hcore_derivative_matrix contractions and the nuclear term of rhf_gradient
 * (scf/gradient.rs:188, 355, 900-990).  Host buffers, or device pointers for
 * the _device form (enqueued on the context stream).
 */
int iqcp_one_electron_grad(iqcp_ctx* ctx, const double* D, const double* W, double* grad);
int iqcp_one_electron_grad_device(iqcp_ctx* ctx, const double* d_D, const double* d_W, double* d_grad);

/*
 * Full RHF nuclear gradient (overwrites grad, n_atoms x 3): the one-electron
 * part above plus the two-electron part of iqcp_eri_grad with hf_frac = 1.
 * Replaces rhf_gradient (scf/gradient.rs:900-990), which takes C and the
 * orbital energies; the caller forms W from them.
 */
int iqcp_rhf_gradient(iqcp_ctx* ctx, const double* D, const double* W, double* grad);

/* Schwarz bounds Q[n_shells*n_shells] (compute_schwarz_bounds, eri/mod.rs:1263). */
int iqcp_schwarz(iqcp_ctx* ctx, double* Q);

/*
 * Batched Boys function F_0..F_m_max(T) and Rys roots (t^2) / weights on the
 * device, host buffers; the device forms of boys_eval_all (boys/mod.rs:327)
 * and rys_roots (rys/mod.rs:253).  F is [n][m_max+1], roots/weights [n][nroots].
 */
int iqcp_boys_batch(int m_max, int n, const double* T, double* F);
int iqcp_rys_batch(int nroots, int n, const double* T, double* roots, double* weights);

/*
 * Counters of the last J/K or gradient call: [0] screened shell quartets,
 * [1] kernel launches, [2] device time of the quartet kernels in microseconds
 * (CUDA events on the context stream), [3] quartets evaluated in FP32.
 */
int iqcp_last_stats(const iqcp_ctx* ctx, double* stats4);

/*
 * Measurement support (no counterpart in the reference, which has no GPU path).
 * iqcp_set_profiling: time every quartet-kernel launch with CUDA events.
 * iqcp_launch_profile: per launch of the last call: kind (0 J/K, 1 gradient,
 *   2 / 3 their FP32 share in a mixed call), bra/ket pair class, device ms,
 *   screened quartets of the class (0 for an FP32-share launch); returns the
 *   count.
 * iqcp_kernel_launches: kernels launched by the last call.
 * iqcp_model_flops: algorithmic FLOPs per (bra class X, ket class Y) [6*6] of
 *   one J/K build (kind 0) or gradient (kind 1), from the closed-form count
 *   per surviving primitive quartet; prim_xy / quart_xy may be NULL.
 * iqcp_measure_peak: FMA throughput probe, which = 0 FP64, 1 FP32, TFLOP/s.
 */
int iqcp_set_profiling(iqcp_ctx* ctx, int on);
int iqcp_launch_profile(const iqcp_ctx* ctx, int max, int* kind, int* X, int* Y, double* ms,
                        long long* quartets);
int iqcp_kernel_launches(const iqcp_ctx* ctx);
int iqcp_model_flops(iqcp_ctx* ctx, int kind, double* flops_xy, long long* prim_xy,
                     long long* quart_xy);
int iqcp_measure_peak(int which, double* tflops);

/*
 * Kernel-variant autotuner (no reference counterpart): for every (bra class,
 * ket class) time each quartet-kernel variant (0: one quartet per thread,
 * 1: one warp per quartet with shared-memory 1D tables) on this device-resident
 * density, best of `reps`, and keep the fastest for J/K and for gradients.
 * With precision IQCP_MIXED the FP64 and FP32 shares of every class are tuned
 * separately at the current cutoff, and a class is split into the two only
 * where that is faster than running it wholly in FP64.  Results agree to
 * rounding whichever variant runs.  iqcp_kernel_modes fills modes[4*6*6] as
 * modes[(kind*6 + X)*6 + Y], kind 0 J/K, 1 gradient, 2 / 3 their FP32 share
 * (-1: class has no quartets; 4 for kinds 2 / 3: the class runs wholly in FP64
 * in the mixed form); iqcp_set_kernel_mode forces one (kind 0..3, mode 0..3,
 * or 4 for kinds 2 / 3; X or Y = -1: all classes).
 */
int iqcp_autotune(iqcp_ctx* ctx, const double* d_D, int reps);
int iqcp_kernel_modes(const iqcp_ctx* ctx, int* modes);
int iqcp_set_kernel_mode(iqcp_ctx* ctx, int kind, int X, int Y, int mode);

#ifdef __cplusplus
}
#endif

#endif /* IQCP_H_ */
