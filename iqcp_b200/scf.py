"""Host-side RHF driver: the caller of the Fock build.

Mirrors the reference's ``rhf_scf`` (crates/qc-core/src/scf/mod.rs:1363-1586):
symmetric orthogonaliser X = S^-1/2 (:709), core-Hamiltonian guess
(:1379-1389), D = 2 C_occ C_occ^T (:780), E = 1/2 Tr D(H+F) + E_nuc (:898),
Pulay DIIS on the AO commutator FDS - SDF (:990, :1116-1327), and the
energy / RMS-density / orbital-gradient convergence test (:1508-1520).
The Fock builder is injected: ``FockEngine.build_fock`` on the B200 for the
product, or any callable with the same signature.
"""
import numpy as np


class ScfResult:
    def __init__(self, **kw):
        self.__dict__.update(kw)


def _orthogonalizer(S, lindep=None):
    """Symmetric S^-1/2 (build_orthogonalizer, scf/mod.rs:709-735: error at
    eigenvalues <= 1e-10).  With lindep set and the smallest eigenvalue below
    it, canonical orthogonalisation instead: the eigenvectors with eigenvalues
    below lindep are dropped (X is nbf x nkept), which keeps near-linearly
    dependent diffuse bases (large molecules in 6-31+G*) from amplifying
    rounding into the orthogonal basis.  Off by default, as in the reference."""
    w, U = np.linalg.eigh(S)
    if w.min() <= 1e-10 and lindep is None:
        raise ValueError("overlap matrix is singular")
    if lindep is not None and w.min() < lindep:
        keep = w >= lindep
        return U[:, keep] / np.sqrt(w[keep])
    return (U / np.sqrt(w)) @ U.T


def rhf_scf(S, H, e_nuc, n_occ, build_fock, e_tol=1e-10, d_tol=1e-8, max_iter=100, diis_size=8,
            use_diis=True, D0=None, lindep=None, level_shift=0.0):
    """Restricted Hartree-Fock; build_fock(H, D) -> F.  Returns ScfResult.
    lindep: optional canonical-orthogonalisation threshold (see _orthogonalizer).
    level_shift: optional shift (Ha) of the virtual space of the current
    density before each diagonalisation, F' + shift (1 - P) with P the
    occupied projector in the orthogonal basis; it damps occupied-virtual
    oscillations of small-gap systems and leaves the converged solution
    unchanged (off by default, as in the reference)."""
    X = _orthogonalizer(S, lindep)
    if D0 is None:
        _, Cp = np.linalg.eigh(X.T @ H @ X)
        C = X @ Cp
        D = 2.0 * C[:, :n_occ] @ C[:, :n_occ].T
    else:
        D = D0.copy()
    F = build_fock(H, D)
    E = 0.5 * np.sum(D * (H + F)) + e_nuc
    focks, errs = [], []
    converged = False
    it = 0
    eps = None
    for it in range(1, max_iter + 1):
        E_old, D_old = E, D
        Fd = F
        if use_diis:
            err = F @ D @ S - S @ D @ F
            focks.append(F.copy())
            errs.append(err)
            if len(focks) > diis_size:
                focks.pop(0)
                errs.pop(0)
            m = len(focks)
            if m >= 2:
                B = -np.ones((m + 1, m + 1))
                B[m, m] = 0.0
                for i in range(m):
                    for j in range(m):
                        B[i, j] = np.sum(errs[i] * errs[j])
                rhs = np.zeros(m + 1)
                rhs[m] = -1.0
                try:
                    c = np.linalg.solve(B, rhs)[:m]
                    Fd = sum(ci * fi for ci, fi in zip(c, focks))
                except np.linalg.LinAlgError:
                    Fd = F
        Fo = X.T @ Fd @ X
        if level_shift:
            P = 0.5 * (X.T @ S @ D @ S @ X)
            Fo = Fo + level_shift * (np.eye(Fo.shape[0]) - P)
        eps, Cp = np.linalg.eigh(Fo)
        C = X @ Cp
        D = 2.0 * C[:, :n_occ] @ C[:, :n_occ].T
        F = build_fock(H, D)
        E = 0.5 * np.sum(D * (H + F)) + e_nuc
        dE = abs(E - E_old)
        rms = np.sqrt(np.mean((D - D_old) ** 2))
        # ||F_vo|| in the MO basis
        Fmo = C.T @ F @ C
        grad = np.linalg.norm(Fmo[n_occ:, :n_occ]) * 2.0
        if dE < e_tol and rms < d_tol and grad < np.sqrt(e_tol):
            converged = True
            break
    eps, Cp = np.linalg.eigh(X.T @ F @ X)
    C = X @ Cp
    return ScfResult(energy=E, converged=converged, iterations=it, density=D, fock=F, mo_coefficients=C,
                     mo_energies=eps, n_occ=n_occ)


def energy_weighted_density(C, eps, n_occ):
    """W = 2 sum_occ eps_i C_mi C_ni  (scf/gradient.rs:101-130)."""
    Co = C[:, :n_occ]
    return 2.0 * (Co * eps[:n_occ]) @ Co.T
