"""CPHF response operator on the device J/K.

The caller side of the reference's ``gen_vind_rhf`` / ``gen_vind_rhf_vo``
(crates/qc-core/src/scf/cphf.rs:828-990): per trial vector ``mo1`` the trial
density dm = C (2 mo1) C_occ^T is symmetrised (dm1 = dm + dm^T), J and K are
built from it, V = J - 1/2 hf_frac K, and the result is C^T V C_occ
(C_vir^T V C_occ for the vo form).  The reference builds J/K one density at a
time from stored ERIs; here all trial densities of one call share a single
pass over the screened quartets (``FockEngine.build_jk_multi``,
``iqcp_jk_multi``).  Same flat layouts: mo1 is nset blocks of nmo x n_occ
(nvir x n_occ), row-major.
"""
import numpy as np


def _trial_densities(C, c_occ, mo1):
    dms = []
    for m in mo1:
        dm = C @ (2.0 * m) @ c_occ.T
        dms.append(dm + dm.T)
    return dms


def gen_vind_rhf(engine, mo_coeff, n_occ, hf_exchange_fraction=1.0):
    """Response function mo1 (nset x nmo x n_occ, flat) -> C^T V[dm1] C_occ (gen_vind_rhf, cphf.rs:828)."""
    C = np.asarray(mo_coeff, dtype=np.float64)
    nmo = C.shape[1]
    c_occ = C[:, :n_occ]

    def vind(mo1_flat):
        mo1 = np.asarray(mo1_flat, dtype=np.float64).reshape(-1, nmo, n_occ)
        J, K = engine.build_jk_multi(_trial_densities(C, c_occ, mo1))
        return np.concatenate([(C.T @ (j - k * (hf_exchange_fraction * 0.5)) @ c_occ).ravel()
                               for j, k in zip(J, K)])
    return vind


def gen_vind_rhf_vo(engine, mo_coeff, n_occ, hf_exchange_fraction=1.0):
    """Virtual-occupied form: mo1 (nset x nvir x n_occ, flat) -> C_vir^T V[dm1] C_occ (cphf.rs:930)."""
    C = np.asarray(mo_coeff, dtype=np.float64)
    nmo = C.shape[1]
    nvir = nmo - n_occ
    c_occ = C[:, :n_occ]

    def vind(mo1_flat):
        mo1 = np.asarray(mo1_flat, dtype=np.float64).reshape(-1, nvir, n_occ)
        full = np.zeros((len(mo1), nmo, n_occ))
        full[:, n_occ:, :] = mo1
        J, K = engine.build_jk_multi(_trial_densities(C, c_occ, full))
        return np.concatenate([(C[:, n_occ:].T @ (j - k * (hf_exchange_fraction * 0.5)) @ c_occ).ravel()
                               for j, k in zip(J, K)])
    return vind
