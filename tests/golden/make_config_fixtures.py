"""Oracle fixtures at the benchmark workloads (seed 0), for the -m gpu parity tests.

Runs the CPU oracle (the reference's FP64 path restated in C++, oracle/) on the
seeded synthetic molecules and writes compressed .npz files next to this
script.  No GPU and no product library: bases come from oracle/basis.py, the
SCF driver is iqcp_b200/scf.py (pure numpy) with the oracle's direct J/K as
its Fock builder.

  config_c2.npz  40-atom C/N/O/H, RHF/6-31G* (392 bf): oracle-converged RHF
                 (energy, occupied orbitals and energies), the two-electron
                 gradient and the full RHF gradient at that density.
  config_c3.npz  30-atom C/N/O/F/H, RHF/cc-pVDZ (300 bf): the same.
  config_c5.npz  100-atom C/N/O/S/H, RHF/6-31+G* (1129 bf): the oracle's J
                 and K at a seeded bounded density (c5_density) as row sums,
                 Tr(DJ), Tr(DK) and 20000 seeded element samples.
  c5x            (optional) adds to config_c5.npz the same quantities with the
                 oracle's Rys roots in extended precision
                 (oracle.set_root_precision), a second reading that separates
                 the reference's double-precision root error (up to ~2e-11
                 relative at five roots) from a device-side difference.

Usage: python tests/golden/make_config_fixtures.py [c2 c3 c5 c5x]   (about 2 h on 8 cores,
c5x about 1 h more)
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle.basis import build_basis  # noqa: E402
from iqcp_b200.molecules import workload  # noqa: E402
from iqcp_b200.scf import energy_weighted_density, rhf_scf  # noqa: E402


def oracle_fock_builder(b, log):
    calls = [0]

    def build(H, D):
        t0 = time.time()
        J, K, cnt = oracle.jk_direct(b, D)
        assert cnt[0] == 0, "Rys failures in the oracle"
        calls[0] += 1
        log("  oracle J/K %d: %.1f s" % (calls[0], time.time() - t0))
        return H + J - 0.5 * K
    return build


def geometry(atoms):
    return np.array([z for z, _ in atoms], np.int32), np.array([p for _, p in atoms], np.float64)


def scf_fixture(name, log):
    atoms, basis = workload(name, 0)
    b = build_basis(atoms, basis)
    log("%s: %d atoms, %d bf, %d electrons" % (name, b.n_atoms, b.n_basis, b.n_electrons))
    S = oracle.one_electron(b, "S")
    H = oracle.hcore(b)
    enuc = oracle.nuclear_repulsion(b)
    n_occ = b.n_electrons // 2
    t0 = time.time()
    res = rhf_scf(S, H, enuc, n_occ, oracle_fock_builder(b, log), e_tol=1e-10, d_tol=1e-8, max_iter=150)
    t_scf = time.time() - t0
    log("  SCF: E = %.12f, %d iterations, converged %s, %.0f s" % (res.energy, res.iterations, res.converged,
                                                                   t_scf))
    C = res.mo_coefficients[:, :n_occ]
    eps = res.mo_energies[:n_occ]
    D = 2.0 * C @ C.T
    W = energy_weighted_density(res.mo_coefficients, res.mo_energies, n_occ)
    t0 = time.time()
    g2, cnt = oracle.eri_gradient(b, D, 1.0)
    t_g = time.time() - t0
    g1 = oracle.one_electron_gradient(b, D, W)
    log("  gradient: %.0f s, max |g| = %.3e" % (t_g, np.abs(g1 + g2).max()))
    z, xyz = geometry(atoms)
    meta = {"workload": name, "seed": 0, "basis": basis, "nbf": b.n_basis, "n_occ": n_occ,
            "energy": res.energy, "scf_iterations": res.iterations, "scf_converged": bool(res.converged),
            "scf_tolerances": {"e_tol": 1e-10, "d_tol": 1e-8}, "oracle_threads": oracle.max_threads(),
            "oracle_scf_s": t_scf, "oracle_gradient_s": t_g,
            "density": "D = 2 C_occ C_occ^T from c_occ", "w": "W = 2 C_occ diag(eps_occ) C_occ^T"}
    np.savez_compressed(os.path.join(HERE, "config_%s.npz" % name), meta=json.dumps(meta), z=z, xyz=xyz,
                        c_occ=C, eps_occ=eps, grad_2e=g2, grad_rhf=g1 + g2, e_nuc=enuc)


def c5_density(n, seed=5, scale=0.02):
    """The C5 parity density: seeded, symmetric, elements of order `scale`.
    (The core-Hamiltonian guess of this near-linearly-dependent 6-31+G* basis,
    overlap eigenvalues down to 1.8e-8, has density elements up to 1e6: each
    J element is then a cancellation of ~1e6-sized terms, and two FP64
    evaluations of it differ by ~1e-9 whatever their quadrature.)"""
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(n, n)) * scale
    return A + A.T


def c5_fixture(log):
    atoms, basis = workload("c5", 0)
    b = build_basis(atoms, basis)
    n = b.n_basis
    log("c5: %d atoms, %d bf" % (b.n_atoms, n))
    D = c5_density(n)
    t0 = time.time()
    J, K, cnt = oracle.jk_direct(b, D)
    t_jk = time.time() - t0
    assert cnt[0] == 0
    log("  oracle J/K: %.0f s" % t_jk)
    rng = np.random.default_rng(5)
    idx = rng.integers(0, n, size=(20000, 2)).astype(np.int32)
    z, xyz = geometry(atoms)
    meta = {"workload": "c5", "seed": 0, "basis": basis, "nbf": n,
            "density": "c5_density(nbf): rng(5) normal(nbf, nbf) * 0.02, D = A + A^T",
            "density_seed": 5, "density_scale": 0.02,
            "oracle_threads": oracle.max_threads(), "oracle_jk_s": t_jk,
            "shell_quartets": int(cnt[3]), "prim_quartets": int(cnt[2])}
    np.savez_compressed(os.path.join(HERE, "config_c5.npz"), meta=json.dumps(meta), z=z, xyz=xyz,
                        idx=idx, j_sample=J[idx[:, 0], idx[:, 1]], k_sample=K[idx[:, 0], idx[:, 1]],
                        j_rowsum=J.sum(1), k_rowsum=K.sum(1), tr_dj=float(np.sum(D * J)),
                        tr_dk=float(np.sum(D * K)))


def c5x_fixture(log):
    path = os.path.join(HERE, "config_c5.npz")
    f = dict(np.load(path))
    meta = json.loads(str(f["meta"]))
    atoms, basis = workload("c5", 0)
    b = build_basis(atoms, basis)
    D = c5_density(b.n_basis, int(meta["density_seed"]), float(meta["density_scale"]))
    idx = f["idx"]
    oracle.set_root_precision(True)
    try:
        t0 = time.time()
        J, K, cnt = oracle.jk_direct(b, D)
        t_jk = time.time() - t0
    finally:
        oracle.set_root_precision(False)
    assert cnt[0] == 0
    log("  oracle J/K, extended-precision roots: %.0f s" % t_jk)
    meta["oracle_jk_extended_s"] = t_jk
    meta["extended"] = "*_x: the same J/K with the Rys roots computed in long double"
    f.update(meta=json.dumps(meta), j_sample_x=J[idx[:, 0], idx[:, 1]], k_sample_x=K[idx[:, 0], idx[:, 1]],
             j_rowsum_x=J.sum(1), k_rowsum_x=K.sum(1), tr_dj_x=float(np.sum(D * J)), tr_dk_x=float(np.sum(D * K)))
    np.savez_compressed(path, **f)


def main():
    which = sys.argv[1:] or ["c2", "c3", "c5"]

    def log(msg):
        print(msg, flush=True)
    for name in which:
        if name == "c5":
            c5_fixture(log)
        elif name == "c5x":
            c5x_fixture(log)
        else:
            scf_fixture(name, log)


if __name__ == "__main__":
    main()
