"""Multi-density J/K (iqcp_jk_multi) for CPHF response densities, and the
compute_fock_decomposition-shaped entry point, against the oracle.

The reference's CPHF (scf/cphf.rs:828-990) builds J and K of each symmetrised
trial density from stored ERIs; iqcp_jk_multi digests every density from one
evaluation of each quartet.  Parity bar: 1e-10 Ha per element."""
import numpy as np
import pytest

from conftest import golden, random_density
from iqcp_b200 import BasisSet, BatchFockEngine, FockEngine
from iqcp_b200.cphf import gen_vind_rhf, gen_vind_rhf_vo
from iqcp_b200.molecules import REFERENCE_MOLECULES, workload
from iqcp_b200.scf import rhf_scf

pytestmark = pytest.mark.gpu
FOCK_TOL = 1e-10


def _basis(mol, basis):
    if basis is None:
        atoms, basis = workload(mol, 0)
        return BasisSet.build(atoms, basis)
    return BasisSet.build(REFERENCE_MOLECULES[mol], basis)


@pytest.mark.parametrize("mol,basis", [("H2O", "6-31g*"), ("NH3", "cc-pvdz"), ("c1", None)])
def test_jk_multi_vs_oracle(oracle_mod, mol, basis):
    b = _basis(mol, basis)
    Ds = [random_density(b.n_basis, 30 + s, 0.05) for s in range(5)]
    with FockEngine(b) as eng:
        J, K = eng.build_jk_multi(Ds)
        Jonly = eng.build_jk_multi(Ds[:2], with_k=False)
        single = [eng.build_jk(D) for D in Ds]
    for s, D in enumerate(Ds):
        Jo, Ko, _ = oracle_mod.jk_direct(b, D)
        assert np.abs(J[s] - Jo).max() < FOCK_TOL, s
        assert np.abs(K[s] - Ko).max() < FOCK_TOL, s
        assert np.abs(J[s] - single[s][0]).max() < 1e-12
        assert np.abs(K[s] - single[s][1]).max() < 1e-12
    for s in range(2):
        assert np.abs(Jonly[s] - J[s]).max() < 1e-12


def test_jk_multi_batched_context(oracle_mod):
    bases = [_basis("H2O", "6-31g*"), _basis("CH4", "6-31+g*")]
    sets = [[random_density(b.n_basis, 50 + 3 * s + m, 0.05) for m, b in enumerate(bases)] for s in range(3)]
    with BatchFockEngine(bases) as eng:
        J, K = eng.build_jk_multi(sets)
    for s in range(3):
        for m in range(len(bases)):
            Jo, Ko, _ = oracle_mod.jk_direct(bases[m], sets[s][m])
            assert np.abs(J[s][m] - Jo).max() < FOCK_TOL
            assert np.abs(K[s][m] - Ko).max() < FOCK_TOL


def _reference_vind(b, oracle_mod, C, n_occ, hf, mo1, vo=False):
    """The reference's loop (cphf.rs:841-917) on the oracle's stored ERIs."""
    eri, _ = oracle_mod.eri_compressed(b)
    nmo = C.shape[1]
    c_occ = C[:, :n_occ]
    out = []
    for m in mo1:
        full = np.zeros((nmo, n_occ))
        if vo:
            full[n_occ:] = m
        else:
            full[:] = m
        dm = C @ (2.0 * full) @ c_occ.T
        J, K = oracle_mod.build_jk_stored(dm + dm.T, eri)
        V = J - K * (hf * 0.5)
        out.append(((C[:, n_occ:] if vo else C).T @ V @ c_occ).ravel())
    return np.concatenate(out)


@pytest.mark.parametrize("hf", [1.0, 0.2])
def test_gen_vind_rhf_vs_reference_loop(oracle_mod, hf):
    b = _basis("H2O", "6-31g*")
    S, H = oracle_mod.one_electron(b, "S"), oracle_mod.hcore(b)
    n_occ = b.n_electrons // 2
    with FockEngine(b) as eng:
        res = rhf_scf(S, H, oracle_mod.nuclear_repulsion(b), n_occ, eng.build_fock)
        C = res.mo_coefficients
        rng = np.random.default_rng(3)
        mo1 = rng.normal(size=(4, C.shape[1], n_occ)) * 0.1
        v = gen_vind_rhf(eng, C, n_occ, hf)(mo1.ravel())
        mo1v = rng.normal(size=(3, C.shape[1] - n_occ, n_occ)) * 0.1
        vv = gen_vind_rhf_vo(eng, C, n_occ, hf)(mo1v.ravel())
    ref = _reference_vind(b, oracle_mod, C, n_occ, hf, mo1)
    refv = _reference_vind(b, oracle_mod, C, n_occ, hf, mo1v, vo=True)
    assert np.abs(v - ref).max() < FOCK_TOL
    assert np.abs(vv - refv).max() < FOCK_TOL


def test_fock_decomposition_h2_pyscf(oracle_mod):
    """compute_fock_decomposition's PySCF matrices for H2 (scf/fock.rs:192-229)."""
    m = golden("fock_h2.json")["matrices"]
    b = _basis("H2", "sto-3g")
    D = np.array(m["PYSCF_D"]).reshape(2, 2)
    H = oracle_mod.hcore(b)
    with FockEngine(b) as eng:
        J, K, G, F = eng.fock_decomposition(H, D)
    for name, X in (("J", J), ("K", K), ("G", G), ("F", F)):
        np.testing.assert_allclose(X, np.array(m["PYSCF_" + name]).reshape(2, 2), atol=1e-8, err_msg=name)


def test_fock_decomposition_vs_oracle(oracle_mod):
    atoms, basis = workload("c1", 0)
    b = BasisSet.build(atoms, basis)
    D = random_density(b.n_basis, 8, 0.05)
    H = oracle_mod.hcore(b)
    Jo, Ko, _ = oracle_mod.jk_direct(b, D)
    with FockEngine(b) as eng:
        J, K, G, F = eng.fock_decomposition(H, D, 0.2)
    assert np.abs(J - Jo).max() < FOCK_TOL and np.abs(K - Ko).max() < FOCK_TOL
    assert np.abs(G - (Jo - 0.1 * Ko)).max() < FOCK_TOL
    assert np.abs(F - (H + Jo - 0.1 * Ko)).max() < FOCK_TOL
