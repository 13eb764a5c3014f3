"""Internal consistency of the oracle: the direct J/K (per-quartet digestion
with 8-fold weights) equals the reference's stored-ERI digestion, and the
analytic gradient matches PySCF goldens and central finite differences."""
import numpy as np
import pytest

from conftest import golden, random_density
from iqcp_b200 import BasisSet
from iqcp_b200.molecules import REFERENCE_MOLECULES
from iqcp_b200.scf import energy_weighted_density, rhf_scf


@pytest.mark.parametrize("mol,basis", [("H2O", "6-31g*"), ("NH3", "cc-pvdz"), ("HF", "6-31+g*")])
def test_direct_jk_equals_stored(oracle_mod, mol, basis):
    b = BasisSet.build(REFERENCE_MOLECULES[mol], basis)
    D = random_density(b.n_basis, 3)
    eri, _ = oracle_mod.eri_compressed(b)
    Js, Ks = oracle_mod.build_jk_stored(D, eri)
    Jd, Kd, cnt = oracle_mod.jk_direct(b, D)
    assert cnt[0] == 0
    np.testing.assert_allclose(Jd, Js, atol=1e-12)
    np.testing.assert_allclose(Kd, Ks, atol=1e-12)
    # build_fock form (scf/mod.rs:825) == H + J - K/2
    H = np.zeros_like(D)
    np.testing.assert_allclose(oracle_mod.build_fock(H, D, eri), Js - 0.5 * Ks, atol=1e-12)


def _scf(oracle_mod, b):
    S, H = oracle_mod.one_electron(b, "S"), oracle_mod.hcore(b)
    eri, _ = oracle_mod.eri_compressed(b)
    res = rhf_scf(S, H, oracle_mod.nuclear_repulsion(b), b.n_electrons // 2,
                  lambda H_, D: oracle_mod.build_fock(H_, D, eri), e_tol=1e-13, d_tol=1e-11)
    return res


def full_gradient(oracle_mod, b, res, two_e):
    W = energy_weighted_density(res.mo_coefficients, res.mo_energies, res.n_occ)
    return oracle_mod.one_electron_gradient(b, res.density, W) + two_e


ROWS = [r for r in golden("gradients.json")["rows"] if r["molecule"] in ("H2", "HF", "H2O", "NH3", "CH4")]


@pytest.mark.parametrize("row", ROWS, ids=lambda r: "%s-%s" % (r["molecule"], r["basis"]))
def test_rhf_gradient_vs_pyscf(oracle_mod, row):
    b = BasisSet.build(REFERENCE_MOLECULES[row["molecule"]], row["basis"])
    res = _scf(oracle_mod, b)
    assert abs(res.energy - row["energy"]) < 1e-7
    g2, cnt = oracle_mod.eri_gradient(b, res.density, 1.0)
    g = full_gradient(oracle_mod, b, res, g2)
    np.testing.assert_allclose(g, np.array(row["gradient"]), atol=2e-5)   # gradient.rs:2741


def test_rhf_gradient_vs_finite_difference(oracle_mod):
    atoms = REFERENCE_MOLECULES["H2O"]
    b = BasisSet.build(atoms, "6-31g*")
    res = _scf(oracle_mod, b)
    g2, _ = oracle_mod.eri_gradient(b, res.density, 1.0)
    g = full_gradient(oracle_mod, b, res, g2)
    h = 1e-4
    for atom, d in [(0, 2), (1, 1), (2, 2)]:
        e = []
        for s in (+1, -1):
            at = [(z, list(x)) for z, x in atoms]
            at[atom][1][d] += s * h
            e.append(_scf(oracle_mod, BasisSet.build([(z, tuple(x)) for z, x in at], "6-31g*")).energy)
        fd = (e[0] - e[1]) / (2 * h)
        assert abs(fd - g[atom, d]) < 1e-7, (atom, d, fd, g[atom, d])


def test_stride_phases_partition_the_workload(oracle_mod):
    """The benchmark's reference arm times the oracle on bra-pair phases
    P % K == k, k = 0..K-1: together they are exactly one full J/K build and
    one full gradient."""
    from iqcp_b200.molecules import REFERENCE_MOLECULES
    from oracle.basis import build_basis
    b = build_basis(REFERENCE_MOLECULES["H2O"], "6-31g*")
    rng = np.random.default_rng(4)
    A = rng.normal(size=(b.n_basis, b.n_basis)) * 0.1
    D = A + A.T
    J, K, _ = oracle_mod.jk_direct(b, D)
    g, _ = oracle_mod.eri_gradient(b, D, 1.0)
    Js, Ks, gs = np.zeros_like(J), np.zeros_like(K), np.zeros_like(g)
    for k in range(3):
        Jk, Kk, _ = oracle_mod.jk_direct(b, D, 3, k)
        gk, _ = oracle_mod.eri_gradient(b, D, 1.0, 3, k)
        Js += Jk
        Ks += Kk
        gs += gk
    assert np.abs(Js - J).max() < 1e-12 and np.abs(Ks - K).max() < 1e-12
    assert np.abs(gs - g).max() < 1e-12
