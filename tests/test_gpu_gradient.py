"""Two-electron nuclear gradient on the B200 against the oracle's fused
gradient (eri_gradient_fused restated), PySCF goldens, and finite differences.
Gradient parity bar: 1e-7 Ha/bohr."""
import numpy as np
import pytest

from conftest import golden, random_density
from iqcp_b200 import BasisSet, FockEngine
from iqcp_b200.molecules import REFERENCE_MOLECULES, workload
from iqcp_b200.scf import energy_weighted_density, rhf_scf

pytestmark = pytest.mark.gpu
GRAD_TOL = 1e-7


@pytest.mark.parametrize("mol,basis", [("H2", "sto-3g"), ("H2O", "6-31g*"), ("NH3", "cc-pvdz"),
                                       ("HF", "6-31+g*"), ("CH4", "6-31g*")])
@pytest.mark.parametrize("hf_frac", [1.0, 0.2])
def test_eri_gradient_vs_oracle(oracle_mod, mol, basis, hf_frac):
    b = BasisSet.build(REFERENCE_MOLECULES[mol], basis)
    D = random_density(b.n_basis, 9)
    go, cnt = oracle_mod.eri_gradient(b, D, hf_frac)
    with FockEngine(b) as eng:
        g = eng.eri_gradient(D, hf_frac)
    assert np.abs(g - go).max() < GRAD_TOL * max(1.0, np.abs(go).max() * 1e-3), np.abs(g - go).max()


def test_eri_gradient_vs_oracle_workload(oracle_mod):
    atoms, basis = workload("c1", 0)
    b = BasisSet.build(atoms, basis)
    D = random_density(b.n_basis, 4, 0.05)
    go, _ = oracle_mod.eri_gradient(b, D, 1.0)
    with FockEngine(b) as eng:
        g = eng.eri_gradient(D, 1.0)
    assert np.abs(g - go).max() < GRAD_TOL


ROWS = [r for r in golden("gradients.json")["rows"]
        if (r["molecule"], r["basis"]) in {("H2O", "6-31g*"), ("NH3", "6-31g*"), ("CH4", "6-31+g*"), ("HF", "3-21g")}]


@pytest.mark.parametrize("row", ROWS, ids=lambda r: "%s-%s" % (r["molecule"], r["basis"]))
def test_rhf_gradient_vs_pyscf(oracle_mod, row):
    b = BasisSet.build(REFERENCE_MOLECULES[row["molecule"]], row["basis"])
    S, H = oracle_mod.one_electron(b, "S"), oracle_mod.hcore(b)
    with FockEngine(b) as eng:
        res = rhf_scf(S, H, oracle_mod.nuclear_repulsion(b), b.n_electrons // 2, eng.build_fock,
                      e_tol=1e-13, d_tol=1e-11)
        g2 = eng.eri_gradient(res.density, 1.0)
    W = energy_weighted_density(res.mo_coefficients, res.mo_energies, res.n_occ)
    g = oracle_mod.one_electron_gradient(b, res.density, W) + g2
    np.testing.assert_allclose(g, np.array(row["gradient"]), atol=2e-5)
    # and against the all-oracle gradient at the same density
    go, _ = oracle_mod.eri_gradient(b, res.density, 1.0)
    assert np.abs(g2 - go).max() < GRAD_TOL


@pytest.mark.parametrize("mol,basis", [("H2O", "6-31g*"), ("NH3", "cc-pvdz"), ("HF", "6-31+g*"), ("CH4", "3-21g")])
def test_one_electron_gradient_vs_oracle(oracle_mod, mol, basis):
    """Device nuclear repulsion + D dH - W dS against the oracle at the same D, W."""
    b = BasisSet.build(REFERENCE_MOLECULES[mol], basis)
    D = random_density(b.n_basis, 21)
    W = random_density(b.n_basis, 22)
    go = oracle_mod.one_electron_gradient(b, D, W)
    with FockEngine(b) as eng:
        g = eng.one_electron_gradient(D, W)
    assert np.abs(g - go).max() < 1e-9, np.abs(g - go).max()


@pytest.mark.parametrize("row", ROWS, ids=lambda r: "%s-%s" % (r["molecule"], r["basis"]))
def test_device_rhf_gradient_vs_pyscf(row):
    """The whole RHF gradient on the device (no oracle on the path) against PySCF."""
    b = BasisSet.build(REFERENCE_MOLECULES[row["molecule"]], row["basis"])
    with FockEngine(b) as eng:
        S, T, V = eng.one_electron()
        res = rhf_scf(S, T + V, b.nuclear_repulsion(), b.n_electrons // 2, eng.build_fock, e_tol=1e-13, d_tol=1e-11)
        W = energy_weighted_density(res.mo_coefficients, res.mo_energies, res.n_occ)
        g = eng.rhf_gradient(res.density, W)
    np.testing.assert_allclose(g, np.array(row["gradient"]), atol=2e-5)
    assert np.abs(g.sum(axis=0)).max() < 1e-8


def _scf(atoms, basis):
    b = BasisSet.build(atoms, basis)
    with FockEngine(b) as eng:
        S, T, V = eng.one_electron()
        res = rhf_scf(S, T + V, b.nuclear_repulsion(), b.n_electrons // 2, eng.build_fock, e_tol=1e-13,
                      d_tol=1e-10)
    assert res.converged
    return res


@pytest.mark.parametrize("mol,basis,coords", [("H2O", "cc-pvdz", None), ("c3", "cc-pvdz", [(0, 0), (7, 1), (20, 2)])])
def test_rhf_gradient_vs_finite_differences(mol, basis, coords):
    """Analytic device gradient against central differences of SCF energies,
    step 1e-4 bohr (the analytic-vs-FD check of scf/gradient.rs:2887-2930),
    on H2O and on a 30-atom C/N/O/F/H cc-pVDZ molecule (subset of coordinates)."""
    atoms = REFERENCE_MOLECULES[mol] if mol in REFERENCE_MOLECULES else workload(mol, 0)[0]
    res = _scf(atoms, basis)
    b = BasisSet.build(atoms, basis)
    W = energy_weighted_density(res.mo_coefficients, res.mo_energies, res.n_occ)
    with FockEngine(b) as eng:
        g = eng.rhf_gradient(res.density, W)
    if coords is None:
        coords = [(a, d) for a in range(len(atoms)) for d in range(3)]
    h = 1e-4
    for a, d in coords:
        e = []
        for sgn in (1, -1):
            moved = [(z, tuple(x[k] + (sgn * h if (i == a and k == d) else 0.0) for k in range(3)))
                     for i, (z, x) in enumerate(atoms)]
            e.append(_scf(moved, basis).energy)
        fd = (e[0] - e[1]) / (2 * h)
        assert abs(fd - g[a, d]) < 1e-6, (a, d, fd, g[a, d])
