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
