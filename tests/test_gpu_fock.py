"""Direct J/K and Fock build on the B200 against the oracle (the reference's
shell_eri numerics, stored or direct digestion).  Fock-element parity bar:
1e-10 Ha (absolute)."""
import numpy as np
import pytest

from conftest import golden, random_density
from iqcp_b200 import BasisSet, FockEngine
from iqcp_b200.molecules import REFERENCE_MOLECULES, workload
from iqcp_b200.scf import rhf_scf

pytestmark = pytest.mark.gpu
FOCK_TOL = 1e-10

SMALL = [("H2", "sto-3g"), ("H2O", "sto-3g"), ("H2O", "6-31g*"), ("NH3", "cc-pvdz"), ("HF", "6-31+g*"),
         ("CH4", "3-21g"), ("CH4", "cc-pvdz")]


@pytest.mark.parametrize("mol,basis", SMALL)
def test_schwarz_and_compressed_eri(oracle_mod, mol, basis):
    b = BasisSet.build(REFERENCE_MOLECULES[mol], basis)
    with FockEngine(b) as eng:
        np.testing.assert_allclose(eng.schwarz(), oracle_mod.schwarz(b), rtol=1e-12, atol=1e-15)
        eri_o, _ = oracle_mod.eri_compressed(b)
        np.testing.assert_allclose(eng.eri_compressed(), eri_o, rtol=0, atol=1e-13)


@pytest.mark.parametrize("mol,basis", SMALL)
def test_jk_vs_oracle_small(oracle_mod, mol, basis):
    b = BasisSet.build(REFERENCE_MOLECULES[mol], basis)
    D = random_density(b.n_basis, 7)
    Jo, Ko, _ = oracle_mod.jk_direct(b, D)
    with FockEngine(b) as eng:
        J, K = eng.build_jk(D)
        assert np.abs(J - Jo).max() < FOCK_TOL
        assert np.abs(K - Ko).max() < FOCK_TOL
        Jonly = eng.build_jk(D, with_k=False)
        assert np.abs(Jonly - Jo).max() < FOCK_TOL
        H = oracle_mod.hcore(b)
        eri, _ = oracle_mod.eri_compressed(b)
        Fo = oracle_mod.build_fock(H, D, eri)
        assert np.abs(eng.build_fock(H, D) - Fo).max() < FOCK_TOL
        # hybrid form F = H + J - 0.5*0.2*K (ks_scf.rs:1953-1960)
        assert np.abs(eng.build_fock(H, D, 0.2) - (H + Jo - 0.1 * Ko)).max() < FOCK_TOL


@pytest.mark.parametrize("name", ["c1"])
def test_jk_vs_oracle_workload(oracle_mod, name):
    atoms, basis = workload(name, 0)
    b = BasisSet.build(atoms, basis)
    D = random_density(b.n_basis, 11, 0.05)
    Jo, Ko, cnt = oracle_mod.jk_direct(b, D)
    assert cnt[0] == 0
    with FockEngine(b) as eng:
        J, K = eng.build_jk(D)
        st = eng.last_stats()
    assert st["quartets"] == cnt[3]
    assert np.abs(J - Jo).max() < FOCK_TOL
    assert np.abs(K - Ko).max() < FOCK_TOL


ENERGY_ROWS = [r for r in golden("rhf_energies.json")["rows"]
               if (r["molecule"], r["basis"]) in {("H2O", "6-31g*"), ("NH3", "cc-pvdz"), ("CH4", "6-31+g*"),
                                                  ("HF", "3-21g"), ("C6H6", "6-31g"), ("C6H6", "6-31g*")}]


@pytest.mark.parametrize("row", ENERGY_ROWS, ids=lambda r: "%s-%s" % (r["molecule"], r["basis"]))
def test_scf_energy_with_device_fock(oracle_mod, row):
    """RHF energy with every Fock build on the B200 == the reference's own
    energy (iqcp_iteration_counts.json) to 1 nHa."""
    b = BasisSet.build(REFERENCE_MOLECULES[row["molecule"]], row["basis"])
    S, H = oracle_mod.one_electron(b, "S"), oracle_mod.hcore(b)
    with FockEngine(b) as eng:
        res = rhf_scf(S, H, oracle_mod.nuclear_repulsion(b), b.n_electrons // 2, eng.build_fock,
                      e_tol=1e-12, d_tol=1e-10)
    assert res.converged
    assert abs(res.energy - row["energy"]) < 1e-9, (res.energy, row["energy"])


def test_translation_invariance_c2():
    """Full-size property: J/K do not change when the molecule is translated."""
    atoms, basis = workload("c2", 0)
    b = BasisSet.build(atoms, basis)
    shift = np.array([0.37, -1.25, 2.5])
    b2 = BasisSet.build([(z, tuple(np.array(x) + shift)) for z, x in atoms], basis)
    D = random_density(b.n_basis, 5, 0.05)
    with FockEngine(b) as e1, FockEngine(b2) as e2:
        J1, K1 = e1.build_jk(D)
        J2, K2 = e2.build_jk(D)
    assert np.abs(J1 - J2).max() < 1e-10
    assert np.abs(K1 - K2).max() < 1e-10
    assert np.abs(J1 - J1.T).max() == 0.0 and np.abs(K1 - K1.T).max() == 0.0


@pytest.mark.parametrize("mol,basis", SMALL)
def test_one_electron_vs_oracle(oracle_mod, mol, basis):
    """Overlap, kinetic and nuclear attraction on the device (integrals/overlap.rs:647,
    integrals/hcore.rs:103, integrals/nuclear.rs:68-305)."""
    b = BasisSet.build(REFERENCE_MOLECULES[mol], basis)
    with FockEngine(b) as eng:
        S, T, V = eng.one_electron()
    np.testing.assert_allclose(S, oracle_mod.one_electron(b, "S"), rtol=0, atol=1e-12)
    np.testing.assert_allclose(T, oracle_mod.one_electron(b, "T"), rtol=0, atol=1e-11)
    np.testing.assert_allclose(V, oracle_mod.one_electron(b, "V"), rtol=0, atol=1e-10)
