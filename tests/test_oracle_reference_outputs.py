"""The oracle against the reference's own FP64 outputs: RHF energies of the
benchmark systems (iqcp_iteration_counts.json, 12 decimals), the IEEE bit
patterns of determinism.json, and the PySCF presets / fock.rs goldens the
reference tests its J/K digestion with."""
import struct

import numpy as np
import pytest

from conftest import golden
from iqcp_b200 import BasisSet
from iqcp_b200.molecules import REFERENCE_MOLECULES
from iqcp_b200.scf import rhf_scf

SYMBOL_Z = {"H": 1, "He": 2, "Li": 3, "N": 7, "O": 8, "C": 6, "F": 9}


def _energy(oracle_mod, mol, basis):
    b = BasisSet.build(REFERENCE_MOLECULES[mol], basis)
    S, H = oracle_mod.one_electron(b, "S"), oracle_mod.hcore(b)
    eri, cnt = oracle_mod.eri_compressed(b)
    assert cnt[0] == 0, "oracle dropped primitive quartets on a Rys failure"
    res = rhf_scf(S, H, oracle_mod.nuclear_repulsion(b), b.n_electrons // 2,
                  lambda H_, D: oracle_mod.build_fock(H_, D, eri), e_tol=1e-12, d_tol=1e-10)
    assert res.converged
    return res.energy


ROWS = [r for r in golden("rhf_energies.json")["rows"] if r["molecule"] != "C6H6"]


@pytest.mark.parametrize("row", ROWS, ids=lambda r: "%s-%s" % (r["molecule"], r["basis"]))
def test_rhf_energy_matches_reference(oracle_mod, row):
    e = _energy(oracle_mod, row["molecule"], row["basis"])
    # printed to 12 decimals; the reference converged to ScfConfig::tight (1e-10)
    assert abs(e - row["energy"]) < 1e-10, (e, row["energy"])


@pytest.mark.slow
def test_rhf_energy_benzene_631g(oracle_mod):
    row = [r for r in golden("rhf_energies.json")["rows"] if r["molecule"] == "C6H6" and r["basis"] == "6-31g"][0]
    e = _energy(oracle_mod, "C6H6", "6-31g")
    assert abs(e - row["energy"]) < 1e-9


def test_determinism_bit_patterns(oracle_mod):
    """determinism.json holds the IEEE bits of the browser runs, which digest
    the preset (PySCF) integrals: the stored-ERI build_fock path."""
    hexes = golden("rhf_energies.json")["determinism_hex"]
    presets = {p["system_id"]: p for p in golden("presets.json")["systems"]}
    for name, sid in [("RHF H2/STO-3G", "h2_sto3g_r1.4"), ("RHF H2O/STO-3G", "h2o_sto3g"),
                      ("RHF NH3/STO-3G", "nh3_sto3g")]:
        ref = struct.unpack(">d", bytes.fromhex(hexes[name]))[0]
        p = presets[sid]
        n = p["nbf"]
        S, H = np.array(p["s_matrix"]).reshape(n, n), np.array(p["h_core"]).reshape(n, n)
        eri = np.array(p["eri_compressed"])
        res = rhf_scf(S, H, p["e_nuc"], p["nelec"] // 2, lambda H_, D: oracle_mod.build_fock(H_, D, eri),
                      e_tol=1e-12, d_tol=1e-10)
        assert abs(res.energy - ref) < 1e-10, (name, res.energy, ref)


def _preset_basis(p):
    atoms = [(SYMBOL_Z[a["symbol"]], tuple(a["xyz"])) for a in p["geometry"]["atoms"]]
    return BasisSet.build(atoms, "sto-3g")


@pytest.mark.parametrize("p", golden("presets.json")["systems"], ids=lambda p: p["system_id"])
def test_presets_integrals_and_digestion(oracle_mod, p):
    b = _preset_basis(p)
    n = p["nbf"]
    assert b.n_basis == n
    S = np.array(p["s_matrix"]).reshape(n, n)
    H = np.array(p["h_core"]).reshape(n, n)
    eri_ref = np.array(p["eri_compressed"])
    np.testing.assert_allclose(oracle_mod.one_electron(b, "S"), S, atol=1e-8)
    np.testing.assert_allclose(oracle_mod.hcore(b), H, atol=1e-8)
    eri, _ = oracle_mod.eri_compressed(b)
    np.testing.assert_allclose(eri, eri_ref, atol=5e-8)   # eri/mod.rs:4415 TOL
    # digestion alone, on the PySCF integrals
    res = rhf_scf(S, H, p["e_nuc"], p["nelec"] // 2, lambda H_, D: oracle_mod.build_fock(H_, D, eri_ref),
                  e_tol=1e-12, d_tol=1e-10)
    assert abs(res.energy - p["reference"]["energy"]) < 1e-8


def test_fock_h2_pyscf_matrices(oracle_mod):
    m = golden("fock_h2.json")["matrices"]
    b = BasisSet.build(REFERENCE_MOLECULES["H2"], "sto-3g")
    eri, _ = oracle_mod.eri_compressed(b)
    D = np.array(m["PYSCF_D"]).reshape(2, 2)
    J, K = oracle_mod.build_jk_stored(D, eri)
    np.testing.assert_allclose(J, np.array(m["PYSCF_J"]).reshape(2, 2), atol=1e-8)
    np.testing.assert_allclose(K, np.array(m["PYSCF_K"]).reshape(2, 2), atol=1e-8)
    np.testing.assert_allclose(J - 0.5 * K, np.array(m["PYSCF_G"]).reshape(2, 2), atol=1e-8)
    F = oracle_mod.build_fock(oracle_mod.hcore(b), D, eri)
    np.testing.assert_allclose(F, np.array(m["PYSCF_F"]).reshape(2, 2), atol=1e-8)
