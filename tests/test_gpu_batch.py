"""Batched contexts: many molecules of uneven size through one context.

Every molecule of a batch must get the same J, K, Fock, gradient and
one-electron matrices as a context of its own (to summation-order rounding),
and the oracle's on the same inputs; pairs of different molecules never
interact.  The reference has no batched form: it loops over geometries
(optimizer/mod.rs:274-320), which is what the per-molecule contexts here do.
"""
import numpy as np
import pytest

from conftest import random_density
from iqcp_b200 import BasisSet, BatchFockEngine, FockEngine, IqcpError
from iqcp_b200.molecules import REFERENCE_MOLECULES, batch_geometries

pytestmark = pytest.mark.gpu
FOCK_TOL = 1e-10
GRAD_TOL = 1e-7


def _mixed_bases():
    out = [BasisSet.build(REFERENCE_MOLECULES[m], b)
           for m, b in [("H2O", "6-31g*"), ("H2", "sto-3g"), ("NH3", "cc-pvdz"), ("CH4", "3-21g"),
                        ("HF", "6-31+g*"), ("C6H6", "6-31g*")]]
    # the same molecule twice, displaced: identical shells in separate blocks
    atoms = [(z, tuple(np.array(x) + 0.05)) for z, x in REFERENCE_MOLECULES["H2O"]]
    out.append(BasisSet.build(atoms, "6-31g*"))
    return out


def test_batch_layout():
    bases = _mixed_bases()
    with BatchFockEngine(bases) as eng:
        assert eng.n_mol == len(bases)
        assert list(eng.nbfs) == [b.n_basis for b in bases]
        assert eng.mat_offset[-1] == sum(b.n_basis ** 2 for b in bases)
        assert list(np.diff(eng.atom_offset)) == [b.n_atoms for b in bases]
        assert eng.nbf == sum(b.n_basis for b in bases)


def test_batch_jk_fock_match_single():
    bases = _mixed_bases()
    Ds = [random_density(b.n_basis, 100 + i) for i, b in enumerate(bases)]
    Hs = [random_density(b.n_basis, 200 + i) for i, b in enumerate(bases)]
    with BatchFockEngine(bases) as beng:
        Jb, Kb = beng.build_jk(Ds)
        Fb = beng.build_fock(Hs, Ds, 0.25)
        st = beng.last_stats()
    nq = 0
    for b, D, H, J, K, F in zip(bases, Ds, Hs, Jb, Kb, Fb):
        with FockEngine(b) as eng:
            J1, K1 = eng.build_jk(D)
            nq += eng.last_stats()["quartets"]
            F1 = eng.build_fock(H, D, 0.25)
        assert np.abs(J - J1).max() < 1e-12
        assert np.abs(K - K1).max() < 1e-12
        assert np.abs(F - F1).max() < 1e-12
    # no cross-molecule quartets: the batch evaluates exactly the sum
    assert st["quartets"] == nq


def test_batch_vs_oracle(oracle_mod):
    bases = _mixed_bases()[:4]
    Ds = [random_density(b.n_basis, 300 + i) for i, b in enumerate(bases)]
    with BatchFockEngine(bases) as eng:
        Jb, Kb = eng.build_jk(Ds)
        gb = eng.eri_gradient(Ds, 0.6)
        Sb, Tb, Vb = eng.one_electron()
    for b, D, J, K, g, S, T, V in zip(bases, Ds, Jb, Kb, gb, Sb, Tb, Vb):
        Jo, Ko, _ = oracle_mod.jk_direct(b, D)
        assert np.abs(J - Jo).max() < FOCK_TOL
        assert np.abs(K - Ko).max() < FOCK_TOL
        go, _ = oracle_mod.eri_gradient(b, D, 0.6)
        assert np.abs(g - go).max() < GRAD_TOL
        np.testing.assert_allclose(S, oracle_mod.one_electron(b, "S"), rtol=0, atol=1e-12)
        np.testing.assert_allclose(T, oracle_mod.one_electron(b, "T"), rtol=0, atol=1e-11)
        np.testing.assert_allclose(V, oracle_mod.one_electron(b, "V"), rtol=0, atol=1e-10)


def test_batch_gradient_match_single():
    bases = _mixed_bases()
    Ds = [random_density(b.n_basis, 400 + i, 0.3) for i, b in enumerate(bases)]
    with BatchFockEngine(bases) as beng:
        gb = beng.eri_gradient(Ds, 1.0)
    for b, D, g in zip(bases, Ds, gb):
        with FockEngine(b) as eng:
            g1 = eng.eri_gradient(D, 1.0)
        assert g.shape == (b.n_atoms, 3)
        assert np.abs(g - g1).max() < 1e-10
        # translational invariance holds per molecule
        assert np.abs(g.sum(axis=0)).max() < 1e-8


def test_batch_uneven_geometries():
    """Perturbed geometries of 8-20 atoms (H..Cl, 6-31G*), like a scan or a
    conformer screen; compared molecule by molecule with single contexts."""
    geoms = batch_geometries(12, seed=3, min_atoms=8, max_atoms=20)
    bases = [BasisSet.build(a, "6-31g*") for a in geoms]
    Ds = [random_density(b.n_basis, 500 + i, 0.05) for i, b in enumerate(bases)]
    with BatchFockEngine(bases) as beng:
        Jb, Kb = beng.build_jk(Ds)
        gb = beng.eri_gradient(Ds, 1.0)
    for i in (0, 5, 11):
        with FockEngine(bases[i]) as eng:
            J1, K1 = eng.build_jk(Ds[i])
            g1 = eng.eri_gradient(Ds[i], 1.0)
        assert np.abs(Jb[i] - J1).max() < 1e-11
        assert np.abs(Kb[i] - K1).max() < 1e-11
        assert np.abs(gb[i] - g1).max() < 1e-9


def test_batch_single_geometry_only_calls():
    bases = _mixed_bases()[:2]
    with BatchFockEngine(bases) as eng:
        with pytest.raises(IqcpError):
            eng.eri_compressed()
        rc = eng._lib.iqcp_eri_compressed(eng._h, None, 0)
        assert rc != 0


def test_batch_rhf_gradient_match_single():
    bases = _mixed_bases()[:4]
    Ds = [random_density(b.n_basis, 600 + i, 0.3) for i, b in enumerate(bases)]
    Ws = [random_density(b.n_basis, 700 + i, 0.3) for i, b in enumerate(bases)]
    with BatchFockEngine(bases) as beng:
        g1b = beng.one_electron_gradient(Ds, Ws)
        gb = beng.rhf_gradient(Ds, Ws)
    for b, D, W, g1, g in zip(bases, Ds, Ws, g1b, gb):
        with FockEngine(b) as eng:
            assert np.abs(g1 - eng.one_electron_gradient(D, W)).max() < 1e-10
            assert np.abs(g - eng.rhf_gradient(D, W)).max() < 1e-10
