"""Mixed-precision form: quartets whose Schwarz bound times density bound
falls below the cutoff run their quadrature in FP32 (roots, weights and
accumulation FP64); the rest stay FP64.

Bars: the FP32 kernels of every class and variant agree with FP64 to FP32
rounding when every quartet is forced into FP32; cutoff 0 reproduces the FP64
form; a batched context selects the same quartets as single contexts; and at
the production cutoff the total energy stays within 1 uHa and the gradient
within 1e-6 Ha/bohr of the all-FP64 result.
"""
import numpy as np
import pytest

from conftest import random_density
from iqcp_b200 import MIXED, BasisSet, BatchFockEngine, FockEngine
from iqcp_b200.molecules import REFERENCE_MOLECULES, workload
from iqcp_b200.scf import rhf_scf

pytestmark = pytest.mark.gpu
PRODUCTION_CUTOFF = 1e-3


@pytest.fixture(scope="module")
def c1_scf():
    atoms, basis = workload("c1", 0)
    b = BasisSet.build(atoms, basis)
    with FockEngine(b) as eng:
        S, T, V = eng.one_electron()
        H = T + V
        res = rhf_scf(S, H, b.nuclear_repulsion(), b.n_electrons // 2, eng.build_fock, e_tol=1e-10, d_tol=1e-8)
    return b, H, res.density


def _energy(H, F, D):
    return 0.5 * float(np.sum(D * (H + F)))


def test_cutoff_zero_is_fp64(c1_scf):
    b, H, D = c1_scf
    with FockEngine(b) as eng:
        J0, K0 = eng.build_jk(D)
        g0 = eng.eri_gradient(D, 1.0)
        eng.set_precision(MIXED, 0.0)
        J1, K1 = eng.build_jk(D)
        assert eng.last_stats()["fp32_quartets"] == 0
        g1 = eng.eri_gradient(D, 1.0)
    assert np.abs(J1 - J0).max() < 1e-12 and np.abs(K1 - K0).max() < 1e-12
    assert np.abs(g1 - g0).max() < 1e-11


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_all_fp32_every_variant(mode):
    """Every quartet in FP32 (cutoff 1e30): each FP32 variant agrees with FP64
    to FP32 rounding on a system with d shells up to (dd|dd)."""
    b = BasisSet.build(REFERENCE_MOLECULES["C6H6"], "6-31g*")
    D = random_density(b.n_basis, 5, 0.2)
    with FockEngine(b) as eng:
        J0, K0 = eng.build_jk(D)
        g0 = eng.eri_gradient(D, 1.0)
        eng.set_precision(MIXED, 1e30)
        eng.set_kernel_mode("jk32", mode=mode)
        eng.set_kernel_mode("grad32", mode=mode)
        J1, K1 = eng.build_jk(D)
        st = eng.last_stats()
        g1 = eng.eri_gradient(D, 1.0)
    assert st["fp32_quartets"] == st["quartets"]
    assert np.abs(J1 - J0).max() < 2e-5 * np.abs(J0).max()
    assert np.abs(K1 - K0).max() < 2e-5 * np.abs(K0).max()
    assert np.abs(g1 - g0).max() < 2e-5 * np.abs(g0).max()


def test_production_cutoff_error(c1_scf):
    b, H, D = c1_scf
    with FockEngine(b) as eng:
        F0 = eng.build_fock(H, D)
        g0 = eng.eri_gradient(D, 1.0)
        eng.set_precision(MIXED, PRODUCTION_CUTOFF)
        F1 = eng.build_fock(H, D)
        st = eng.last_stats()
        g1 = eng.eri_gradient(D, 1.0)
    assert st["fp32_quartets"] > 0
    assert abs(_energy(H, F1, D) - _energy(H, F0, D)) < 1e-6
    assert np.abs(g1 - g0).max() < 1e-6


def test_autotuned_mixed_keeps_bounds(c1_scf):
    import torch
    b, H, D = c1_scf
    with FockEngine(b) as eng:
        F0 = eng.build_fock(H, D)
        g0 = eng.eri_gradient(D, 1.0)
        eng.set_precision(MIXED, PRODUCTION_CUTOFF)
        dD = torch.from_numpy(D).cuda()
        modes = eng.autotune(dD.data_ptr(), 1)
        assert set(np.unique(modes[2:])) <= {-1, 0, 1, 2, 4}
        F1 = eng.build_fock(H, D)
        g1 = eng.eri_gradient(D, 1.0)
    assert abs(_energy(H, F1, D) - _energy(H, F0, D)) < 1e-6
    assert np.abs(g1 - g0).max() < 1e-6


def test_batch_mixed_matches_single():
    bases = [BasisSet.build(REFERENCE_MOLECULES[m], bn)
             for m, bn in [("H2O", "6-31g*"), ("C6H6", "6-31g*"), ("NH3", "cc-pvdz")]]
    Ds = [random_density(b.n_basis, 40 + i, 0.2) for i, b in enumerate(bases)]
    cut = 1e-3
    with BatchFockEngine(bases, precision=MIXED, mixed_cutoff=cut) as beng:
        Jb, Kb = beng.build_jk(Ds)
        nb = beng.last_stats()["fp32_quartets"]
        gb = beng.eri_gradient(Ds, 1.0)
    n1 = 0
    for b, D, J, K, g in zip(bases, Ds, Jb, Kb, gb):
        with FockEngine(b, precision=MIXED, mixed_cutoff=cut) as eng:
            J1, K1 = eng.build_jk(D)
            n1 += eng.last_stats()["fp32_quartets"]
            g1 = eng.eri_gradient(D, 1.0)
        assert np.abs(J - J1).max() < 1e-11 and np.abs(K - K1).max() < 1e-11
        assert np.abs(g - g1).max() < 1e-10
    assert nb == n1 and nb > 0
