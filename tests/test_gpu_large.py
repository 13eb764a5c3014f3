"""The large workload: a 100-atom C/N/O/S/H molecule in 6-31+G* (about 1100
Cartesian basis functions, diffuse sp shells, weak screening).  The oracle is
too slow at this size, so the checks are size-independent properties:
symmetric J and K, invariance of J and K under a rigid translation, the hybrid
Fock matrix H + J - 0.1 K (0.2 K exchange scaling) against the separate J and
K, translational invariance of the gradient, and the mixed form's energy and
gradient errors against FP64 at a converged RHF density (host SCF with
canonical orthogonalisation: the overlap matrix is nearly singular)."""
import numpy as np
import pytest

from iqcp_b200 import MIXED, BasisSet, FockEngine
from iqcp_b200.molecules import workload
from iqcp_b200.scf import rhf_scf

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c5():
    atoms, basis = workload("c5", 0)
    b = BasisSet.build(atoms, basis)
    assert 1000 < b.n_basis < 1300
    with FockEngine(b) as eng:
        S, T, V = eng.one_electron()
        H = T + V
        # S has eigenvalues down to ~2e-8 (diffuse shells on 100 atoms): canonical
        # orthogonalisation drops those directions, as quantum-chemistry codes do;
        # a 0.2 Ha virtual-level shift steadies the small-gap iterations
        res = rhf_scf(S, H, b.nuclear_repulsion(), b.n_electrons // 2, eng.build_fock, e_tol=1e-9, d_tol=1e-7,
                      lindep=1e-6, level_shift=0.2, max_iter=200)
    assert res.converged
    return atoms, basis, b, H, res.density


def test_jk_symmetry_translation_and_hybrid(c5):
    atoms, basis, b, H, D = c5
    with FockEngine(b) as eng:
        J, K = eng.build_jk(D)
        F = eng.build_fock(H, D, 0.2)
    assert np.abs(J - J.T).max() < 1e-12 and np.abs(K - K.T).max() < 1e-12
    assert np.abs(F - (H + J - 0.1 * K)).max() < 1e-11
    shift = np.array([3.1, -2.7, 5.3])
    b2 = BasisSet.build([(z, tuple(np.array(x) + shift)) for z, x in atoms], basis)
    with FockEngine(b2) as eng:
        J2, K2 = eng.build_jk(D)
    assert np.abs(J2 - J).max() < 1e-10 and np.abs(K2 - K).max() < 1e-10


def test_gradient_translational_invariance(c5):
    atoms, basis, b, H, D = c5
    with FockEngine(b) as eng:
        g = eng.eri_gradient(D, 1.0)
        g02 = eng.eri_gradient(D, 0.2)
    assert np.abs(g.sum(axis=0)).max() < 1e-7
    assert np.abs(g02.sum(axis=0)).max() < 1e-7


def test_mixed_bounds_large(c5):
    import torch
    atoms, basis, b, H, D = c5
    with FockEngine(b) as eng:
        F0 = eng.build_fock(H, D)
        g0 = eng.eri_gradient(D, 1.0)
        eng.set_precision(MIXED, 1e-3)
        eng.autotune(torch.from_numpy(D).cuda().data_ptr(), 1)
        F1 = eng.build_fock(H, D)
        g1 = eng.eri_gradient(D, 1.0)
    de = 0.5 * float(np.sum(D * (F1 - F0)))
    assert abs(de) < 1e-6
    assert np.abs(g1 - g0).max() < 1e-6
