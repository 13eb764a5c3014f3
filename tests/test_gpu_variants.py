"""Every quartet-kernel variant the autotuner can choose gives the oracle's
J/K and gradient: 0 one quartet per thread, 1 one warp per quartet
(shared-memory tables), 2 / 3 eight / thirty-two lanes per quartet for J/K;
for gradients 2 is one quartet per thread with its weights in shared memory
and 3 thirty-two lanes over (primitive quartet, root) items."""
import numpy as np
import pytest

from conftest import random_density
from iqcp_b200 import BasisSet, FockEngine
from iqcp_b200.molecules import REFERENCE_MOLECULES, workload

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def systems(oracle_mod):
    out = []
    for mol, basis in [("NH3", "cc-pvdz"), ("CH4", "6-31+g*")]:
        b = BasisSet.build(REFERENCE_MOLECULES[mol], basis)
        D = random_density(b.n_basis, 13)
        Jo, Ko, _ = oracle_mod.jk_direct(b, D)
        go, _ = oracle_mod.eri_gradient(b, D, 1.0)
        out.append((b, D, Jo, Ko, go))
    atoms, basis = workload("c1", 1)
    b = BasisSet.build(atoms, basis)
    D = random_density(b.n_basis, 17, 0.05)
    Jo, Ko, _ = oracle_mod.jk_direct(b, D)
    go, _ = oracle_mod.eri_gradient(b, D, 1.0)
    out.append((b, D, Jo, Ko, go))
    return out


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_variant_parity(systems, mode):
    for b, D, Jo, Ko, go in systems:
        with FockEngine(b) as eng:
            eng.set_kernel_mode("jk", mode=mode)
            eng.set_kernel_mode("grad", mode=mode)
            J, K = eng.build_jk(D)
            g = eng.eri_gradient(D, 1.0)
        assert np.abs(J - Jo).max() < 1e-10
        assert np.abs(K - Ko).max() < 1e-10
        assert np.abs(g - go).max() < 1e-7


def test_autotune_keeps_parity(systems):
    import torch
    b, D, Jo, Ko, go = systems[-1]
    with FockEngine(b) as eng:
        dD = torch.from_numpy(D).cuda()
        modes = eng.autotune(dD.data_ptr(), 1)
        assert set(np.unique(modes)) <= {-1, 0, 1, 2, 3}
        J, K = eng.build_jk(D)
        g = eng.eri_gradient(D, 1.0)
    assert np.abs(J - Jo).max() < 1e-10 and np.abs(K - Ko).max() < 1e-10
    assert np.abs(g - go).max() < 1e-7
