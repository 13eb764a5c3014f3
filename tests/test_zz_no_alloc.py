"""The J/K entry point that allocates nothing (iqcp_jk_device_noalloc).

It exists for callers whose Fock-build loop may not call cudaMalloc: a
process that has given all of HBM to its own pool, or a solver that must not
stall on the device synchronisation an allocation can bring.  Its scratch is a
fixed file-scope device array (nbf <= 512).  Its results must equal those of
iqcp_jk_device, on two calls in a row (the array keeps the previous call's
contents, so the second call checks that it is cleared).  This file is
collected last so that a failure here does not hide the other tests.
"""
import ctypes

import numpy as np
import pytest

from conftest import random_density

pytestmark = pytest.mark.gpu
FOCK_TOL = 1e-10


def _run(eng, torch, D, noalloc):
    dD = torch.from_numpy(D).to("cuda")
    dJ = torch.empty_like(dD)
    dK = torch.empty_like(dD)
    lib = eng._lib
    fn = lib.iqcp_jk_device_noalloc if noalloc else lib.iqcp_jk_device
    torch.cuda.synchronize()  # the input copy is on torch's stream, the build on the context's own
    rc = fn(eng._h, ctypes.c_void_p(dD.data_ptr()), ctypes.c_void_p(dJ.data_ptr()), ctypes.c_void_p(dK.data_ptr()))
    assert rc == 0, lib.iqcp_last_error(eng._h).decode()
    torch.cuda.synchronize()
    return dJ.cpu().numpy(), dK.cpu().numpy()


@pytest.mark.parametrize("mol,basis", [("H2O", "6-31g*"), ("c1", None)])
def test_noalloc_matches_jk_device_twice(mol, basis):
    torch = pytest.importorskip("torch")
    from iqcp_b200 import BasisSet, FockEngine
    from iqcp_b200.molecules import REFERENCE_MOLECULES, workload
    if basis is None:
        atoms, basis = workload(mol, 0)
    else:
        atoms = REFERENCE_MOLECULES[mol]
    b = BasisSet.build(atoms, basis)
    with FockEngine(b) as eng:
        for seed in (1, 2):
            D = random_density(b.n_basis, seed, 0.05)
            J0, K0 = _run(eng, torch, D, noalloc=False)
            J1, K1 = _run(eng, torch, D, noalloc=True)
            assert np.abs(J1 - J0).max() < FOCK_TOL
            assert np.abs(K1 - K0).max() < FOCK_TOL


def test_noalloc_rejects_large_basis():
    torch = pytest.importorskip("torch")
    from iqcp_b200 import BasisSet, FockEngine
    from iqcp_b200.molecules import workload
    atoms, basis = workload("c5", 0)
    b = BasisSet.build(atoms, basis)
    assert b.n_basis > 512
    with FockEngine(b) as eng:
        n = b.n_basis
        d = torch.zeros((n, n), dtype=torch.float64, device="cuda")
        rc = eng._lib.iqcp_jk_device_noalloc(eng._h, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(d.data_ptr()),
                                             None)
        assert rc == -1
        assert "512" in eng._lib.iqcp_last_error(eng._h).decode()
