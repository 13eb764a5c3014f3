"""The J/K entry point that allocates nothing (iqcp_jk_device_noalloc).

It exists for callers whose Fock-build loop may not call cudaMalloc: a
process that has given all of HBM to its own pool, or a solver that must not
stall on the device synchronisation an allocation can bring.  Its scratch is a
fixed file-scope device array (nbf <= 512).  Its results must equal those of
iqcp_jk_device, in both precisions, on two calls in a row (the array keeps the
previous call's contents, so the second call checks that it is cleared), and
the C1 workload's are checked against the oracle too.  This file is collected
last so that a failure here does not hide the other tests.
"""
import ctypes

import numpy as np
import pytest

from conftest import random_density

pytestmark = pytest.mark.gpu
FOCK_TOL = 1e-10


def _run(eng, torch, D, noalloc, want_k=True):
    dD = torch.from_numpy(D).to("cuda")
    dJ = torch.empty_like(dD)
    dK = torch.empty_like(dD)
    lib = eng._lib
    fn = lib.iqcp_jk_device_noalloc if noalloc else lib.iqcp_jk_device
    torch.cuda.synchronize()  # the input copy is on torch's stream, the build on the context's own
    rc = fn(eng._h, ctypes.c_void_p(dD.data_ptr()), ctypes.c_void_p(dJ.data_ptr()),
            ctypes.c_void_p(dK.data_ptr()) if want_k else None)
    assert rc == 0, lib.iqcp_last_error(eng._h).decode()
    torch.cuda.synchronize()  # device-wide: the call returns once enqueued on the context stream
    return dJ.cpu().numpy(), dK.cpu().numpy() if want_k else None


def _basis(mol, basis):
    from iqcp_b200 import BasisSet
    from iqcp_b200.molecules import REFERENCE_MOLECULES, workload
    if basis is None:
        atoms, basis = workload(mol, 0)
    else:
        atoms = REFERENCE_MOLECULES[mol]
    return BasisSet.build(atoms, basis)


@pytest.mark.parametrize("mol,basis", [("H2O", "6-31g*"), ("c1", None)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_matches_jk_device_twice(mol, basis, precision):
    torch = pytest.importorskip("torch")
    from iqcp_b200 import FockEngine, MIXED
    b = _basis(mol, basis)
    with FockEngine(b) as eng:
        if precision == "mixed":
            eng.set_precision(MIXED, 1e-3)
            eng.set_kernel_mode("jk32", mode=0)  # every class split into FP64 + FP32 passes
        for seed in (1, 2):
            D = random_density(b.n_basis, seed, 0.05)
            J0, K0 = _run(eng, torch, D, noalloc=False)
            J1, K1 = _run(eng, torch, D, noalloc=True)
            assert np.abs(J1 - J0).max() < FOCK_TOL
            assert np.abs(K1 - K0).max() < FOCK_TOL


def test_noalloc_vs_oracle_and_j_only(oracle_mod):
    torch = pytest.importorskip("torch")
    from iqcp_b200 import FockEngine
    b = _basis("c1", None)
    D = random_density(b.n_basis, 7, 0.05)
    Jo, Ko, _ = oracle_mod.jk_direct(b, D)
    with FockEngine(b) as eng:
        J, K = _run(eng, torch, D, noalloc=True)
        assert np.abs(J - Jo).max() < FOCK_TOL
        assert np.abs(K - Ko).max() < FOCK_TOL
        Jonly, _ = _run(eng, torch, D, noalloc=True, want_k=False)
        assert np.abs(Jonly - Jo).max() < FOCK_TOL


def test_noalloc_allocates_nothing_and_captures():
    """Free device memory is unchanged over repeated calls after the first, and
    a call recorded into a CUDA graph (after an ordinary one) replays to the
    same J/K as iqcp_jk_device."""
    torch = pytest.importorskip("torch")
    from iqcp_b200 import FockEngine
    b = _basis("H2O", "6-31g*")
    n = b.n_basis
    D = random_density(n, 3, 0.05)
    with FockEngine(b) as eng:
        J0, K0 = _run(eng, torch, D, noalloc=False)
        dD = torch.from_numpy(D).to("cuda")
        dJ = torch.zeros_like(dD)
        dK = torch.zeros_like(dD)
        stream = torch.cuda.current_stream()
        eng.set_stream(stream.cuda_stream)
        eng.jk_device_noalloc(dD.data_ptr(), dJ.data_ptr(), dK.data_ptr())
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        for _ in range(5):
            eng.jk_device_noalloc(dD.data_ptr(), dJ.data_ptr(), dK.data_ptr())
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0
        dJ.zero_()
        dK.zero_()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            eng.set_stream(torch.cuda.current_stream().cuda_stream)
            eng.jk_device_noalloc(dD.data_ptr(), dJ.data_ptr(), dK.data_ptr())
        eng.set_stream(stream.cuda_stream)
        g.replay()
        torch.cuda.synchronize()
        assert np.abs(dJ.cpu().numpy() - J0).max() < FOCK_TOL
        assert np.abs(dK.cpu().numpy() - K0).max() < FOCK_TOL
        del g


def test_noalloc_rejects_large_basis_and_batches():
    torch = pytest.importorskip("torch")
    from iqcp_b200 import BatchFockEngine, FockEngine
    b = _basis("c5", None)
    assert b.n_basis > 512
    with FockEngine(b) as eng:
        n = b.n_basis
        d = torch.zeros((n, n), dtype=torch.float64, device="cuda")
        rc = eng._lib.iqcp_jk_device_noalloc(eng._h, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(d.data_ptr()),
                                             None)
        assert rc == -1
        assert "512" in eng._lib.iqcp_last_error(eng._h).decode()
    small = _basis("H2O", "6-31g*")
    with BatchFockEngine([small, small]) as beng:
        d = torch.zeros(beng.packed_size, dtype=torch.float64, device="cuda")
        rc = beng._lib.iqcp_jk_device_noalloc(beng._h, ctypes.c_void_p(d.data_ptr()),
                                              ctypes.c_void_p(d.data_ptr()), None)
        assert rc == -1
        assert "single-geometry" in beng._lib.iqcp_last_error(beng._h).decode()
