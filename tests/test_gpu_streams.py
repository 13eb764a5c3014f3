"""Concurrent class launches (the context stream plus three side streams,
forked and joined with events) against the serialised form (profiling on),
and their ordering with the caller's stream: a density written on the
caller's stream just before a call is the one the kernels read, and work
queued just after a call sees the finished J, K and gradient."""
import numpy as np
import pytest
import torch

from conftest import random_density
from iqcp_b200 import BasisSet, FockEngine
from iqcp_b200.molecules import workload

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    atoms, basis = workload("c2", 0)     # 21 class launches per call
    b = BasisSet.build(atoms, basis)
    eng = FockEngine(b)
    yield b, eng
    eng.close()


def _device_call(eng, b, D, stream):
    dD = torch.from_numpy(D).cuda()
    dJ, dK = torch.empty_like(dD), torch.empty_like(dD)
    dg = torch.zeros((b.n_atoms, 3), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    eng.jk_device(dD.data_ptr(), dJ.data_ptr(), dK.data_ptr())
    eng.eri_gradient_device(dD.data_ptr(), 1.0, dg.data_ptr())
    torch.cuda.synchronize()
    return dJ.cpu().numpy(), dK.cpu().numpy(), dg.cpu().numpy()


def test_concurrent_matches_serialised(engine):
    b, eng = engine
    stream = torch.cuda.current_stream()
    eng.set_stream(stream.cuda_stream)
    D = random_density(b.n_basis, 7, 0.05)
    J0, K0, g0 = _device_call(eng, b, D, stream)
    eng.set_profiling(True)          # one stream: every launch timed alone
    try:
        J1, K1, g1 = _device_call(eng, b, D, stream)
    finally:
        eng.set_profiling(False)
    # the same quartets, added in another order
    assert np.abs(J0 - J1).max() < 1e-12 and np.abs(K0 - K1).max() < 1e-12
    assert np.abs(g0 - g1).max() < 1e-12


def test_ordering_with_caller_stream(engine):
    b, eng = engine
    side = torch.cuda.Stream()
    eng.set_stream(side.cuda_stream)
    D1 = random_density(b.n_basis, 8, 0.05)
    D2 = random_density(b.n_basis, 9, 0.05)
    J2, K2, g2 = _device_call(eng, b, D2, side)
    with torch.cuda.stream(side):
        dD = torch.from_numpy(D1).cuda()
        dD2 = torch.from_numpy(D2).cuda()
        dJ, dK = torch.empty_like(dD), torch.empty_like(dD)
        dg = torch.zeros((b.n_atoms, 3), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        for _ in range(3):
            torch.cuda._sleep(2_000_000)        # keep the stream busy, then overwrite D on it
            dD.copy_(dD2)
            eng.jk_device(dD.data_ptr(), dJ.data_ptr(), dK.data_ptr())
            dJ.mul_(2.0)                        # queued after the call: must see the finished J
            dg.zero_()
            eng.eri_gradient_device(dD.data_ptr(), 1.0, dg.data_ptr())
            dg.mul_(-1.0)
            side.synchronize()
            assert np.abs(dJ.cpu().numpy() - 2.0 * J2).max() < 1e-12
            assert np.abs(dK.cpu().numpy() - K2).max() < 1e-12
            assert np.abs(dg.cpu().numpy() + g2).max() < 1e-12
            dD.copy_(torch.from_numpy(D1).cuda())
    eng.set_stream(torch.cuda.current_stream().cuda_stream)
