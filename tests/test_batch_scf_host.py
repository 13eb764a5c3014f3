"""Host-side pieces of the batched device SCF, run on CPU tensors: canonical
purification reproduces the aufbau projector of an eigensolver, and the
unrolled small-system solver matches LAPACK."""
import numpy as np
import torch

from iqcp_b200.batch_scf import _purify, _solve_spd


def test_purification_matches_eigenprojector():
    rng = np.random.default_rng(0)
    B, n = 4, 30
    mats, nocc = [], []
    for b in range(B):
        # core-like levels far below, a gap at the Fermi level
        k = 5 + b
        ev = np.concatenate([rng.uniform(-80, -1, k), rng.uniform(0.2, 5, n - k)])
        Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
        mats.append((Q * ev) @ Q.T)
        nocc.append(k)
    P = _purify(torch.tensor(np.array(mats)), torch.tensor(nocc), 64).numpy()
    for b in range(B):
        w, U = np.linalg.eigh(mats[b])
        ref = U[:, : nocc[b]] @ U[:, : nocc[b]].T
        assert np.abs(P[b] - ref).max() < 1e-11
        assert abs(np.trace(P[b]) - nocc[b]) < 1e-10


def test_solve_spd_matches_lapack():
    rng = np.random.default_rng(1)
    A = rng.standard_normal((5, 8, 8))
    A = A @ A.transpose(0, 2, 1) + 0.1 * np.eye(8)
    b = rng.standard_normal((5, 8))
    x = _solve_spd(torch.tensor(A), torch.tensor(b)).numpy()
    np.testing.assert_allclose(x, np.linalg.solve(A, b[..., None])[..., 0], rtol=1e-10, atol=1e-12)
