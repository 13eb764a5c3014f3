"""The oracle's Rys roots: the reference's double-precision moment method and
the same algorithm in extended precision, against a 50-digit evaluation.

The reference computes the n-point rule from the Boys moments by Schmidt
orthogonalisation and the roots of the orthogonal polynomial (rys/mod.rs:
253-286, 468-660); the Hankel conditioning costs digits as n grows.  The
extended form (oracle.set_root_precision) is the checker for large workloads,
where those digits add up over billions of quartets.  The 50-digit rule comes
from the moments by Golub-Welsch on the Cholesky factor of the Hankel matrix
(mpmath)."""
import numpy as np
import pytest

import oracle

mp = pytest.importorskip("mpmath")


def rule_mp(n, T):
    mp.mp.dps = 50
    T = mp.mpf(T)
    m = [mp.quad(lambda t: t ** (2 * k) * mp.e ** (-T * t * t), [0, 1]) for k in range(2 * n + 1)]
    H = mp.matrix(n + 1, n + 1)
    for i in range(n + 1):
        for j in range(n + 1):
            H[i, j] = m[i + j]
    R = mp.cholesky(H).T
    a = [R[j, j + 1] / R[j, j] - (R[j - 1, j] / R[j - 1, j - 1] if j > 0 else 0) for j in range(n)]
    b = [R[j + 1, j + 1] / R[j, j] for j in range(n - 1)]
    Jm = mp.matrix(n, n)
    for i in range(n):
        Jm[i, i] = a[i]
        if i < n - 1:
            Jm[i, i + 1] = Jm[i + 1, i] = b[i]
    E, Q = mp.eighe(Jm)
    order = sorted(range(n), key=lambda i: E[i])
    return (np.array([float(E[i]) for i in order]), np.array([float(m[0] * Q[0, i] ** 2) for i in order]))


def rel_err(n, T):
    rc, r, w = oracle.rys_roots(n, T)
    assert rc == 0
    rx, wx = rule_mp(n, T)
    return max(np.max(np.abs(r - rx) / rx), np.max(np.abs(w - wx) / wx))


@pytest.mark.parametrize("n,T", [(5, 3.91e-4), (5, 0.3), (5, 7.0), (6, 0.384), (6, 12.0)])
def test_extended_roots_accurate(n, T):
    oracle.set_root_precision(True)
    try:
        e = rel_err(n, T)
    finally:
        oracle.set_root_precision(False)
    assert e < 2e-13, e


def test_double_roots_lose_digits_at_five_roots():
    """What the extended form is for: in double, the reference's method is
    ~1e-11 off at five roots for small T (the C5 J/K deviation's source)."""
    assert not oracle.root_precision()
    e = rel_err(5, 3.91e-4)
    assert 1e-13 < e < 1e-9, e


def test_double_path_unchanged_by_switch():
    """Switching back restores the reference arithmetic bit for bit."""
    rc0, r0, w0 = oracle.rys_roots(4, 1.7)
    oracle.set_root_precision(True)
    oracle.rys_roots(4, 1.7)
    oracle.set_root_precision(False)
    rc1, r1, w1 = oracle.rys_roots(4, 1.7)
    assert rc0 == rc1 == 0 and r0.tobytes() == r1.tobytes() and w0.tobytes() == w1.tobytes()
