"""Device Boys function and Rys rule against the oracle (reference algorithm)
and the golden vectors."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

TS = np.concatenate([[0.0, 1e-15, 1e-12, 1e-9, 1e-6], np.geomspace(1e-4, 2e3, 1500),
                     np.linspace(0, 80, 801)[1:], [35.999, 36.0, 36.001, 62.999, 63.0, 63.001]])


def test_device_boys_vs_oracle(oracle_mod):
    import iqcp_b200 as iq
    for m in (2, 4, 8, 12, 16):
        F = iq.boys_eval_all(m, TS)
        Fo = np.array([oracle_mod.boys_all(m, t) for t in TS])
        np.testing.assert_allclose(F, Fo, rtol=5e-13, atol=1e-300)


def test_device_boys_golden():
    import iqcp_b200 as iq
    for m, T, v in golden("boys.json")["values"]:
        f = iq.boys_eval_all(max(m, 2), [T])[0, m]
        assert abs(f - v) <= (1e-6 * abs(v) if abs(v) < 1e-10 else 1e-12), (m, T)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 7])
def test_device_rys_moments(oracle_mod, n):
    """Gauss property: sum_k w_k x_k^m = F_m(T) for m < 2n (relative to F_m)."""
    import iqcp_b200 as iq
    R, W = iq.rys_roots(n, TS)
    assert np.all(R >= 0) and np.all(R < 1) and np.all(W > 0)
    worst = 0.0
    for i, t in enumerate(TS):
        F = oracle_mod.boys_all(2 * n, t)
        for m in range(2 * n):
            worst = max(worst, abs(np.sum(W[i] * R[i] ** m) - F[m]) / F[m])
    assert worst < (2e-13 if n <= 6 else 5e-13), worst


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6])
def test_device_rys_vs_reference_rdk(oracle_mod, n):
    """Table rule vs the reference's per-call RDK: they differ by the RDK's own
    error, which grows with n (moment method, rys/mod.rs:468-660)."""
    import iqcp_b200 as iq
    R, W = iq.rys_roots(n, TS)
    tol = {1: 1e-13, 2: 1e-12, 3: 1e-11, 4: 1e-10, 5: 2e-9, 6: 5e-8}[n]
    for i, t in enumerate(TS):
        rc, r, w = oracle_mod.rys_roots(n, t)
        assert rc == 0
        np.testing.assert_allclose(R[i], r, rtol=tol, atol=1e-300)
        np.testing.assert_allclose(W[i], w, rtol=tol, atol=1e-300)
