"""CPU oracle: TEST INFRASTRUCTURE ONLY.

ctypes binding of ``oracle/liboracle.so``, a plain C++ restatement of the
reference's FP64 path (Boys, RDK Rys roots, shell-quartet ERIs, Schwarz,
stored and direct J/K, ERI derivatives, fused two-electron gradient) plus the
one-electron support integrals needed for end-to-end energies and gradients.
Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use it, as the checker; the product library never does.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_dp_t = ctypes.POINTER(ctypes.c_double)
_ip_t = ctypes.POINTER(ctypes.c_int)
_llp_t = ctypes.POINTER(ctypes.c_longlong)


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        B = [ctypes.c_int, _ip_t, _ip_t, _ip_t, _dp_t, _dp_t, _dp_t, ctypes.c_int, _dp_t, _ip_t]
        sig = {
            "or_set_threads": (None, [ctypes.c_int]),
            "or_max_threads": (ctypes.c_int, []),
            "or_boys_all": (None, [ctypes.c_int, ctypes.c_double, _dp_t]),
            "or_rys_roots": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, _dp_t, _dp_t]),
            "or_set_root_precision": (None, [ctypes.c_int]),
            "or_root_precision": (ctypes.c_int, []),
            "or_cart_norm": (ctypes.c_double, [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
            "or_shell_eri": (None, B + [ctypes.c_int] * 4 + [_dp_t, _llp_t]),
            "or_shell_eri_deriv": (None, B + [ctypes.c_int] * 4 + [_dp_t]),
            "or_schwarz": (None, B + [_dp_t]),
            "or_eri_compressed": (None, B + [_dp_t, _llp_t]),
            "or_build_fock": (None, [ctypes.c_int, _dp_t, _dp_t, _dp_t, _dp_t]),
            "or_build_jk_stored": (None, [ctypes.c_int, _dp_t, _dp_t, _dp_t, _dp_t]),
            "or_jk_direct": (None, B + [_dp_t, _dp_t, _dp_t, ctypes.c_int, ctypes.c_int, _llp_t]),
            "or_eri_gradient": (None, B + [_dp_t, ctypes.c_double, _dp_t, ctypes.c_int, ctypes.c_int, _llp_t]),
            "or_one_electron": (None, B + [ctypes.c_int, _dp_t]),
            "or_one_electron_gradient": (None, B + [_dp_t, _dp_t, _dp_t]),
            "or_nuclear_repulsion": (ctypes.c_double, B),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def _dp(a):
    return a.ctypes.data_as(_dp_t)


def _basis_args(b):
    ns, l, nprim, aos, center, exps, coefs, na, xyz, z = b.as_args()
    return (ns, l.ctypes.data_as(_ip_t), nprim.ctypes.data_as(_ip_t), aos.ctypes.data_as(_ip_t), _dp(center),
            _dp(exps), _dp(coefs), na, _dp(xyz), z.ctypes.data_as(_ip_t))


def set_threads(n):
    lib().or_set_threads(int(n))


def max_threads():
    return lib().or_max_threads()


def set_root_precision(extended):
    """Rys roots in the reference's double arithmetic (False, the default) or
    the same algorithm in long double (True), for every later call."""
    lib().or_set_root_precision(1 if extended else 0)


def root_precision():
    return bool(lib().or_root_precision())


def boys_all(m_max, t):
    f = np.zeros(m_max + 1)
    lib().or_boys_all(m_max, float(t), _dp(f))
    return f


def rys_roots(n, t):
    """(status, roots t^2, weights) -- status != 0 is the reference's RysError."""
    r = np.zeros(n)
    w = np.zeros(n)
    rc = lib().or_rys_roots(n, float(t), _dp(r), _dp(w))
    return rc, r, w


def cart_norm(alpha, i, j, k):
    return lib().or_cart_norm(alpha, i, j, k)


def _ncart(l):
    return (l + 1) * (l + 2) // 2


def shell_eri(b, si, sj, sk, sl):
    n = [_ncart(int(b.l[s])) for s in (si, sj, sk, sl)]
    out = np.zeros(n)
    cnt = np.zeros(3, np.int64)
    lib().or_shell_eri(*_basis_args(b), si, sj, sk, sl, _dp(out), cnt.ctypes.data_as(_llp_t))
    return out, cnt


def shell_eri_deriv(b, si, sj, sk, sl):
    n = [_ncart(int(b.l[s])) for s in (si, sj, sk, sl)]
    out = np.zeros([13] + n)
    lib().or_shell_eri_deriv(*_basis_args(b), si, sj, sk, sl, _dp(out))
    return out


def schwarz(b):
    q = np.zeros((b.n_shells, b.n_shells))
    lib().or_schwarz(*_basis_args(b), _dp(q))
    return q


def eri_compressed(b):
    n = b.n_basis
    npair = n * (n + 1) // 2
    out = np.zeros(npair * (npair + 1) // 2)
    cnt = np.zeros(3, np.int64)
    lib().or_eri_compressed(*_basis_args(b), _dp(out), cnt.ctypes.data_as(_llp_t))
    return out, cnt


def build_fock(H, D, eri):
    n = H.shape[0]
    F = np.zeros((n, n))
    lib().or_build_fock(n, _dp(np.ascontiguousarray(H)), _dp(np.ascontiguousarray(D)), _dp(eri), _dp(F))
    return F


def build_jk_stored(D, eri):
    n = D.shape[0]
    J = np.zeros((n, n))
    K = np.zeros((n, n))
    lib().or_build_jk_stored(n, _dp(np.ascontiguousarray(D)), _dp(eri), _dp(J), _dp(K))
    return J, K


def jk_direct(b, D, stride=1, phase=0):
    """Direct J/K with the reference's shell_eri numerics; counters = [rys failures,
    T=0 fallbacks, primitive quartets, shell quartets]."""
    n = b.n_basis
    J = np.zeros((n, n))
    K = np.zeros((n, n))
    cnt = np.zeros(4, np.int64)
    lib().or_jk_direct(*_basis_args(b), _dp(np.ascontiguousarray(D)), _dp(J), _dp(K), stride, phase,
                       cnt.ctypes.data_as(_llp_t))
    return J, K, cnt


def eri_gradient(b, D, hf_frac=1.0, stride=1, phase=0):
    g = np.zeros((b.n_atoms, 3))
    cnt = np.zeros(3, np.int64)
    lib().or_eri_gradient(*_basis_args(b), _dp(np.ascontiguousarray(D)), float(hf_frac), _dp(g), stride, phase,
                          cnt.ctypes.data_as(_llp_t))
    return g, cnt


def one_electron(b, kind):
    """kind: 'S' overlap, 'T' kinetic, 'V' nuclear attraction."""
    n = b.n_basis
    out = np.zeros((n, n))
    lib().or_one_electron(*_basis_args(b), {"S": 0, "T": 1, "V": 2}[kind], _dp(out))
    return out


def hcore(b):
    return one_electron(b, "T") + one_electron(b, "V")


def one_electron_gradient(b, D, W):
    g = np.zeros((b.n_atoms, 3))
    lib().or_one_electron_gradient(*_basis_args(b), _dp(np.ascontiguousarray(D)), _dp(np.ascontiguousarray(W)),
                                   _dp(g))
    return g


def nuclear_repulsion(b):
    return lib().or_nuclear_repulsion(*_basis_args(b))
