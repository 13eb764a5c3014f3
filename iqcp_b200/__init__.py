"""iqcp_b200: B200-native direct Fock build and two-electron gradient.

Thin ctypes binding of ``libiqcp_gpu.so`` (C ABI in ``include/iqcp.h``).  The
names mirror the reference's qc-core entry points on this path:

=============================  ==================================================
here                           reference (ExaPsi/IQCP crates/qc-core)
=============================  ==================================================
``BasisSet.build``             ``BasisSet::build`` (basis/mod.rs:164)
``FockEngine.build_jk``        ``build_jk`` (dft/ks_scf.rs:1369)
``FockEngine.build_fock``      ``build_fock`` (scf/mod.rs:825)
``FockEngine.eri_gradient``    ``eri_gradient_fused`` (scf/gradient.rs:1430)
``FockEngine.eri_compressed``  ``eri_compressed`` (integrals/eri/mod.rs:992)
``FockEngine.schwarz``         ``compute_schwarz_bounds`` (eri/mod.rs:1263)
``boys_eval_all``              ``boys_eval_all`` (boys/mod.rs:327), batched
``rys_roots``                  ``rys_roots`` (rys/mod.rs:253), batched
=============================  ==================================================

There is no CPU fallback: every compute call goes to the CUDA library and
raises ``IqcpError`` when the library or a B200 is missing.
"""
import ctypes
import os

import numpy as np

__all__ = ["BasisSet", "FockEngine", "BatchFockEngine", "IqcpError", "ScfOptions", "boys_eval_all", "rys_roots",
           "lib_path", "load_library", "ANGSTROM_TO_BOHR", "FP64", "MIXED"]

ANGSTROM_TO_BOHR = 1.8897261245650618  # constants.rs:63
FP64, MIXED = 0, 1
_CUDA_STREAM_LEGACY = 0x1   # cudaStreamLegacy

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_dbl_p = ctypes.POINTER(ctypes.c_double)

STATUS = {0: "ok", -1: "invalid argument", -2: "CUDA error", -3: "out of memory",
          -4: "non-finite value", -5: "no usable sm_100 device", -6: "unknown basis or element"}


class IqcpError(RuntimeError):
    """A libiqcp_gpu call returned a non-zero status."""

    def __init__(self, code, msg=""):
        self.code = code
        super().__init__("iqcp status %d (%s)%s" % (code, STATUS.get(code, "?"), (": " + msg) if msg else ""))


class _BasisDesc(ctypes.Structure):
    _fields_ = [("n_shells", ctypes.c_int), ("n_atoms", ctypes.c_int),
                ("l", _c_int_p), ("nprim", _c_int_p), ("atom_of_shell", _c_int_p),
                ("center", _c_dbl_p), ("exps", _c_dbl_p), ("coefs", _c_dbl_p),
                ("atom_xyz", _c_dbl_p), ("z", _c_int_p)]


class _Options(ctypes.Structure):
    _fields_ = [("schwarz_threshold", ctypes.c_double), ("prim_threshold", ctypes.c_double),
                ("precision", ctypes.c_int), ("mixed_cutoff", ctypes.c_double), ("device", ctypes.c_int)]


class ScfOptions(ctypes.Structure):
    """iqcp_scf_options of include/iqcp.h."""
    _fields_ = [("e_tol", ctypes.c_double), ("d_tol", ctypes.c_double), ("err_tol", ctypes.c_double),
                ("max_iter", ctypes.c_int), ("diis_size", ctypes.c_int), ("purify_iters", ctypes.c_int)]


def lib_path():
    return os.path.join(_HERE, "libiqcp_gpu.so")


EXPORTS = {
    "iqcp_default_options": (None, [ctypes.POINTER(_Options)]),
    "iqcp_basis_build": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, _c_int_p, _c_dbl_p, _c_int_p, _c_int_p,
                                        _c_int_p, _c_int_p, _c_int_p, _c_int_p, _c_dbl_p, _c_dbl_p, _c_dbl_p]),
    "iqcp_create": (ctypes.c_int, [ctypes.POINTER(_BasisDesc), ctypes.POINTER(_Options),
                                   ctypes.POINTER(ctypes.c_void_p)]),
    "iqcp_destroy": (None, [ctypes.c_void_p]),
    "iqcp_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "iqcp_nbf": (ctypes.c_int, [ctypes.c_void_p]),
    "iqcp_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "iqcp_set_precision": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]),
    "iqcp_jk": (ctypes.c_int, [ctypes.c_void_p, _c_dbl_p, _c_dbl_p, _c_dbl_p]),
    "iqcp_fock": (ctypes.c_int, [ctypes.c_void_p, _c_dbl_p, _c_dbl_p, ctypes.c_double, _c_dbl_p]),
    "iqcp_jk_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "iqcp_fock_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                        ctypes.c_void_p]),
    "iqcp_eri_grad": (ctypes.c_int, [ctypes.c_void_p, _c_dbl_p, ctypes.c_double, _c_dbl_p]),
    "iqcp_eri_grad_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]),
    "iqcp_eri_compressed": (ctypes.c_int, [ctypes.c_void_p, _c_dbl_p, ctypes.c_longlong]),
    "iqcp_schwarz": (ctypes.c_int, [ctypes.c_void_p, _c_dbl_p]),
    "iqcp_one_electron": (ctypes.c_int, [ctypes.c_void_p, _c_dbl_p, _c_dbl_p, _c_dbl_p]),
    "iqcp_boys_batch": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _c_dbl_p, _c_dbl_p]),
    "iqcp_rys_batch": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _c_dbl_p, _c_dbl_p, _c_dbl_p]),
    "iqcp_last_stats": (ctypes.c_int, [ctypes.c_void_p, _c_dbl_p]),
    "iqcp_jk_device_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "iqcp_set_profiling": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "iqcp_launch_profile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _c_int_p, _c_int_p, _c_int_p, _c_dbl_p,
                                           ctypes.POINTER(ctypes.c_longlong)]),
    "iqcp_kernel_launches": (ctypes.c_int, [ctypes.c_void_p]),
    "iqcp_model_flops": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _c_dbl_p, ctypes.POINTER(ctypes.c_longlong),
                                        ctypes.POINTER(ctypes.c_longlong)]),
    "iqcp_measure_peak": (ctypes.c_int, [ctypes.c_int, _c_dbl_p]),
    "iqcp_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "iqcp_kernel_modes": (ctypes.c_int, [ctypes.c_void_p, _c_int_p]),
    "iqcp_set_kernel_mode": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "iqcp_one_electron_grad": (ctypes.c_int, [ctypes.c_void_p, _c_dbl_p, _c_dbl_p, _c_dbl_p]),
    "iqcp_one_electron_grad_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                     ctypes.c_void_p]),
    "iqcp_rhf_gradient": (ctypes.c_int, [ctypes.c_void_p, _c_dbl_p, _c_dbl_p, _c_dbl_p]),
    "iqcp_create_batch": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_BasisDesc), ctypes.POINTER(_Options),
                                         ctypes.POINTER(ctypes.c_void_p)]),
    "iqcp_batch_layout": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong), _c_int_p, _c_int_p]),
    "iqcp_jk_multi": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _c_dbl_p, _c_dbl_p, _c_dbl_p]),
    "iqcp_jk_multi_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_void_p]),
    "iqcp_fock_decomposition": (ctypes.c_int, [ctypes.c_void_p, _c_dbl_p, _c_dbl_p, ctypes.c_double, _c_dbl_p,
                                               _c_dbl_p, _c_dbl_p, _c_dbl_p]),
    "iqcp_nbf_spherical": (ctypes.c_int, [ctypes.c_void_p]),
    "iqcp_jk_spherical": (ctypes.c_int, [ctypes.c_void_p, _c_dbl_p, _c_dbl_p, _c_dbl_p]),
    "iqcp_scf_default_options": (None, [ctypes.POINTER(ScfOptions)]),
    "iqcp_batch_scf": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ScfOptions), _c_dbl_p, _c_dbl_p, _c_int_p,
                                      _c_int_p, _c_dbl_p, _c_dbl_p]),
    "iqcp_sad_density": (ctypes.c_int, [ctypes.POINTER(_BasisDesc), ctypes.POINTER(_Options), _c_dbl_p]),
}

PAIR_CLASSES = ["ss", "ps", "pp", "ds", "dp", "dd"]


def load_library():
    """Load libiqcp_gpu.so from the package directory (raises if it is missing)."""
    global _LIB
    if _LIB is None:
        path = lib_path()
        if not os.path.exists(path):
            raise IqcpError(-5, "libiqcp_gpu.so not built (run __graft_entry__.build())")
        lib = ctypes.CDLL(path)
        for name, (res, args) in EXPORTS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def _dp(a):
    return a.ctypes.data_as(_c_dbl_p)


def _ip(a):
    return a.ctypes.data_as(_c_int_p)


class BasisSet:
    """Cartesian Gaussian basis for a molecule, in qc-core's shell order."""

    def __init__(self, name, z, xyz, l, nprim, atom_of_shell, center, exps, coefs):
        self.name = name
        self.z = np.ascontiguousarray(z, dtype=np.int32)
        self.xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        self.l = np.ascontiguousarray(l, dtype=np.int32)
        self.nprim = np.ascontiguousarray(nprim, dtype=np.int32)
        self.atom_of_shell = np.ascontiguousarray(atom_of_shell, dtype=np.int32)
        self.center = np.ascontiguousarray(center, dtype=np.float64).reshape(-1, 3)
        self.exps = np.ascontiguousarray(exps, dtype=np.float64)
        self.coefs = np.ascontiguousarray(coefs, dtype=np.float64)
        ncart = (self.l + 1) * (self.l + 2) // 2
        self.offsets = np.concatenate([[0], np.cumsum(ncart)[:-1]]).astype(np.int32)
        self.n_basis = int(ncart.sum())
        self.n_electrons = int(self.z.sum())

    @property
    def n_shells(self):
        return len(self.l)

    @property
    def n_atoms(self):
        return len(self.z)

    @classmethod
    def build(cls, atoms, basis_name):
        """atoms: list of (Z, (x, y, z) in bohr) -- BasisSet::build (basis/mod.rs:164)."""
        lib = load_library()
        z = np.array([a[0] for a in atoms], dtype=np.int32)
        xyz = np.array([a[1] for a in atoms], dtype=np.float64).reshape(-1, 3)
        ns, npr, nb = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        name = basis_name.encode()
        rc = lib.iqcp_basis_build(name, len(z), _ip(z), _dp(xyz), ctypes.byref(ns), ctypes.byref(npr),
                                  ctypes.byref(nb), None, None, None, None, None, None)
        if rc:
            raise IqcpError(rc, "basis %r" % basis_name)
        l = np.zeros(ns.value, np.int32)
        nprim = np.zeros(ns.value, np.int32)
        aos = np.zeros(ns.value, np.int32)
        center = np.zeros((ns.value, 3))
        exps = np.zeros(npr.value)
        coefs = np.zeros(npr.value)
        rc = lib.iqcp_basis_build(name, len(z), _ip(z), _dp(xyz), ctypes.byref(ns), ctypes.byref(npr),
                                  ctypes.byref(nb), _ip(l), _ip(nprim), _ip(aos), _dp(center), _dp(exps),
                                  _dp(coefs))
        if rc:
            raise IqcpError(rc)
        return cls(basis_name.lower(), z, xyz, l, nprim, aos, center, exps, coefs)

    def nuclear_repulsion(self):
        e = 0.0
        for i in range(self.n_atoms):
            for j in range(i):
                e += self.z[i] * self.z[j] / np.linalg.norm(self.xyz[i] - self.xyz[j])
        return float(e)

    def as_args(self):
        """Plain arrays in the C ABI's shell layout (also used by the oracle)."""
        return (self.n_shells, self.l, self.nprim, self.atom_of_shell, self.center, self.exps, self.coefs,
                self.n_atoms, self.xyz, self.z)

    def sad_density(self, device=0):
        """SAD initial density (iqcp_sad_density; build_sad_density, scf/sad.rs:698):
        superposed spherically averaged atomic RHF densities, nbf x nbf."""
        lib = load_library()
        opts = _Options()
        lib.iqcp_default_options(ctypes.byref(opts))
        opts.device = device
        D = np.empty((self.n_basis, self.n_basis))
        desc = self._desc()
        rc = lib.iqcp_sad_density(ctypes.byref(desc), ctypes.byref(opts), _dp(D))
        if rc:
            raise IqcpError(rc, "iqcp_sad_density")
        return D

    def _desc(self):
        d = _BasisDesc()
        d.n_shells, d.n_atoms = self.n_shells, self.n_atoms
        d.l, d.nprim, d.atom_of_shell = _ip(self.l), _ip(self.nprim), _ip(self.atom_of_shell)
        d.center, d.exps, d.coefs = _dp(self.center), _dp(self.exps), _dp(self.coefs)
        d.atom_xyz, d.z = _dp(self.xyz), _ip(self.z)
        return d


class FockEngine:
    """A per-geometry context of libiqcp_gpu (iqcp_create ... iqcp_destroy)."""

    def __init__(self, basis, precision=FP64, schwarz_threshold=1e-12, prim_threshold=1e-15,
                 mixed_cutoff=1e-9, device=0):
        lib = load_library()
        self._lib = lib
        self.basis = basis
        opts = _Options()
        lib.iqcp_default_options(ctypes.byref(opts))
        opts.schwarz_threshold = schwarz_threshold
        opts.prim_threshold = prim_threshold
        opts.precision = precision
        opts.mixed_cutoff = mixed_cutoff
        opts.device = device
        self._desc = basis._desc()
        h = ctypes.c_void_p()
        rc = lib.iqcp_create(ctypes.byref(self._desc), ctypes.byref(opts), ctypes.byref(h))
        self._h = h
        if rc:
            msg = lib.iqcp_last_error(h).decode() if h.value else ""
            self.close()
            raise IqcpError(rc, msg)
        self.nbf = lib.iqcp_nbf(h)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.iqcp_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        if rc:
            raise IqcpError(rc, self._lib.iqcp_last_error(self._h).decode())

    def _mat(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape != (self.nbf, self.nbf):
            raise ValueError("expected a %dx%d matrix" % (self.nbf, self.nbf))
        return a

    def build_jk(self, D, with_k=True):
        D = self._mat(D)
        J = np.empty_like(D)
        K = np.empty_like(D) if with_k else None
        self._check(self._lib.iqcp_jk(self._h, _dp(D), _dp(J), _dp(K) if with_k else None))
        return (J, K) if with_k else J

    def build_fock(self, H, D, k_scale=1.0):
        H, D = self._mat(H), self._mat(D)
        F = np.empty_like(D)
        self._check(self._lib.iqcp_fock(self._h, _dp(H), _dp(D), float(k_scale), _dp(F)))
        return F

    def build_jk_multi(self, Ds, with_k=True):
        """J and K of several symmetric densities with one pass over the quartets
        (iqcp_jk_multi): the response-density J/K of gen_vind_rhf (scf/cphf.rs:828)."""
        D = np.ascontiguousarray(np.stack([self._mat(d) for d in Ds]))
        J = np.empty_like(D)
        K = np.empty_like(D) if with_k else None
        self._check(self._lib.iqcp_jk_multi(self._h, len(D), _dp(D), _dp(J), _dp(K) if with_k else None))
        return (list(J), list(K)) if with_k else list(J)

    def jk_multi_device(self, nset, d_D, d_J, d_K=None):
        self._check(self._lib.iqcp_jk_multi_device(self._h, int(nset), ctypes.c_void_p(d_D), ctypes.c_void_p(d_J),
                                                   ctypes.c_void_p(d_K) if d_K else None))

    def build_jk_spherical(self, D, with_k=True):
        """J and K in the spherical basis (nsph x nsph, m = -l..l per shell):
        the reference's use_spherical path (EriSphericalTransform, spherical.rs:390)."""
        n = self._lib.iqcp_nbf_spherical(self._h)
        D = np.ascontiguousarray(D, dtype=np.float64)
        if D.shape != (n, n):
            raise ValueError("expected a %dx%d matrix" % (n, n))
        J = np.empty_like(D)
        K = np.empty_like(D) if with_k else None
        self._check(self._lib.iqcp_jk_spherical(self._h, _dp(D), _dp(J), _dp(K) if with_k else None))
        return (J, K) if with_k else J

    def fock_decomposition(self, H, D, k_scale=1.0):
        """(J, K, G, F) with G = J - k_scale/2 K, F = H + G: compute_fock_decomposition
        (scf/fock.rs:104-179)."""
        H, D = self._mat(H), self._mat(D)
        J, K, G, F = (np.empty_like(D) for _ in range(4))
        self._check(self._lib.iqcp_fock_decomposition(self._h, _dp(H), _dp(D), float(k_scale), _dp(J), _dp(K),
                                                      _dp(G), _dp(F)))
        return J, K, G, F

    def eri_gradient(self, D, hf_frac=1.0):
        D = self._mat(D)
        g = np.zeros((self.basis.n_atoms, 3))
        self._check(self._lib.iqcp_eri_grad(self._h, _dp(D), float(hf_frac), _dp(g)))
        return g

    def eri_compressed(self):
        n = self.nbf
        npair = n * (n + 1) // 2
        out = np.empty(npair * (npair + 1) // 2)
        self._check(self._lib.iqcp_eri_compressed(self._h, _dp(out), out.size))
        return out

    def schwarz(self):
        q = np.zeros((self.basis.n_shells, self.basis.n_shells))
        self._check(self._lib.iqcp_schwarz(self._h, _dp(q)))
        return q

    def one_electron(self):
        """(S, T, V) on the device: overlap_matrix / kinetic / nuclear attraction."""
        n = self.nbf
        S, T, V = np.empty((n, n)), np.empty((n, n)), np.empty((n, n))
        self._check(self._lib.iqcp_one_electron(self._h, _dp(S), _dp(T), _dp(V)))
        return S, T, V

    def one_electron_gradient(self, D, W):
        """Nuclear repulsion + sum D dH - sum W dS (W: energy-weighted density, factor 2)."""
        D, W = self._mat(D), self._mat(W)
        g = np.zeros((self.basis.n_atoms, 3))
        self._check(self._lib.iqcp_one_electron_grad(self._h, _dp(D), _dp(W), _dp(g)))
        return g

    def rhf_gradient(self, D, W):
        """Full RHF nuclear gradient (rhf_gradient, scf/gradient.rs:900-990)."""
        D, W = self._mat(D), self._mat(W)
        g = np.zeros((self.basis.n_atoms, 3))
        self._check(self._lib.iqcp_rhf_gradient(self._h, _dp(D), _dp(W), _dp(g)))
        return g

    def last_stats(self):
        s = np.zeros(4)
        self._check(self._lib.iqcp_last_stats(self._h, _dp(s)))
        return {"quartets": int(s[0]), "launches": int(s[1]), "kernel_us": float(s[2]), "fp32_quartets": int(s[3])}

    def set_profiling(self, on=True):
        self._check(self._lib.iqcp_set_profiling(self._h, int(bool(on))))

    def launch_profile(self):
        """Per quartet-kernel launch of the last call: dicts with kind, class, ms, quartets."""
        m = 64
        kind, X, Y = (np.zeros(m, np.int32) for _ in range(3))
        ms = np.zeros(m)
        q = np.zeros(m, np.int64)
        n = self._lib.iqcp_launch_profile(self._h, m, _ip(kind), _ip(X), _ip(Y), _dp(ms),
                                          q.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)))
        return [{"kind": ("jk", "grad", "jk32", "grad32")[kind[i]], "cls": "(%s|%s)" % (PAIR_CLASSES[X[i]], PAIR_CLASSES[Y[i]]),
                 "X": int(X[i]), "Y": int(Y[i]), "ms": float(ms[i]), "quartets": int(q[i])} for i in range(min(n, m))]

    def autotune(self, d_D, reps=2):
        """Pick the fastest quartet-kernel variant per class on this device density pointer."""
        self._check(self._lib.iqcp_autotune(self._h, ctypes.c_void_p(d_D), int(reps)))
        return self.kernel_modes()

    def kernel_modes(self):
        """Variant per [kind, X, Y]; kind 0 J/K, 1 gradient, 2 / 3 their FP32 share
        (mixed form; 4 = the class runs wholly in FP64)."""
        m = np.zeros(144, np.int32)
        self._check(self._lib.iqcp_kernel_modes(self._h, _ip(m)))
        return m.reshape(4, 6, 6)

    def set_kernel_mode(self, kind, X=-1, Y=-1, mode=0):
        k = {"jk": 0, "grad": 1, "jk32": 2, "grad32": 3}[kind]
        self._check(self._lib.iqcp_set_kernel_mode(self._h, k, X, Y, mode))

    def kernel_launches(self):
        return self._lib.iqcp_kernel_launches(self._h)

    def model_flops(self, kind="jk"):
        """Algorithmic FLOPs [6x6] per (bra, ket) pair class, surviving primitive quartets, quartets."""
        f = np.zeros(36)
        p = np.zeros(36, np.int64)
        q = np.zeros(36, np.int64)
        LL = ctypes.POINTER(ctypes.c_longlong)
        self._check(self._lib.iqcp_model_flops(self._h, {"jk": 0, "grad": 1}[kind], _dp(f), p.ctypes.data_as(LL),
                                               q.ctypes.data_as(LL)))
        return f.reshape(6, 6), p.reshape(6, 6), q.reshape(6, 6)

    # device-resident forms (pointers to nbf*nbf doubles in HBM, e.g. torch tensors' data_ptr())
    def jk_device(self, d_D, d_J, d_K=None):
        self._check(self._lib.iqcp_jk_device(self._h, ctypes.c_void_p(d_D), ctypes.c_void_p(d_J),
                                             ctypes.c_void_p(d_K) if d_K else None))

    def jk_device_noalloc(self, d_D, d_J, d_K=None):
        """iqcp_jk_device with its scratch in a fixed device array (nbf <= 512): allocates nothing."""
        self._check(self._lib.iqcp_jk_device_noalloc(self._h, ctypes.c_void_p(d_D), ctypes.c_void_p(d_J),
                                                     ctypes.c_void_p(d_K) if d_K else None))

    def fock_device(self, d_H, d_D, k_scale, d_F):
        self._check(self._lib.iqcp_fock_device(self._h, ctypes.c_void_p(d_H), ctypes.c_void_p(d_D),
                                               float(k_scale), ctypes.c_void_p(d_F)))

    def eri_gradient_device(self, d_D, hf_frac, d_grad):
        self._check(self._lib.iqcp_eri_grad_device(self._h, ctypes.c_void_p(d_D), float(hf_frac),
                                                   ctypes.c_void_p(d_grad)))

    def set_precision(self, precision, mixed_cutoff=1e-9):
        """FP64 (0) or MIXED (1): FP32 quadrature for quartets with Q_ij Q_kl max|D| < mixed_cutoff."""
        self._check(self._lib.iqcp_set_precision(self._h, int(precision), float(mixed_cutoff)))

    def set_stream(self, stream_handle):
        """Enqueue the device forms on this CUDA stream (e.g. torch's
        current_stream().cuda_stream).  Handle 0, torch's default stream, is
        the legacy default stream: it is passed as cudaStreamLegacy, since a
        NULL stream selects the context's own non-blocking stream, which would
        not order with work on the default stream."""
        h = int(stream_handle or 0)
        self._check(self._lib.iqcp_set_stream(self._h, ctypes.c_void_p(h if h else _CUDA_STREAM_LEGACY)))


class BatchFockEngine(FockEngine):
    """One context over many molecules or geometries (iqcp_create_batch).

    Each call covers every molecule with one launch per angular-momentum
    class.  Matrices travel packed: molecule m is the nbf[m] x nbf[m] block at
    offset mat_offset[m] of one flat array; pack()/unpack() convert lists of
    per-molecule matrices.  Gradients come back as a list of [n_atoms_m, 3]
    arrays.
    """

    def __init__(self, bases, precision=FP64, schwarz_threshold=1e-12, prim_threshold=1e-15,
                 mixed_cutoff=1e-9, device=0):
        lib = load_library()
        self._lib = lib
        self.bases = list(bases)
        self.basis = None
        opts = _Options()
        lib.iqcp_default_options(ctypes.byref(opts))
        opts.schwarz_threshold = schwarz_threshold
        opts.prim_threshold = prim_threshold
        opts.precision = precision
        opts.mixed_cutoff = mixed_cutoff
        opts.device = device
        self.device = device
        n = len(self.bases)
        self._descs = (_BasisDesc * n)(*[b._desc() for b in self.bases])
        h = ctypes.c_void_p()
        rc = lib.iqcp_create_batch(n, self._descs, ctypes.byref(opts), ctypes.byref(h))
        self._h = h
        if rc:
            msg = lib.iqcp_last_error(h).decode() if h.value else ""
            self.close()
            raise IqcpError(rc, msg)
        self.n_mol = n
        self.mat_offset = np.zeros(n + 1, np.int64)
        self.nbfs = np.zeros(n, np.int32)
        self.atom_offset = np.zeros(n + 1, np.int32)
        lib.iqcp_batch_layout(h, self.mat_offset.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                              _ip(self.nbfs), _ip(self.atom_offset))
        self.nbf = lib.iqcp_nbf(h)
        self.packed_size = int(self.mat_offset[-1])
        self.n_atoms = int(self.atom_offset[-1])

    def pack(self, mats):
        out = np.empty(self.packed_size)
        for m, a in enumerate(mats):
            n = int(self.nbfs[m])
            a = np.asarray(a, dtype=np.float64)
            if a.shape != (n, n):
                raise ValueError("molecule %d: expected a %dx%d matrix" % (m, n, n))
            out[self.mat_offset[m]:self.mat_offset[m + 1]] = a.ravel()
        return out

    def unpack(self, flat):
        return [flat[self.mat_offset[m]:self.mat_offset[m + 1]].reshape(self.nbfs[m], self.nbfs[m]).copy()
                for m in range(self.n_mol)]

    def split_atoms(self, g):
        g = np.asarray(g).reshape(-1, 3)
        return [g[self.atom_offset[m]:self.atom_offset[m + 1]].copy() for m in range(self.n_mol)]

    def build_jk(self, Ds, with_k=True):
        D = self.pack(Ds)
        J = np.empty_like(D)
        K = np.empty_like(D) if with_k else None
        self._check(self._lib.iqcp_jk(self._h, _dp(D), _dp(J), _dp(K) if with_k else None))
        return (self.unpack(J), self.unpack(K)) if with_k else self.unpack(J)

    def build_jk_multi(self, sets, with_k=True):
        """sets[s] = per-molecule densities of response set s -> (J sets, K sets)."""
        D = np.ascontiguousarray(np.stack([self.pack(Ds) for Ds in sets]))
        J = np.empty_like(D)
        K = np.empty_like(D) if with_k else None
        self._check(self._lib.iqcp_jk_multi(self._h, len(D), _dp(D), _dp(J), _dp(K) if with_k else None))
        Js = [self.unpack(x) for x in J]
        return (Js, [self.unpack(x) for x in K]) if with_k else Js

    def fock_decomposition(self, H, D, k_scale=1.0):
        raise IqcpError(-1, "use build_jk on a batched context")

    def build_fock(self, Hs, Ds, k_scale=1.0):
        H, D = self.pack(Hs), self.pack(Ds)
        F = np.empty_like(D)
        self._check(self._lib.iqcp_fock(self._h, _dp(H), _dp(D), float(k_scale), _dp(F)))
        return self.unpack(F)

    def eri_gradient(self, Ds, hf_frac=1.0):
        D = self.pack(Ds)
        g = np.zeros((self.n_atoms, 3))
        self._check(self._lib.iqcp_eri_grad(self._h, _dp(D), float(hf_frac), _dp(g)))
        return self.split_atoms(g)

    def one_electron_gradient(self, Ds, Ws):
        D, W = self.pack(Ds), self.pack(Ws)
        g = np.zeros((self.n_atoms, 3))
        self._check(self._lib.iqcp_one_electron_grad(self._h, _dp(D), _dp(W), _dp(g)))
        return self.split_atoms(g)

    def rhf_gradient(self, Ds, Ws):
        D, W = self.pack(Ds), self.pack(Ws)
        g = np.zeros((self.n_atoms, 3))
        self._check(self._lib.iqcp_rhf_gradient(self._h, _dp(D), _dp(W), _dp(g)))
        return self.split_atoms(g)

    def one_electron(self):
        S, T, V = (np.empty(self.packed_size) for _ in range(3))
        self._check(self._lib.iqcp_one_electron(self._h, _dp(S), _dp(T), _dp(V)))
        return self.unpack(S), self.unpack(T), self.unpack(V)

    def eri_compressed(self):
        raise IqcpError(-1, "stored ERIs are single-geometry only")

    def jk_device_noalloc(self, d_D, d_J, d_K=None):
        raise IqcpError(-1, "the fixed-scratch form is single-geometry only")


def boys_eval_all(m_max, T):
    """F_0..F_m_max at each T on the device: array [len(T), m_max+1]."""
    lib = load_library()
    T = np.ascontiguousarray(T, dtype=np.float64).ravel()
    F = np.empty((T.size, m_max + 1))
    rc = lib.iqcp_boys_batch(int(m_max), T.size, _dp(T), _dp(F))
    if rc:
        raise IqcpError(rc)
    return F


def measure_peak(which="fp64"):
    """FMA-throughput probe on the current device, TFLOP/s."""
    lib = load_library()
    t = ctypes.c_double()
    rc = lib.iqcp_measure_peak({"fp64": 0, "fp32": 1}[which], ctypes.byref(t))
    if rc:
        raise IqcpError(rc)
    return t.value


def rys_roots(nroots, T):
    """Rys roots (t^2) and weights on the device: two arrays [len(T), nroots]."""
    lib = load_library()
    T = np.ascontiguousarray(T, dtype=np.float64).ravel()
    R = np.empty((T.size, nroots))
    W = np.empty((T.size, nroots))
    rc = lib.iqcp_rys_batch(int(nroots), T.size, _dp(T), _dp(R), _dp(W))
    if rc:
        raise IqcpError(rc)
    return R, W
