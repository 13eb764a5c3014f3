"""Batched restricted Hartree-Fock on the device, through the C ABI.

The caller side of the Fock build for many geometries at once (the reference
runs ``rhf_scf``, crates/qc-core/src/scf/mod.rs:1363-1586, once per geometry
inside its optimiser and scan loops, optimizer/mod.rs:274-320).  The whole
iteration lives in ``libiqcp_gpu.so`` (``iqcp_batch_scf``, csrc/scf.cu): one
CUDA-graph replay per iteration runs the Fock build of every geometry, the
energies, Pulay DIIS on the orthogonalised commutator and the new densities
by canonical purification; the host only reads back the convergence
figures.  This module is a thin ctypes wrapper with the shapes of a batched
``BatchFockEngine``: matrices packed per geometry, gradients split per
geometry.
"""
import ctypes

import numpy as np

from . import FP64, BatchFockEngine, ScfOptions, _dp


class BatchScfResult:
    def __init__(self, **kw):
        self.__dict__.update(kw)


class BatchRHF:
    """Device-resident batched RHF over the geometries of a BatchFockEngine."""

    def __init__(self, bases, precision=FP64, mixed_cutoff=1e-9, device=0, engine=None, diis_size=8,
                 purify_iters=64):
        self.eng = engine if engine is not None else BatchFockEngine(bases, precision=precision,
                                                                    mixed_cutoff=mixed_cutoff, device=device)
        self.bases = list(bases)
        if any(b.n_electrons % 2 for b in self.bases):
            raise ValueError("closed-shell geometries only")
        self.diis_size = diis_size
        self.purify_iters = purify_iters
        self._D = None
        self._grad = None

    def _opts(self, e_tol, d_tol, err_tol, max_iter):
        o = ScfOptions()
        self.eng._lib.iqcp_scf_default_options(ctypes.byref(o))
        o.e_tol, o.d_tol, o.err_tol, o.max_iter = e_tol, d_tol, err_tol, max_iter
        o.diis_size, o.purify_iters = self.diis_size, self.purify_iters
        return o

    def core_guess(self):
        """Packed core-Hamiltonian guess densities (scf/mod.rs:1379-1389), by purification."""
        eng = self.eng
        D = np.empty(eng.packed_size)
        o = self._opts(1e-9, 1e-7, 1e-5, 0)
        eng._check(eng._lib.iqcp_batch_scf(eng._h, ctypes.byref(o), None, None, None, None, _dp(D), None))
        return D

    def sad_guess(self):
        """Packed SAD densities of every geometry (iqcp_sad_density per geometry;
        the reference's guess for its optimiser and scan callers, scf/sad.rs:698)."""
        return self.eng.pack([b.sad_density(self.eng.device) for b in self.bases])

    def run(self, e_tol=1e-9, d_tol=1e-7, err_tol=1e-5, max_iter=80, D0=None, gradients=True):
        """Iterate every geometry until all meet the three thresholds or max_iter;
        D0: optional starting densities, a list per geometry or a packed array
        (sad_guess(); default: the core-Hamiltonian guess).
        With gradients, the RHF nuclear gradient at the final density comes back
        too (gradients())."""
        eng = self.eng
        n = eng.n_mol
        E = np.zeros(n)
        conv = np.zeros(n, np.int32)
        iters = ctypes.c_int(0)
        D = np.empty(eng.packed_size)
        g = np.zeros((eng.n_atoms, 3)) if gradients else None
        d0 = None
        if D0 is not None:
            d0 = np.ascontiguousarray(D0, dtype=np.float64) if np.ndim(D0) == 1 else eng.pack(D0)
        o = self._opts(e_tol, d_tol, err_tol, max_iter)
        eng._check(eng._lib.iqcp_batch_scf(eng._h, ctypes.byref(o), _dp(d0) if d0 is not None else None, _dp(E),
                                           conv.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.byref(iters),
                                           _dp(D), _dp(g) if gradients else None))
        self._D = D
        self._grad = g
        return BatchScfResult(energies=E, converged=conv.astype(bool), iterations=iters.value)

    def densities(self):
        return self.eng.unpack(self._D)

    def gradients(self):
        """RHF nuclear gradients of all geometries at the final density of run()."""
        if self._grad is None:
            raise RuntimeError("run(gradients=True) first")
        return self.eng.split_atoms(self._grad)

    def close(self):
        self.eng.close()
