"""Batched restricted Hartree-Fock on the device, one CUDA graph per iteration.

The caller side of the Fock build for many geometries at once (the reference
runs ``rhf_scf``, crates/qc-core/src/scf/mod.rs:1363-1586, once per geometry
inside its optimiser and scan loops, optimizer/mod.rs:274-320).  Every
iteration is one replay of a captured CUDA graph:

  1. F = H + J - K/2 for all geometries: ``iqcp_fock_device`` on the packed
     batch (one launch per angular-momentum class for the whole batch);
  2. E = 1/2 Tr D (H + F) + E_nuc per geometry;
  3. Pulay DIIS on the orthogonalised commutator X^T (F D S - S D F) X
     (scf/mod.rs:990, 1116-1327), with a ring buffer of 8 Fock matrices whose
     slot and fill count live on the device;
  4. the new density from the extrapolated Fock matrix without an
     eigensolver: canonical purification (Palser and Manolopoulos, Phys. Rev.
     B 58, 12704 (1998)) of F' = X^T F X, D = 2 X P X^T.  For a closed shell
     with a HOMO-LUMO gap, P converges to the projector on the n_occ lowest
     eigenvectors of F' -- the aufbau density that the reference obtains from
     ``sorted_eigen`` (scf/mod.rs:743) and D = 2 C_occ C_occ^T (:780).
     Every step is a batched FP64 matrix product, so nothing in the iteration
     needs the host.

The host reads back only the per-geometry energy change, density change and
DIIS error after each replay to decide convergence.  Geometries are grouped
by basis size; each group's dense matrices are padded to its largest member
(padding rows of X are the identity, padding levels of F' sit at the top of
the spectrum and stay empty).  X = S^-1/2 (scf/mod.rs:709) and the
core-Hamiltonian guess (:1379-1389) are formed once, before capture.

At convergence W = 1/2 D F D equals the energy-weighted density
2 sum_occ e_i C_i C_i^T (scf/gradient.rs:101-130), so the nuclear gradient of
every geometry follows from ``iqcp_one_electron_grad_device`` and
``iqcp_eri_grad_device`` on the packed batch.
"""
import ctypes

import numpy as np
import torch

from . import FP64, BatchFockEngine, _dp

DIIS_SIZE = 8


class BatchScfResult:
    def __init__(self, **kw):
        self.__dict__.update(kw)


def _groups(nbf, n_groups):
    order = np.argsort(nbf, kind="stable")
    return [g for g in np.array_split(order, min(n_groups, len(order))) if len(g)]


class _Group:
    """Dense padded view of some geometries of the packed batch."""

    def __init__(self, eng, mols, dev):
        self.mols = np.asarray(mols)
        self.n = int(eng.nbfs[self.mols].max())
        B, n = len(self.mols), self.n
        idx = np.zeros((B, n, n), np.int64)
        valid = np.zeros((B, n, n), bool)
        pad = np.ones((B, n), bool)
        for k, m in enumerate(self.mols):
            nm = int(eng.nbfs[m])
            idx[k, :nm, :nm] = int(eng.mat_offset[m]) + np.arange(nm * nm).reshape(nm, nm)
            valid[k, :nm, :nm] = True
            pad[k, :nm] = False
        flat = np.flatnonzero(valid)
        self.gidx = torch.from_numpy(idx).to(dev)
        self.valid = torch.from_numpy(valid).to(dev)
        self.vpos = torch.from_numpy(flat).to(dev)                 # positions in the padded group
        self.vidx = torch.from_numpy(idx.ravel()[flat]).to(dev)    # the same elements in the packed batch
        self.pad = torch.from_numpy(pad).to(dev)
        self.nvalid = self.valid.sum(dim=(1, 2)).to(torch.float64)

    def unpack(self, flat):
        return torch.where(self.valid, flat[self.gidx], torch.zeros((), dtype=flat.dtype, device=flat.device))

    def pack_into(self, flat, t):
        flat[self.vidx] = t.reshape(-1)[self.vpos]


def _purify(Fp, nocc, n_iter):
    """Canonical purification: density projector (eigenvalues 0/1, trace nocc)
    on the lowest nocc levels of the symmetric Fp [B, n, n]."""
    B, n, _ = Fp.shape
    eye = torch.eye(n, dtype=Fp.dtype, device=Fp.device).expand(B, n, n)
    diag = torch.diagonal(Fp, dim1=1, dim2=2)
    radius = Fp.abs().sum(dim=2) - diag.abs()
    emax = (diag + radius).amax(dim=1)
    emin = (diag - radius).amin(dim=1)
    mu = diag.sum(dim=1) / n
    ne = nocc.to(Fp.dtype)
    lam = torch.minimum(ne / (emax - mu).clamp_min(1e-30), (n - ne) / (mu - emin).clamp_min(1e-30))
    P = (lam / n)[:, None, None] * (mu[:, None, None] * eye - Fp) + (ne / n)[:, None, None] * eye
    for _ in range(n_iter):
        P2 = torch.bmm(P, P)
        P3 = torch.bmm(P2, P)
        t1 = torch.diagonal(P - P2, dim1=1, dim2=2).sum(dim=1)
        t2 = torch.diagonal(P2 - P3, dim1=1, dim2=2).sum(dim=1)
        # once idempotent to rounding the coefficient is 0/0: take the McWeeny step
        small = t1.abs() < 1e-13
        c = torch.where(small, torch.full_like(t1, 0.5), t2 / torch.where(small, torch.ones_like(t1), t1))
        ch = c[:, None, None]
        P_hi = ((1.0 + ch) * P2 - P3) / ch.clamp_min(1e-30)
        P_lo = ((1.0 - 2.0 * ch) * P + (1.0 + ch) * P2 - P3) / (1.0 - ch).clamp_min(1e-30)
        P = torch.where((c >= 0.5)[:, None, None], P_hi, P_lo)
    return P


def _solve_spd(A, b):
    """Solve A x = b for a batch of small symmetric positive definite systems
    by unrolled Gaussian elimination (fixed shapes, no host synchronisation)."""
    A = A.clone()
    x = b.clone()
    K = A.shape[-1]
    for k in range(K):
        piv = A[:, k, k].clone()
        for i in range(k + 1, K):
            f = A[:, i, k] / piv
            A[:, i, :] = A[:, i, :] - f[:, None] * A[:, k, :]
            x[:, i] = x[:, i] - f * x[:, k]
    out = torch.zeros_like(x)
    for k in range(K - 1, -1, -1):
        s = x[:, k] - (A[:, k, k + 1:] * out[:, k + 1:]).sum(dim=1)
        out[:, k] = s / A[:, k, k]
    return out


class BatchRHF:
    """Device-resident batched RHF over the geometries of a BatchFockEngine."""

    def __init__(self, bases, n_groups=8, purify_iters=64, precision=FP64, mixed_cutoff=1e-9, device=0,
                 engine=None, level_shift=0.0, D0=None):
        """D0: optional list of starting densities (default: core-Hamiltonian guess)."""
        self._opts = dict(purify_iters=purify_iters, precision=precision, mixed_cutoff=mixed_cutoff,
                          device=device, level_shift=level_shift)
        self.dev = torch.device("cuda", device)
        self.eng = engine if engine is not None else BatchFockEngine(bases, precision=precision,
                                                                    mixed_cutoff=mixed_cutoff, device=device)
        eng = self.eng
        self.bases = list(bases)
        if any(b.n_electrons % 2 for b in self.bases):
            raise ValueError("closed-shell geometries only")
        self.purify_iters = purify_iters
        # virtual-level shift (Ha) of the extrapolated Fock matrix: F' + s (1 - P),
        # P the occupied projector of the current density; damps occupied-virtual
        # oscillations of small-gap geometries, converged solution unchanged
        self.level_shift = float(level_shift)
        S, T, V = (torch.from_numpy(x).to(self.dev) for x in self._one_electron_packed())
        self.H_p = T + V
        self.D_p = torch.zeros_like(S)
        self.F_p = torch.zeros_like(S)
        enuc = torch.tensor([b.nuclear_repulsion() for b in self.bases], dtype=torch.float64, device=self.dev)
        nocc = np.array([b.n_electrons // 2 for b in self.bases])
        self.groups = [_Group(eng, g, self.dev) for g in _groups(eng.nbfs, n_groups)]
        for g in self.groups:
            mols = torch.from_numpy(g.mols).to(self.dev)
            g.nocc = torch.from_numpy(nocc[g.mols]).to(self.dev)
            g.enuc = enuc[mols]
            g.S = g.unpack(S)
            g.H = g.unpack(self.H_p)
            eye = torch.eye(g.n, dtype=torch.bool, device=self.dev)
            Sp = torch.where(g.pad[:, :, None] & g.pad[:, None, :] & eye, 1.0, g.S)
            w, U = torch.linalg.eigh(Sp)
            if float(w.min()) <= 1e-10:
                raise ValueError("overlap matrix is singular")
            g.X = (U / torch.sqrt(w)[:, None, :]) @ U.transpose(1, 2)
            if D0 is None:
                # core-Hamiltonian guess (scf/mod.rs:1379-1389), eagerly, before capture
                Hp = g.X.transpose(1, 2) @ g.H @ g.X + torch.diag_embed(g.pad.to(torch.float64) * 1e6)
                _, C = torch.linalg.eigh(Hp)
                Cx = g.X @ C
                occ = (torch.arange(g.n, device=self.dev)[None, :] < g.nocc[:, None]).to(torch.float64)
                g.D = (2.0 * (Cx * occ[:, None, :]) @ Cx.transpose(1, 2)) * g.valid
            else:
                g.D = g.unpack(torch.from_numpy(eng.pack(D0)).to(self.dev))
            g.pack_into(self.D_p, g.D)
            B = len(g.mols)
            g.Fbuf = torch.zeros((DIIS_SIZE, B, g.n, g.n), dtype=torch.float64, device=self.dev)
            g.Ebuf = torch.zeros_like(g.Fbuf)
            g.E = torch.zeros(B, dtype=torch.float64, device=self.dev)
            g.dE = torch.zeros_like(g.E)
            g.dD = torch.zeros_like(g.E)
            g.err = torch.zeros_like(g.E)
            g.idem = torch.zeros_like(g.E)
        self.slot = torch.zeros(1, dtype=torch.int64, device=self.dev)
        self.count = torch.zeros(1, dtype=torch.int64, device=self.dev)
        self.graph = None

    def _one_electron_packed(self):
        eng = self.eng
        out = [np.empty(eng.packed_size) for _ in range(3)]
        eng._check(eng._lib.iqcp_one_electron(eng._h, _dp(out[0]), _dp(out[1]), _dp(out[2])))
        return out

    def _step(self):
        """One SCF iteration of every geometry, enqueued on the current stream."""
        self.eng.fock_device(self.H_p.data_ptr(), self.D_p.data_ptr(), 1.0, self.F_p.data_ptr())
        K = DIIS_SIZE
        kk = torch.arange(K, device=self.dev)
        new_count = torch.clamp(self.count + 1, max=K)
        filled = kk < new_count
        eye = torch.eye(K, dtype=torch.float64, device=self.dev)
        for g in self.groups:
            F = g.unpack(self.F_p)
            D = g.D
            E = 0.5 * (D * (g.H + F)).sum(dim=(1, 2)) + g.enuc
            g.dE.copy_(E - g.E)
            g.E.copy_(E)
            FDS = F @ D @ g.S
            err = g.X.transpose(1, 2) @ (FDS - FDS.transpose(1, 2)) @ g.X
            g.err.copy_(err.abs().amax(dim=(1, 2)))
            g.Fbuf.index_copy_(0, self.slot, F[None])
            g.Ebuf.index_copy_(0, self.slot, err[None])
            Bm = torch.einsum("kbij,lbij->bkl", g.Ebuf, g.Ebuf)
            mask = (filled[:, None] & filled[None, :]).to(Bm.dtype)
            scale = torch.diagonal(Bm, dim1=1, dim2=2).amax(dim=1).clamp_min(1e-300)[:, None, None]
            unfilled = torch.diag_embed((~filled).to(Bm.dtype).expand(Bm.shape[0], K))
            Bm = Bm / scale * mask + unfilled + 1e-14 * eye
            rhs = filled.to(Bm.dtype).expand(Bm.shape[0], K).contiguous()
            c = _solve_spd(Bm, rhs)
            c = c / c.sum(dim=1, keepdim=True)
            Fx = torch.einsum("bk,kbij->bij", c, g.Fbuf)
            Fp = g.X.transpose(1, 2) @ Fx @ g.X
            if self.level_shift:
                XS = g.X.transpose(1, 2) @ g.S
                Pocc = 0.5 * (XS @ D @ XS.transpose(1, 2))
                eye_n = torch.eye(g.n, dtype=Fp.dtype, device=self.dev)
                Fp = Fp + self.level_shift * (eye_n - Pocc)
            # padding levels at the top of the spectrum, above every real level
            top = Fp.abs().sum(dim=2).amax(dim=1) + 1.0
            real = (~g.pad[:, :, None] & ~g.pad[:, None, :]).to(Fp.dtype)
            Fp = Fp * real + torch.diag_embed(g.pad.to(Fp.dtype) * top[:, None])
            P = _purify(Fp, g.nocc, self.purify_iters)
            g.idem.copy_((P - torch.bmm(P, P)).abs().amax(dim=(1, 2)))
            Dn = (2.0 * g.X @ P @ g.X.transpose(1, 2)) * g.valid
            g.dD.copy_(torch.sqrt(((Dn - D) ** 2).sum(dim=(1, 2)) / g.nvalid))
            g.D.copy_(Dn)
            g.pack_into(self.D_p, Dn)
        self.slot.copy_((self.slot + 1) % K)
        self.count.copy_(new_count)

    def capture(self):
        """Record one iteration as a CUDA graph (after one eager warm-up step)."""
        s = torch.cuda.Stream(device=self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(s):
            self.eng.set_stream(s.cuda_stream)
            self._step()
        torch.cuda.current_stream(self.dev).wait_stream(s)
        torch.cuda.synchronize(self.dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.eng.set_stream(torch.cuda.current_stream(self.dev).cuda_stream)
            self._step()
        self.eng.set_stream(torch.cuda.current_stream(self.dev).cuda_stream)
        self.graph = g
        return g

    def _gather(self, name):
        order = np.concatenate([g.mols for g in self.groups])
        v = np.empty(len(self.bases))
        v[order] = torch.cat([getattr(g, name) for g in self.groups]).cpu().numpy()
        return v

    def _set_density(self, m, D):
        """Overwrite geometry m's density (packed array and its group's block)."""
        lo, hi = int(self.eng.mat_offset[m]), int(self.eng.mat_offset[m + 1])
        Dt = torch.from_numpy(np.ascontiguousarray(D)).to(self.dev)
        self.D_p[lo:hi] = Dt.reshape(-1)
        for g in self.groups:
            k = np.flatnonzero(g.mols == m)
            if len(k):
                n = D.shape[0]
                g.D[int(k[0]), :n, :n] = Dt

    def run(self, e_tol=1e-9, d_tol=1e-7, err_tol=1e-5, max_iter=80, use_graph=True, handoff=None,
            handoff_after=10):
        """Iterate until every geometry meets the three thresholds or max_iter.

        handoff: optional fraction; once at least that share of the geometries
        has converged (after handoff_after iterations), the others continue in a
        new batched context of their own, seeded with their current densities
        (DIIS restarts), so the converged ones stop costing Fock builds.  Their
        results and densities are written back, so gradients() still covers the
        whole batch."""
        if use_graph and self.graph is None:
            self.capture()
        self.eng.set_stream(torch.cuda.current_stream(self.dev).cuda_stream)
        it = 0
        order = np.concatenate([g.mols for g in self.groups])
        conv = np.zeros(len(self.bases), bool)
        for it in range(1, max_iter + 1):
            if use_graph:
                self.graph.replay()
            else:
                self._step()
            stats = torch.stack([torch.cat([g.dE.abs() for g in self.groups]),
                                 torch.cat([g.dD for g in self.groups]),
                                 torch.cat([g.err for g in self.groups])]).cpu().numpy()
            conv = np.empty(len(self.bases), bool)
            conv[order] = (stats[0] < e_tol) & (stats[1] < d_tol) & (stats[2] < err_tol)
            if it > 2 and conv.all():
                break
            if (handoff is not None and it >= handoff_after and it < max_iter and conv.mean() >= handoff
                    and len(self.bases) > 1):
                break
        energies, idem = self._gather("E"), self._gather("idem")
        iterations = it
        pending = np.flatnonzero(~conv)
        if handoff is not None and len(pending) and it < max_iter and len(pending) < len(self.bases):
            dens = self.densities()
            sub = BatchRHF([self.bases[i] for i in pending], n_groups=min(len(pending), 8),
                           D0=[dens[i] for i in pending], **self._opts)
            sub.eng.set_stream(torch.cuda.current_stream(self.dev).cuda_stream)
            sub.eng.autotune(sub.D_p.data_ptr(), 1)
            r = sub.run(e_tol=e_tol, d_tol=d_tol, err_tol=err_tol, max_iter=max_iter - it, use_graph=use_graph)
            for j, i in enumerate(pending):
                energies[i], idem[i], conv[i] = r.energies[j], r.idempotency[j], r.converged[j]
            for j, D in enumerate(sub.densities()):
                self._set_density(int(pending[j]), D)
            iterations = it + r.iterations
            sub.graph = None
            sub.eng.close()
            self.eng.set_stream(torch.cuda.current_stream(self.dev).cuda_stream)
        return BatchScfResult(energies=energies, converged=conv, iterations=iterations, idempotency=idem)

    def densities(self):
        return self.eng.unpack(self.D_p.cpu().numpy())

    def gradients(self):
        """RHF nuclear gradients of all geometries at the current density, with
        W = 1/2 D F D (valid at convergence)."""
        eng = self.eng
        eng.set_stream(torch.cuda.current_stream(self.dev).cuda_stream)
        eng.fock_device(self.H_p.data_ptr(), self.D_p.data_ptr(), 1.0, self.F_p.data_ptr())
        W_p = torch.zeros_like(self.D_p)
        for g in self.groups:
            F = g.unpack(self.F_p)
            g.pack_into(W_p, (0.5 * g.D @ F @ g.D) * g.valid)
        grad = torch.zeros((eng.n_atoms, 3), dtype=torch.float64, device=self.dev)
        eng._check(eng._lib.iqcp_one_electron_grad_device(eng._h, ctypes.c_void_p(self.D_p.data_ptr()),
                                                          ctypes.c_void_p(W_p.data_ptr()),
                                                          ctypes.c_void_p(grad.data_ptr())))
        eng.eri_gradient_device(self.D_p.data_ptr(), 1.0, grad.data_ptr())
        return eng.split_atoms(grad.cpu().numpy())
