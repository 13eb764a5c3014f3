"""CPU oracle (TEST INFRASTRUCTURE ONLY): the SAD initial density.

Restates build_sad_density (crates/qc-core/src/scf/sad.rs:698-760) and the
spherically averaged atomic RHF it runs per element (sad.rs:145-640, after
PySCF's AtomSphAverageRHF), on the oracle's own one-electron integrals and
compressed ERIs, with numpy's symmetric eigensolver for the small radial
blocks.  Only tests import it, as the checker of iqcp_sad_density.
"""
import numpy as np

from . import eri_compressed, one_electron
from .basis import OracleBasis

# (n_s, n_p, n_d) electrons of the ground configuration (sad.rs:67-90)
_CONFIG = {1: (1, 0, 0), 2: (2, 0, 0), 3: (3, 0, 0), 4: (4, 0, 0), 5: (4, 1, 0), 6: (4, 2, 0), 7: (4, 3, 0),
           8: (4, 4, 0), 9: (4, 5, 0), 10: (4, 6, 0), 11: (5, 6, 0), 12: (6, 6, 0), 13: (6, 7, 0), 14: (6, 8, 0),
           15: (6, 9, 0), 16: (6, 10, 0), 17: (6, 11, 0), 18: (6, 12, 0)}


def _ncart(l):
    return (l + 1) * (l + 2) // 2


def _groups(shell_l):
    """Per l in order of first appearance: (l, n_comp, [bf of radial shell r, component m])
    (analyze_shell_structure, sad.rs:145-198)."""
    groups, off = [], 0
    for l in shell_l:
        g = next((x for x in groups if x[0] == l), None)
        if g is None:
            g = (l, _ncart(l), [])
            groups.append(g)
        g[2].append([off + c for c in range(_ncart(l))])
        off += _ncart(l)
    return groups


def _gen_eig(f, s):
    """F c = S c e by symmetric orthogonalisation (solve_gen_eig, sad.rs:289-356)."""
    n = f.shape[0]
    if n == 1:
        return np.array([f[0, 0] / s[0, 0]]), np.array([[1.0 / np.sqrt(s[0, 0])]])
    w, v = np.linalg.eigh(s)
    keep = w >= 1e-10
    x = (v[:, keep] / np.sqrt(w[keep])) @ v[:, keep].T
    e, cp = np.linalg.eigh(x.T @ f @ x)
    return e, x @ cp


def _density(F, S, groups, cfg):
    """Spherically averaged eigenproblem per l and fractional occupations
    (spherical_average_eig + build_density_fractional, sad.rs:207-520)."""
    n = F.shape[0]
    D = np.zeros((n, n))
    for l, nc, shells in groups:
        bf = np.array(shells)                      # [radial, component]
        fa = np.einsum("imjm->ij", F[bf[:, :, None, None], bf[None, None, :, :]]) / nc
        sa = np.einsum("imjm->ij", S[bf[:, :, None, None], bf[None, None, :, :]]) / nc
        if l >= 3 or cfg[l] == 0:
            continue
        e, C = _gen_eig(fa, sa)
        ne, per = cfg[l], 2 * nc
        ndocc, rem = ne // per, ne - (ne // per) * per
        for i in range(len(shells)):
            occ = 2.0 if i < ndocc else (rem / nc if (i == ndocc and rem > 0) else 0.0)
            if occ == 0.0:
                continue
            for m in range(nc):
                idx = bf[:, m]
                D[np.ix_(idx, idx)] += occ * np.outer(C[:, i], C[:, i])
    return D


def _pair(i, j):
    return np.where(i >= j, i * (i + 1) // 2 + j, j * (j + 1) // 2 + i)


def atomic_density(z, one):
    """Atomic SCF of one element on its one-atom basis (atomic_scf, sad.rs:525-590)."""
    S = one_electron(one, "S")
    H = one_electron(one, "T") + one_electron(one, "V")
    groups = _groups(list(one.l))
    cfg = _CONFIG.get(int(z), (0, 0, 0))
    D = _density(H, S, groups, cfg)
    if z <= 1:
        return D
    n = S.shape[0]
    eri, _ = eri_compressed(one)
    i = np.arange(n)
    ij = _pair(i[:, None], i[None, :])
    full = eri[_pair(ij[:, :, None, None], ij[None, None, :, :])]   # (mn|ls)
    e_old = np.inf
    for _ in range(40):
        G = np.einsum("ls,mnls->mn", D, full) - 0.5 * np.einsum("ls,mlns->mn", D, full)
        F = H + G
        e = 0.5 * np.sum(D * (H + F).T)
        if abs(e - e_old) < 1e-10:
            break
        e_old = e
        D = _density(F, S, groups, cfg)
    return D


def sad_density(b):
    """SAD density of basis b (an OracleBasis or anything with the same
    arrays): atomic blocks per element, copied to each atom of it."""
    l = np.asarray(b.l)
    off = np.concatenate([[0], np.cumsum([_ncart(x) for x in l])])
    pstart = np.concatenate([[0], np.cumsum(b.nprim)])
    n = int(off[-1])
    D = np.zeros((n, n))
    cache = {}
    for a in range(b.n_atoms):
        sh = [s for s in range(len(l)) if b.atom_of_shell[s] == a]
        if not sh:
            continue
        z = int(b.z[a])
        if z not in cache:
            pos = np.asarray(b.xyz[a], dtype=np.float64)
            one = OracleBasis("", [z], [pos], [int(l[s]) for s in sh], [int(b.nprim[s]) for s in sh],
                              [0] * len(sh), [pos] * len(sh),
                              np.concatenate([b.exps[pstart[s]:pstart[s + 1]] for s in sh]),
                              np.concatenate([b.coefs[pstart[s]:pstart[s + 1]] for s in sh]))
            cache[z] = atomic_density(z, one)
        gbf = np.concatenate([np.arange(off[s], off[s + 1]) for s in sh])
        D[np.ix_(gbf, gbf)] = cache[z]
    return D
