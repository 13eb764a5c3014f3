"""The oracle's SAD density against the reference's own SAD tests
(crates/qc-core/src/scf/sad.rs:1164-1553): PySCF's AtomSphAverageRHF block of
H in 6-31G*, the H2/STO-3G density, Tr(DS) = N, zero inter-atom blocks."""
import numpy as np
import pytest

import oracle
from oracle.basis import build_basis
from oracle.sad import sad_density

H2 = [(1, (0.0, 0.0, 0.0)), (1, (0.0, 0.0, 1.4))]
H2O = [(8, (0.0, 0.0, 0.2216)), (1, (0.0, 1.4309, -0.8864)), (1, (0.0, -1.4309, -0.8864))]
LIH = [(3, (0.0, 0.0, 0.0)), (1, (0.0, 0.0, 3.0139))]
CH4 = [(6, (0.0, 0.0, 0.0)), (1, (1.1851, 1.1851, 1.1851)), (1, (-1.1851, -1.1851, 1.1851)),
       (1, (-1.1851, 1.1851, -1.1851)), (1, (1.1851, -1.1851, -1.1851))]


def test_h_631gs_matches_pyscf():
    """sad.rs:1533-1552: D00 0.18269670, D01 0.28443329, D11 0.44282296 (1e-6 there)."""
    D = sad_density(build_basis(H2, "6-31g*"))
    assert abs(D[0, 0] - 0.18269670) < 1e-7
    assert abs(D[0, 1] - 0.28443329) < 1e-7
    assert abs(D[1, 1] - 0.44282296) < 1e-7


def test_h2_sto3g():
    """sad.rs:1164-1188: one normalised function per H, occupation 1."""
    D = sad_density(build_basis(H2, "sto-3g"))
    assert np.allclose(D, np.eye(2), atol=1e-10)


@pytest.mark.parametrize("atoms,n", [(H2, 2), (H2O, 10), (LIH, 4), (CH4, 10)])
@pytest.mark.parametrize("basis", ["sto-3g", "6-31g*"])
def test_electron_count(atoms, n, basis):
    """sad.rs:1191-1258 asks Tr(DS) within 0.1 of N; the fractional
    occupations make it exact."""
    b = build_basis(atoms, basis)
    D = sad_density(b)
    S = oracle.one_electron(b, "S")
    assert abs(np.sum(D * S) - n) < 1e-8
    assert np.allclose(D, D.T, atol=1e-14)


def test_inter_atom_blocks_zero_and_shared_per_element():
    b = build_basis(H2O, "6-31g*")
    D = sad_density(b)
    off = np.concatenate([[0], np.cumsum([(l + 1) * (l + 2) // 2 for l in b.l])])
    atom_bf = [np.concatenate([np.arange(off[s], off[s + 1]) for s in range(b.n_shells) if b.atom_of_shell[s] == a])
               for a in range(b.n_atoms)]
    assert np.all(D[np.ix_(atom_bf[0], atom_bf[1])] == 0.0)
    assert np.array_equal(D[np.ix_(atom_bf[1], atom_bf[1])], D[np.ix_(atom_bf[2], atom_bf[2])])
    assert np.abs(D[np.ix_(atom_bf[0], atom_bf[0])] - np.diag(np.diag(D[np.ix_(atom_bf[0], atom_bf[0])]))).max() > 1e-3
