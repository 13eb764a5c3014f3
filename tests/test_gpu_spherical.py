"""J/K in the real spherical-harmonic basis (iqcp_jk_spherical) against the
reference's spherical path restated on the oracle: Cartesian ERIs from the
oracle's eri_compressed, each index transformed with the Cartesian-to-
spherical coefficients (EriSphericalTransform, integrals/spherical.rs:390-470),
then digested into J and K.  Parity bar: 1e-10 Ha per element."""
import numpy as np
import pytest

from conftest import random_density
from iqcp_b200 import BasisSet, FockEngine
from iqcp_b200.molecules import REFERENCE_MOLECULES

pytestmark = pytest.mark.gpu


def cart2sph_d():
    """C[cart][sph] for d (xx xy xz yy yz zz -> d-2 d-1 d0 d+1 d+2), from the
    real solid harmonics' normalisation constants."""
    a = np.sqrt(15.0 / (4.0 * np.pi))          # xy, xz, yz
    b = np.sqrt(5.0 / (16.0 * np.pi))          # d0: 2zz - xx - yy
    c = np.sqrt(15.0 / (16.0 * np.pi))         # d+2: xx - yy
    C = np.zeros((6, 5))
    C[1, 0] = C[4, 1] = C[2, 3] = a
    C[0, 2] = C[3, 2] = -b
    C[5, 2] = 2 * b
    C[0, 4], C[3, 4] = c, -c
    return C


def transform_matrix(b):
    blocks = []
    for l in b.l:
        blocks.append(np.eye(1) if l == 0 else (np.eye(3) if l == 1 else cart2sph_d()))
    nc = sum(x.shape[0] for x in blocks)
    ns = sum(x.shape[1] for x in blocks)
    C = np.zeros((nc, ns))
    i = j = 0
    for x in blocks:
        C[i:i + x.shape[0], j:j + x.shape[1]] = x
        i += x.shape[0]
        j += x.shape[1]
    return C


def full_eri(b, oracle_mod):
    eri, _ = oracle_mod.eri_compressed(b)
    n = b.n_basis
    i, j = np.tril_indices(n)
    pair = np.zeros((n, n), np.int64)
    pair[i, j] = i * (i + 1) // 2 + j
    pair[j, i] = pair[i, j]
    P = pair[:, :, None, None]
    Q = pair[None, None, :, :]
    hi, lo = np.maximum(P, Q), np.minimum(P, Q)
    return eri[hi * (hi + 1) // 2 + lo]


@pytest.mark.parametrize("mol,basis", [("H2O", "6-31g*"), ("NH3", "cc-pvdz"), ("CH4", "6-31+g*")])
def test_jk_spherical_vs_transformed_eris(oracle_mod, mol, basis):
    b = BasisSet.build(REFERENCE_MOLECULES[mol], basis)
    C = transform_matrix(b)
    ns = C.shape[1]
    eri_s = np.einsum("abcd,ai,bj,ck,dl->ijkl", full_eri(b, oracle_mod), C, C, C, C, optimize=True)
    D = random_density(ns, 5, 0.1)
    Jr = np.einsum("ijkl,kl->ij", eri_s, D)
    Kr = np.einsum("ikjl,kl->ij", eri_s, D)
    with FockEngine(b) as eng:
        assert eng._lib.iqcp_nbf_spherical(eng._h) == ns
        J, K = eng.build_jk_spherical(D)
        Jonly = eng.build_jk_spherical(D, with_k=False)
    assert np.abs(J - Jr).max() < 1e-10, np.abs(J - Jr).max()
    assert np.abs(K - Kr).max() < 1e-10, np.abs(K - Kr).max()
    assert np.abs(Jonly - J).max() < 1e-13
