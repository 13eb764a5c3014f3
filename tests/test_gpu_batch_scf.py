"""Batched device RHF (one CUDA graph per iteration) against the per-geometry
host driver: converged energies within 1e-8 Ha and RHF gradients within
1e-6 Ha/bohr of rhf_scf + rhf_gradient run geometry by geometry."""
import numpy as np
import pytest

from iqcp_b200 import BasisSet, FockEngine
from iqcp_b200.molecules import REFERENCE_MOLECULES, batch_geometries
from iqcp_b200.scf import energy_weighted_density, rhf_scf

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bases():
    out = [BasisSet.build(REFERENCE_MOLECULES[m], b)
           for m, b in [("H2O", "6-31g*"), ("NH3", "cc-pvdz"), ("CH4", "3-21g"), ("HF", "6-31+g*"),
                        ("C6H6", "6-31g*")]]
    out += [BasisSet.build(a, "6-31g*") for a in batch_geometries(3, seed=11, min_atoms=8, max_atoms=14)]
    return out


@pytest.fixture(scope="module")
def reference(bases):
    ref = []
    for b in bases:
        with FockEngine(b) as eng:
            S, T, V = eng.one_electron()
            res = rhf_scf(S, T + V, b.nuclear_repulsion(), b.n_electrons // 2, eng.build_fock, e_tol=1e-11,
                          d_tol=1e-9)
            W = energy_weighted_density(res.mo_coefficients, res.mo_energies, res.n_occ)
            ref.append((res.energy, eng.rhf_gradient(res.density, W), res.density))
    return ref


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_rhf_energies_and_gradients(bases, reference, use_graph):
    from iqcp_b200.batch_scf import BatchRHF

    scf = BatchRHF(bases, n_groups=3)
    res = scf.run(e_tol=1e-10, d_tol=1e-8, err_tol=1e-7, use_graph=use_graph)
    assert res.converged.all(), res.__dict__
    assert res.idempotency.max() < 1e-10
    grads = scf.gradients()
    dens = scf.densities()
    for (e_ref, g_ref, d_ref), e, g, d in zip(reference, res.energies, grads, dens):
        assert abs(e - e_ref) < 1e-8, (e, e_ref)
        assert np.abs(d - d_ref).max() < 1e-5
        assert np.abs(g - g_ref).max() < 1e-6


def test_batch_rhf_handoff(bases, reference):
    """Hand-off of the unconverged geometries to a smaller batch after a few
    iterations reaches the same energies, densities and gradients."""
    from iqcp_b200.batch_scf import BatchRHF

    scf = BatchRHF(bases, n_groups=3)
    res = scf.run(e_tol=1e-10, d_tol=1e-8, err_tol=1e-7, handoff=0.3, handoff_after=3)
    assert res.converged.all(), res.__dict__
    grads = scf.gradients()
    # the device calls and the torch steps between them share one stream: a
    # second evaluation agrees to rounding
    again = scf.gradients()
    assert max(np.abs(a - b).max() for a, b in zip(grads, again)) < 1e-10
    dens = scf.densities()
    for (e_ref, g_ref, d_ref), e, g, d in zip(reference, res.energies, grads, dens):
        assert abs(e - e_ref) < 1e-8, (e, e_ref)
        assert np.abs(d - d_ref).max() < 1e-5
        assert np.abs(g - g_ref).max() < 1e-6
