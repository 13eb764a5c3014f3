"""Host SCF driver options on the oracle's stored-ERI Fock build (CPU): the
virtual-level shift and the canonical orthogonalisation path converge to the
same RHF energy as the reference's plain symmetric-orthogonaliser DIIS loop."""
from iqcp_b200 import BasisSet
from iqcp_b200.molecules import REFERENCE_MOLECULES
from iqcp_b200.scf import rhf_scf


def test_level_shift_and_canonical_orthogonaliser_same_energy(oracle_mod):
    b = BasisSet.build(REFERENCE_MOLECULES["H2O"], "6-31g*")
    S, H = oracle_mod.one_electron(b, "S"), oracle_mod.hcore(b)
    eri, _ = oracle_mod.eri_compressed(b)

    def fock(H_, D):
        return oracle_mod.build_fock(H_, D, eri)

    args = (S, H, b.nuclear_repulsion(), b.n_electrons // 2, fock)
    r0 = rhf_scf(*args, e_tol=1e-12, d_tol=1e-10)
    r1 = rhf_scf(*args, e_tol=1e-12, d_tol=1e-10, level_shift=0.2, max_iter=200)
    r2 = rhf_scf(*args, e_tol=1e-12, d_tol=1e-10, lindep=1e-20)
    assert r0.converged and r1.converged and r2.converged
    assert abs(r1.energy - r0.energy) < 1e-10
    assert abs(r2.energy - r0.energy) < 1e-10
