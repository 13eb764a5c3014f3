"""The C ABI without a GPU: the library loads, exports every entry point that
include/iqcp.h declares, builds bases like BasisSet::build, and reports
errors the way the header documents (no compute call needs a device here)."""
import ctypes
import os
import re

import numpy as np
import pytest

import iqcp_b200 as iq
from iqcp_b200 import BasisSet, IqcpError
from iqcp_b200.molecules import REFERENCE_MOLECULES

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "iqcp.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(iqcp_\w+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    lib = iq.load_library()
    names = declared_symbols()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    # and the Python binding covers them all
    assert set(names) <= set(iq.EXPORTS), set(names) - set(iq.EXPORTS)


@pytest.mark.parametrize("mol,basis,nbf", [("H2O", "sto-3g", 7), ("H2O", "6-31g*", 19), ("H2O", "cc-pvdz", 25),
                                           ("C6H6", "6-31g*", 102), ("C6H6", "6-31+g*", 126),
                                           ("CH4", "3-21g", 17), ("NH3", "6-31+G*", 25)])
def test_basis_build_counts(mol, basis, nbf):
    b = BasisSet.build(REFERENCE_MOLECULES[mol], basis)
    assert b.n_basis == nbf       # iqcp_iteration_counts.json n_basis
    assert np.all(b.exps > 0)
    assert b.offsets[-1] + (b.l[-1] + 1) * (b.l[-1] + 2) // 2 == nbf


def test_basis_name_aliases_and_errors():
    atoms = REFERENCE_MOLECULES["HF"]
    n = BasisSet.build(atoms, "6-31g(d)").n_basis
    assert n == BasisSet.build(atoms, "631gs").n_basis == BasisSet.build(atoms, "6-31G*").n_basis == 17
    with pytest.raises(IqcpError) as e:
        BasisSet.build(atoms, "def2-tzvp")
    assert e.value.code == -6
    with pytest.raises(IqcpError) as e:
        BasisSet.build([(19, (0.0, 0.0, 0.0))], "sto-3g")   # K: outside H..Ar
    assert e.value.code == -6


def test_631gs_d_exponents_follow_the_table():
    # builtin.rs:1039-1049: Li 0.2, Be 0.4, B 0.6, C..Ne 0.8; dedicated Na..Ar tables
    for z, e in [(3, 0.2), (4, 0.4), (5, 0.6), (6, 0.8), (9, 0.8)]:
        b = BasisSet.build([(z, (0.0, 0.0, 0.0))], "6-31g*")
        d = [i for i in range(b.n_shells) if b.l[i] == 2]
        assert len(d) == 1
        start = int(np.sum(b.nprim[:d[0]]))
        assert b.exps[start] == e and b.coefs[start] == 1.0


def test_compute_calls_fail_loudly_without_a_device():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    b = BasisSet.build(REFERENCE_MOLECULES["H2O"], "sto-3g")
    with pytest.raises(IqcpError) as e:
        iq.FockEngine(b)
    assert e.value.code == -5
    with pytest.raises(IqcpError):
        iq.rys_roots(3, [0.5])
    with pytest.raises(IqcpError):
        iq.boys_eval_all(4, [0.5])


def test_invalid_arguments_are_rejected():
    lib = iq.load_library()
    assert lib.iqcp_jk(None, None, None, None) == -1
    assert lib.iqcp_eri_grad(None, None, 1.0, None) == -1
    assert lib.iqcp_create(None, None, None) == -1
    assert lib.iqcp_rys_batch(0, 1, None, None, None) == -1
    assert lib.iqcp_rys_batch(8, 1, None, None, None) == -1
