"""The oracle's basis builder (oracle/basis.py, no product library) against the
product's iqcp_basis_build, for every element H..Ar in every built-in basis
and for the benchmark workloads; both restate BasisSet::build
(basis/mod.rs:164) over the tables extracted from basis/builtin.rs."""
import numpy as np
import pytest

from iqcp_b200 import BasisSet, IqcpError
from iqcp_b200.molecules import workload
from oracle.basis import build_basis

FIELDS = ["l", "nprim", "atom_of_shell", "center", "exps", "coefs", "z", "xyz"]


@pytest.mark.parametrize("basis", ["sto-3g", "3-21g", "6-31g", "6-31g*", "6-31+g*", "cc-pvdz"])
def test_every_element(basis):
    atoms = [(z, (0.1 * z, -0.2 * z, 0.05 * z)) for z in range(1, 19)]
    try:
        pb = BasisSet.build(atoms, basis)
    except IqcpError:
        pytest.skip("basis lacks an element")
    ob = build_basis(atoms, basis)
    for f in FIELDS:
        assert np.array_equal(getattr(ob, f), getattr(pb, f)), f
    assert ob.n_basis == pb.n_basis


@pytest.mark.parametrize("name", ["c1", "c2", "c3", "c5"])
def test_workloads(name):
    atoms, basis = workload(name, 0)
    ob, pb = build_basis(atoms, basis), BasisSet.build(atoms, basis)
    for f in FIELDS:
        assert np.array_equal(getattr(ob, f), getattr(pb, f)), f


def test_unknown_basis_and_element():
    with pytest.raises(KeyError):
        build_basis([(1, (0, 0, 0))], "def2-svp")
    with pytest.raises(ValueError):
        build_basis([(19, (0, 0, 0))], "sto-3g")
