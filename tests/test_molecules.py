"""The seeded workload generator keeps its geometric rules and is
deterministic per seed."""
import numpy as np
import pytest

from iqcp_b200 import ANGSTROM_TO_BOHR, BasisSet
from iqcp_b200.molecules import VALENCE, WORKLOADS, batch_geometries, generate, workload


@pytest.mark.parametrize("name", ["c1", "c2", "c3"])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_workload_rules(name, seed):
    atoms, basis = workload(name, seed)
    Z = np.array([a[0] for a in atoms])
    X = np.array([a[1] for a in atoms]) / ANGSTROM_TO_BOHR
    assert Z.sum() % 2 == 0                     # closed shell
    assert abs(len(atoms) - WORKLOADS[name]["n_atoms"]) <= 1
    heavy = np.where(Z > 1)[0]
    assert len(heavy) == WORKLOADS[name]["n_heavy"]
    d = np.linalg.norm(X[:, None] - X[None], axis=-1)
    # every heavy atom but the first has a bonded heavy neighbour at 1.40-1.55 A
    for i in heavy[1:]:
        dd = d[i, heavy[heavy != i]]
        assert np.any((dd >= 1.40 - 1e-9) & (dd <= 1.55 + 1e-9))
    # hydrogens sit 1.09 A from one heavy atom
    for h in np.where(Z == 1)[0]:
        assert np.isclose(d[h, heavy].min(), 1.09)
    # valences are respected
    b = BasisSet.build(atoms, basis)
    assert b.n_atoms == len(atoms)


def test_generator_is_deterministic():
    a1, _ = workload("c2", 3)
    a2, _ = workload("c2", 3)
    assert a1 == a2
    assert workload("c2", 4)[0] != a1


def test_workload_sizes():
    sizes = {n: BasisSet.build(*workload(n, 0)).n_basis for n in ("c1", "c2", "c3")}
    assert 60 <= sizes["c1"] <= 80          # ~70 basis functions, 6-31G
    assert 370 <= sizes["c2"] <= 420        # ~400, 6-31G*
    assert 280 <= sizes["c3"] <= 320        # ~300, cc-pVDZ


def test_batch_geometries_uneven():
    mols = batch_geometries(8, seed=0)
    n = [len(m) for m in mols]
    assert min(n) >= 7 and max(n) <= 48 and len(set(n)) > 1
    for m in mols:
        assert sum(z for z, _ in m) % 2 == 0
