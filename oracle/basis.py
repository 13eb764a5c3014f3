"""Oracle-side basis builder: TEST INFRASTRUCTURE ONLY.

A pure-Python restatement of ``BasisSet::build`` (crates/qc-core/src/basis/mod.rs:164)
with ``get_element_basis`` (basis/builtin.rs:97): shells per atom in table order,
raw tabulated contraction coefficients, Cartesian function counts.  The table
data are read as text from the generated ``iqcp_b200/csrc/basis_tables.inc``
(mechanically extracted from builtin.rs), so the oracle, the CPU baseline and
the reference arm of the benchmark build bases without loading the product
library.  ``tests/test_oracle_basis.py`` checks this builder against the
product's ``iqcp_basis_build`` for every element and basis.
"""
import os
import re

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_TABLES = os.path.join(os.path.dirname(_HERE), "iqcp_b200", "csrc", "basis_tables.inc")
_CACHE = None

BASIS_IDS = {"sto-3g": 0, "sto3g": 0, "3-21g": 1, "321g": 1, "6-31g": 2, "631g": 2,
             "6-31g*": 3, "631g*": 3, "6-31gs": 3, "631gs": 3, "6-31g(d)": 3, "631g(d)": 3,
             "6-31+g*": 4, "631+g*": 4, "6-31+gs": 4, "631+gs": 4, "6-31+g(d)": 4, "631+g(d)": 4,
             "cc-pvdz": 5, "ccpvdz": 5}


def _tables():
    global _CACHE
    if _CACHE is None:
        src = open(_TABLES).read()
        rec = src[src.index("kShellRecords["):src.index("kPrimitives[")]
        prim = src[src.index("kPrimitives["):]
        records = [tuple(int(x) for x in m) for m in
                   re.findall(r"\{\s*(\d+),\s*(\d+),\s*(\d+),\s*(\d+),\s*(\d+)\s*\}", rec)]
        num = r"[-+]?\d+\.?\d*(?:[eE][-+]?\d+)?"
        prims = [(float(a), float(b)) for a, b in re.findall(r"\{\s*(%s),\s*(%s)\s*\}" % (num, num), prim)]
        _CACHE = (records, prims)
    return _CACHE


class OracleBasis:
    """Shell arrays in the layout the oracle's C entry points take."""

    def __init__(self, name, z, xyz, l, nprim, atom_of_shell, center, exps, coefs):
        self.name = name
        self.z = np.ascontiguousarray(z, dtype=np.int32)
        self.xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        self.l = np.ascontiguousarray(l, dtype=np.int32)
        self.nprim = np.ascontiguousarray(nprim, dtype=np.int32)
        self.atom_of_shell = np.ascontiguousarray(atom_of_shell, dtype=np.int32)
        self.center = np.ascontiguousarray(center, dtype=np.float64).reshape(-1, 3)
        self.exps = np.ascontiguousarray(exps, dtype=np.float64)
        self.coefs = np.ascontiguousarray(coefs, dtype=np.float64)
        self.n_basis = int(((self.l + 1) * (self.l + 2) // 2).sum())
        self.n_electrons = int(self.z.sum())

    @property
    def n_shells(self):
        return len(self.l)

    @property
    def n_atoms(self):
        return len(self.z)

    def as_args(self):
        return (self.n_shells, self.l, self.nprim, self.atom_of_shell, self.center, self.exps, self.coefs,
                self.n_atoms, self.xyz, self.z)


def build_basis(atoms, basis_name):
    """atoms: list of (Z, (x, y, z) bohr).  Raises KeyError / ValueError like
    the reference's unknown-basis / unsupported-element errors."""
    key = "".join(ch for ch in basis_name.lower() if ch not in " _")
    bid = BASIS_IDS[key]
    records, prims = _tables()
    l, nprim, aos, center, exps, coefs = [], [], [], [], [], []
    for a, (z, pos) in enumerate(atoms):
        if not 1 <= z <= 18:
            raise ValueError("element Z=%d outside H..Ar" % z)
        for (b, zz, ll, npr, first) in records:
            if b != bid or zz != z:
                continue
            l.append(ll)
            nprim.append(npr)
            aos.append(a)
            center.append(pos)
            for k in range(npr):
                exps.append(prims[first + k][0])
                coefs.append(prims[first + k][1])
    return OracleBasis(key, [z for z, _ in atoms], [p for _, p in atoms], l, nprim, aos, center, exps, coefs)
