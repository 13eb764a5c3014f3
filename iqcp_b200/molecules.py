"""Seeded synthetic closed-shell molecules for the Fock-build workloads.

The workloads are the reference-style synthetic molecules: heavy atoms on a
random tree with 1.40-1.55 A bonds, hydrogens at 1.09 A on the remaining
valences, non-bonded atoms at least 2.0 A apart (two hydrogens on the same
parent at least 1.5 A, since three 1.09 A bonds cannot also keep 2.0 A), and
the hydrogen count adjusted by one when needed so the electron count is even.
Coordinates are returned in bohr (ANGSTROM_TO_BOHR, constants.rs:63).
"""
import numpy as np

from . import ANGSTROM_TO_BOHR

VALENCE = {1: 1, 6: 4, 7: 3, 8: 2, 9: 1, 16: 2, 17: 1, 3: 1, 4: 2, 5: 3, 11: 1, 12: 2, 13: 3, 14: 4, 15: 3}
SYMBOL = {1: "H", 3: "Li", 4: "Be", 5: "B", 6: "C", 7: "N", 8: "O", 9: "F", 11: "Na", 12: "Mg", 13: "Al",
          14: "Si", 15: "P", 16: "S", 17: "Cl"}


def _unit(rng):
    v = rng.normal(size=3)
    return v / np.linalg.norm(v)


def generate(n_atoms, heavy_elements, n_heavy, seed, bond=(1.40, 1.55), h_bond=1.09, min_nonbonded=2.0,
             min_geminal_hh=1.5, max_tries=20000, weights=None):
    """Return a list of (Z, xyz_bohr) for a seeded random tree molecule.

    Heavy elements are drawn with `weights` (default: carbon-rich, so the tree
    keeps enough free valences for the hydrogens).  Element draws whose
    electron count would be odd at the requested hydrogen count are redrawn
    first; only if that keeps failing is the hydrogen count changed by one.
    """
    rng = np.random.default_rng(seed)
    heavy_elements = list(heavy_elements)
    if weights is None:
        weights = [0.55 if z == 6 else 1.0 for z in heavy_elements]
        weights = [w if z == 6 else 0.45 / (len(heavy_elements) - 1) for z, w in zip(heavy_elements, weights)] \
            if 6 in heavy_elements and len(heavy_elements) > 1 else [1.0] * len(heavy_elements)
    weights = np.array(weights, dtype=float) / np.sum(weights)
    for attempt in range(200):
        Z = [int(rng.choice(heavy_elements, p=weights)) for _ in range(n_heavy)]
        if attempt < 100 and (sum(Z) + n_atoms - n_heavy) % 2:
            continue
        pos = [np.zeros(3)]
        bonds = [0] * n_heavy
        parent = [-1] * n_heavy
        ok = True
        for i in range(1, n_heavy):
            placed = False
            for _ in range(max_tries):
                cands = [j for j in range(i) if bonds[j] < VALENCE[Z[j]]]
                if not cands:
                    break
                j = int(rng.choice(cands))
                p = pos[j] + _unit(rng) * rng.uniform(*bond)
                d = np.sqrt(((np.asarray(pos) - p) ** 2).sum(axis=1))
                d[j] = np.inf
                if np.all(d >= min_nonbonded):
                    pos.append(p)
                    bonds[j] += 1
                    bonds[i] = 1
                    parent[i] = j
                    placed = True
                    break
            if not placed:
                ok = False
                break
        if not ok:
            continue
        n_h = n_atoms - n_heavy
        free = sum(VALENCE[Z[i]] - bonds[i] for i in range(n_heavy))
        n_h = min(n_h, free)
        if (sum(Z) + n_h) % 2:
            n_h = n_h - 1 if n_h > 0 else n_h + 1
        h_pos, h_par = [], []
        heavy_xyz = np.asarray(pos)
        for _ in range(n_h):
            placed = False
            for _ in range(max_tries):
                cands = [j for j in range(n_heavy) if bonds[j] < VALENCE[Z[j]]]
                if not cands:
                    break
                j = int(rng.choice(cands))
                p = pos[j] + _unit(rng) * h_bond
                d = np.sqrt(((heavy_xyz - p) ** 2).sum(axis=1))
                d[j] = np.inf
                good = bool(np.all(d >= min_nonbonded))
                if good:
                    for q, par in zip(h_pos, h_par):
                        lim = min_geminal_hh if par == j else min_nonbonded
                        if np.linalg.norm(p - q) < lim:
                            good = False
                            break
                if good:
                    h_pos.append(p)
                    h_par.append(j)
                    bonds[j] += 1
                    placed = True
                    break
            if not placed:
                ok = False
                break
        if not ok or (sum(Z) + len(h_pos)) % 2:
            continue
        atoms = [(z, tuple(p * ANGSTROM_TO_BOHR)) for z, p in zip(Z, pos)]
        atoms += [(1, tuple(p * ANGSTROM_TO_BOHR)) for p in h_pos]
        return atoms
    raise RuntimeError("could not place the molecule; relax the constraints")


# Workload definitions: (atoms, heavy elements, heavy-atom count, basis)
WORKLOADS = {
    # ~70 basis functions, RHF/6-31G
    "c1": dict(n_atoms=12, heavy=(6, 7, 8), n_heavy=7, basis="6-31g"),
    # ~400 basis functions, RHF/6-31G*, (dd|dd) at Rys order 5
    "c2": dict(n_atoms=40, heavy=(6, 7, 8), n_heavy=24, basis="6-31g*"),
    # ~300 basis functions, RHF/cc-pVDZ gradient
    "c3": dict(n_atoms=30, heavy=(6, 7, 8, 9), n_heavy=15, basis="cc-pvdz"),
    # ~1100 basis functions, RHF/6-31+G*
    "c5": dict(n_atoms=100, heavy=(6, 7, 8, 16), n_heavy=53, basis="6-31+g*"),
}


def workload(name, seed=0):
    w = WORKLOADS[name]
    atoms = generate(w["n_atoms"], w["heavy"], w["n_heavy"], seed)
    return atoms, w["basis"]


def batch_geometries(n=256, seed=0, min_atoms=8, max_atoms=48, displacement=0.1):
    """Uneven batch: 8-48 atoms from H..Cl, each displaced by up to +-0.1 A.

    Heavy elements C, N, O, F, S, Cl (carbon-rich, so that the trees keep
    enough free valences); a draw that cannot be placed under the distance
    rules, or that ends with fewer atoms than drawn, is redrawn from the same
    seeded stream, so the set is reproducible."""
    rng = np.random.default_rng(seed)
    heavy = (6, 7, 8, 9, 16, 17)
    weights = (0.62, 0.12, 0.12, 0.04, 0.06, 0.04)
    out = []
    for g in range(n):
        na = int(rng.integers(min_atoms, max_atoms + 1))
        while True:
            nh = max(1, int(round(na * rng.uniform(0.45, 0.6))))
            try:
                atoms = generate(na, heavy, nh, int(rng.integers(1 << 30)), max_tries=400, weights=weights)
            except RuntimeError:
                continue
            if len(atoms) >= na - 1:
                break
        d = rng.uniform(-displacement, displacement, size=(len(atoms), 3)) * ANGSTROM_TO_BOHR
        out.append([(z, tuple(np.array(x) + dx)) for (z, x), dx in zip(atoms, d)])
    return out


# Reference test geometries (bohr), crates/qc-core/benches/scf_bench.rs:21-120
REFERENCE_MOLECULES = {
    "H2": [(1, (0.0, 0.0, 0.0)), (1, (0.0, 0.0, 1.4))],
    "HF": [(1, (0.0, 0.0, 0.0)), (9, (0.0, 0.0, 1.7328))],
    "H2O": [(8, (0.0, 0.0, 0.2217282)), (1, (0.0, 1.4305447, -0.8869128)), (1, (0.0, -1.4305447, -0.8869128))],
    "NH3": [(7, (0.0, 0.0, 0.219705)), (1, (0.0, 1.7714918, -0.512645)), (1, (1.5342036, -0.8857459, -0.512645)),
            (1, (-1.5342036, -0.8857459, -0.512645))],
    "CH4": [(6, (0.0, 0.0, 0.0)), (1, (1.1851, 1.1851, 1.1851)), (1, (-1.1851, -1.1851, 1.1851)),
            (1, (-1.1851, 1.1851, -1.1851)), (1, (1.1851, -1.1851, -1.1851))],
    "C6H6": [(6, (0.0, 2.6399473960, 0.0)), (6, (2.2861906655, 1.3199736980, 0.0)),
             (6, (2.2861906655, -1.3199736980, 0.0)), (6, (0.0, -2.6399473960, 0.0)),
             (6, (-2.2861906655, -1.3199736980, 0.0)), (6, (-2.2861906655, 1.3199736980, 0.0)),
             (1, (0.0, 4.6884105150, 0.0)), (1, (4.0602655512, 2.3442052575, 0.0)),
             (1, (4.0602655512, -2.3442052575, 0.0)), (1, (0.0, -4.6884105150, 0.0)),
             (1, (-4.0602655512, -2.3442052575, 0.0)), (1, (-4.0602655512, 2.3442052575, 0.0))],
}
