"""Molecule and basis construction feeding the Fock engine.

Mirrors the reference's host-side basis setup, which produces the Shell data
the C ABI consumes:
  * Angstrom -> Bohr with the reference's constant (src/base/tables.h:8);
  * shells per atom in basis-file order, SP split into S then P
    (src/basis/gaussian.cpp:122-143, 230-298);
  * primitive norms sqrt((2^(2L+1.5)/pi^1.5) alpha^(L+1.5)) (basis.cpp:39-48);
  * contracted norm folded into the coefficients (basis.cpp:50-75,
    gaussian.cpp:273-281);
  * Cartesian order lx descending then ly descending (basis.cpp:20-37) and
    component norms 1/sqrt((2lx-1)!!(2ly-1)!!(2lz-1)!!) (gaussian.cpp:283-296).
"""
import json
import os

import numpy as np

ANGSTROM_TO_BOHR = 1.8897259886
ZNUC = {"H": 1, "He": 2, "Li": 3, "Be": 4, "B": 5, "C": 6, "N": 7, "O": 8, "F": 9, "Ne": 10}
_PI = 3.1415926535897932384626433832795


DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "basis_sets.json")


def load_library(path=DATA):
    """Parsed basis sets {name: {element: [[L, [[exponent, raw coefficient], ...]], ...]}}
    for H, C, N, O in sto-3g, 3-21g, 6-31g*, 6-31g**, cc-pvdz (Basis Set
    Exchange data, SP shells split into S and P as the reference's parser does)."""
    with open(path) as f:
        return json.load(f)["basis"]


class Molecule:
    def __init__(self, atoms, charge=0, units="angstrom"):
        self.symbols = [a[0] for a in atoms]
        xyz = np.array([[a[1], a[2], a[3]] for a in atoms], dtype=np.float64).reshape(-1, 3)
        self.coords = xyz * ANGSTROM_TO_BOHR if units == "angstrom" else xyz
        self.Z = np.array([ZNUC[s] for s in self.symbols], dtype=np.float64)
        self.charge = charge

    def nelectron(self):
        return int(self.Z.sum()) - self.charge


def cartesian_order(L):
    return [(lx, ly, L - lx - ly) for lx in range(L, -1, -1) for ly in range(L - lx, -1, -1)]


def _dfact(n):
    r = 1
    while n > 0:
        r *= n
        n -= 2
    return r


def component_norm(lx, ly, lz):
    return 1.0 / np.sqrt(float(_dfact(2 * lx - 1) * _dfact(2 * ly - 1) * _dfact(2 * lz - 1)))


def normalize(L, expo, raw):
    """Primitive norms and Nc-folded coefficients (basis.cpp:39-75)."""
    expo = np.asarray(expo, dtype=np.float64)
    raw = np.asarray(raw, dtype=np.float64)
    prefactor = 2.0 ** (2.0 * L + 1.5) / _PI ** 1.5
    norm = np.sqrt(expo ** (L + 1.5) * prefactor)
    aij = expo[:, None] + expo[None, :]
    sij = (_PI ** 1.5 / 2.0 ** L) / aij ** (L + 1.5)
    total = 0.0
    n = len(expo)
    for j in range(n):            # same summation order as the oracle
        for i in range(n):
            total += raw[i] * raw[j] * norm[i] * norm[j] * sij[i, j]
    return raw * (1.0 / np.sqrt(total)), norm


def read_gbs_basis(library, basis_name, mol):
    """Shell arrays for `mol` from a parsed basis library
    {basis: {element: [[L, [[exponent, raw coefficient], ...]], ...]}}."""
    data = library[basis_name]
    L, nprim, center, expo, coef, norm = [], [], [], [], [], []
    for sym, xyz in zip(mol.symbols, mol.coords):
        if sym not in data:
            raise ValueError(f"Unsupported Element: {sym}")
        for l, prims in data[sym]:
            e = [p[0] for p in prims]
            c, nrm = normalize(l, e, [p[1] for p in prims])
            L.append(l)
            nprim.append(len(prims))
            center.append(xyz)
            expo.extend(e)
            coef.extend(c)
            norm.extend(nrm)
    return {"L": np.array(L, dtype=np.int32), "nprim": np.array(nprim, dtype=np.int32),
            "center": np.ascontiguousarray(np.array(center, dtype=np.float64).reshape(-1, 3)),
            "expo": np.array(expo, dtype=np.float64), "coef": np.array(coef, dtype=np.float64),
            "norm": np.array(norm, dtype=np.float64)}


def shells_for(atoms, basis_name, library, charge=0, units="angstrom"):
    mol = Molecule(atoms, charge=charge, units=units)
    return mol, read_gbs_basis(library, basis_name, mol)
