"""Geometry of the learned guess (CPU tests): rotation of Cartesian shells,
invariance of the pair features and of the local-frame density blocks under
rigid motions, block assembly and the purification step.  The density of
the block test comes from the oracle's conventional RHF (the reference's
algorithm restated)."""
import importlib

import numpy as np
import pytest

import oracle
from helpers import pfk


def _rot(seed):
    q, _ = np.linalg.qr(np.random.default_rng(seed).normal(size=(3, 3)))
    return q * np.sign(np.linalg.det(q))


@pytest.mark.parametrize("L", [0, 1, 2, 3])
def test_shell_rotation_is_a_representation(L):
    G = importlib.import_module("planck-refactored_b200.guess")
    R1, R2 = _rot(1), _rot(2)
    D = G.shell_rotation
    n = (L + 1) * (L + 2) // 2
    assert np.allclose(D(L, R1) @ D(L, R1.T), np.eye(n), atol=1e-12)
    assert np.allclose(D(L, R2 @ R1), D(L, R2) @ D(L, R1), atol=1e-12)
    assert np.allclose(D(L, np.stack([R1, R2]))[1], D(L, R2), atol=1e-14)


def _moved(atoms, R, shift):
    return [[a[0], *(R @ np.array(a[1:]) + shift)] for a in atoms]


def test_features_invariant_under_rigid_motion():
    P = pfk()
    G = importlib.import_module("planck-refactored_b200.guess")
    atoms = P.workloads.alkane_conformer(7, seed=4)
    moved = _moved(atoms, _rot(7), np.array([1.5, -2.0, 0.3]))
    d1 = G.pair_data(P.Molecule(atoms))
    d2 = G.pair_data(P.Molecule(moved))
    for t in G.TYPES:
        assert np.array_equal(d1[t][0], d2[t][0])
        assert np.abs(d1[t][2] - d2[t][2]).max() < 1e-5
        assert d1[t][2].shape[1] == G.NFEAT


def test_local_blocks_invariant_and_assembly_exact():
    """Ethane/6-31G*: the converged density's local-frame blocks are the same
    for the molecule and a rigidly moved copy, and assembling them gives the
    density back (all pairs are within the cutoff)."""
    P = pfk()
    G = importlib.import_module("planck-refactored_b200.guess")
    atoms = P.workloads.alkane_conformer(2, seed=1)
    moved = _moved(atoms, _rot(3), np.array([0.4, 0.1, -0.7]))
    res = []
    for at in (atoms, moved):
        r = oracle.rhf_conventional(at, "6-31g*")
        assert r["converged"]
        mol = P.Molecule(at)
        _, shells = P.shells_for(at, "6-31g*", P.basis.load_library())
        layout = G.atom_layout(mol, shells)
        data = G.pair_data(mol)
        blocks = {t: G.local_blocks(r["P"], layout, v[0], v[1]) for t, v in data.items()}
        Pa = G.assemble(r["P"].shape[0], layout, {t: (v[0], v[1]) for t, v in data.items()}, blocks)
        assert np.abs(Pa - r["P"]).max() < 1e-12
        res.append(blocks)
    for t in G.TYPES:
        if res[0][t].size:
            assert np.abs(res[0][t] - res[1][t]).max() < 1e-6


def test_purify_gives_idempotent_density_with_the_electron_count():
    P = pfk()
    G = importlib.import_module("planck-refactored_b200.guess")
    atoms = P.workloads.alkane_conformer(3, seed=2)
    mol = oracle.Molecule(atoms)
    ob = oracle.Basis(oracle.shells_for(mol, "6-31g*"))
    S, T, V = ob.one_electron(mol)
    nocc = mol.nelectron() // 2
    rng = np.random.default_rng(0)
    A = rng.normal(size=S.shape) * 0.1
    Pp = G.purify(A + A.T, S, nocc)
    assert np.allclose(Pp @ S @ Pp, 2.0 * Pp, atol=1e-10)
    assert abs(np.trace(Pp @ S) - 2 * nocc) < 1e-10
    assert np.allclose(G.purify(Pp, S, nocc), Pp, atol=1e-10)
