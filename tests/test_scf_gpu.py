"""One-electron integrals on the device and the RHF driver around the GPU
Fock build (GPU tests).

pfk_one_electron is checked against the oracle's restatement of the
reference's one-electron code (os.cpp:294-602), and the driver
(planck-refactored_b200/scf.py, the loop of scf.cpp:175-441) against the
reference's regression energies and iteration counts, with every matrix it
uses coming from this repository's GPU code."""
import numpy as np
import pytest

import oracle
from helpers import (WATER, alkane, basis_library, onee_highprec, pfk, random_shells, regression_cases,
                     water_cluster)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", ["water_631gss", "ethylene_ccpvdz", "random_f"])
def test_one_electron_matches_oracle(which):
    P = pfk()
    if which == "random_f":
        shells = random_shells(10, lmax=3, seed=31, box=3.0)
        rng = np.random.default_rng(2)
        coords = rng.uniform(0, 3.0 * P.basis.ANGSTROM_TO_BOHR, (4, 3))
        Z = np.array([1.0, 6.0, 8.0, 7.0])

        class M:  # oracle's one_electron reads coords and Z
            pass
        mol = M()
        mol.coords, mol.Z = coords, Z
    else:
        atoms, basis = (WATER, "6-31g**") if which == "water_631gss" else \
            (regression_cases()["ethylene_rhf_ccpvdz_auto"]["atoms"], "cc-pvdz")
        mol, shells = P.shells_for(atoms, basis, basis_library())
        coords, Z = mol.coords, mol.Z
    S, T, V = P.one_electron(shells, coords, Z)
    So, To, Vo = oracle.Basis(shells).one_electron(mol)
    if which == "random_f":
        # the reference's own V is off by up to 7e-9 on this basis (its
        # (f|V|f) diagonal blocks); the 40-digit values decide V instead
        assert np.array_equal(coords, onee_highprec()["coords"])
        Vo = onee_highprec()["V"]
    for A, B in ((S, So), (T, To), (V, Vo)):
        assert np.abs(A - B).max() < 1e-10 * max(1.0, np.abs(B).max())
    assert np.array_equal(S, S.T) and np.array_equal(V, V.T)


@pytest.mark.parametrize("case_id", ["ethylene_rhf_ccpvdz_auto", "ethylene_rhf_ccpvdz_rys",
                                     "water_rhf_stability_stable"])
def test_rhf_driver_matches_reference_regressions(case_id):
    """Energy within the reference's own tolerance (1e-9 Eh) and, where the
    regression records it, the same iteration count."""
    P = pfk()
    c = regression_cases()[case_id]
    sysm = P.scf.System(c["atoms"], c["basis"], basis_library(), engine=c["engine"])
    r = sysm.run(max_iter=c["max_cycles"] or None)
    sysm.close()
    assert r["converged"]
    assert abs(r["energy"] - c["energy"]) < c["atol"]
    if "iterations" in c:
        # the iteration that first meets the 1e-10 tests can move by one with
        # 1e-12-level integral differences (the reference's Rys engine is less
        # accurate than its OS engine and than this library's Rys kernels);
        # engine auto matches exactly
        assert abs(r["iterations"] - c["iterations"]) <= (0 if c["engine"] == "auto" else 1)


def test_incremental_fp32_difference_builds():
    """Difference-density builds in FP32 once max|dP| < 1e-4 (full FP64
    builds otherwise, at least every 8 iterations and at the end): converged
    energy within 1e-6 Eh of the all-FP64 run, at most 3 more iterations."""
    P = pfk()
    sysm = P.scf.System(water_cluster(4, seed=7), "6-31g**", basis_library())
    r64 = sysm.run()
    r32 = sysm.run(incremental=True)
    sysm.close()
    assert r64["converged"] and r32["converged"]
    assert abs(r32["energy"] - r64["energy"]) < 1e-6
    assert r32["iterations"] <= r64["iterations"] + 3


def test_rhf_driver_on_an_alkane_matches_oracle_loop():
    """Butane / 6-31G*: the driver and the oracle's restated loop, both on
    the GPU Fock build, converge to the same energy (1e-8 Eh)."""
    P = pfk()
    atoms = alkane(4)
    sysm = P.scf.System(atoms, "6-31g*", basis_library())
    r = sysm.run()
    omol = oracle.Molecule(atoms)
    ob = oracle.Basis(oracle.shells_for(omol, "6-31g*"))
    S, T, V = ob.one_electron(omol)
    ro = oracle.rhf(T + V, S, omol.nuclear_repulsion(), omol.nelectron() // 2, sysm.engine.fock_rhf)
    sysm.close()
    assert r["converged"] and ro["converged"]
    assert abs(r["energy"] - ro["energy"]) < 1e-8


def test_density_screening_of_a_difference_build():
    """Screened build of a small difference density: within 1e-10 of the
    unscreened one (every skipped AO quartet contributes below 1e-12 per
    density element; a G element collects a few thousand of them), and a
    screened build of a zero density is exactly zero."""
    P = pfk()
    mol, shells = P.shells_for(water_cluster(3, seed=2), "6-31g**", basis_library())
    eng = P.FockEngine(shells)
    nb = eng.nbasis
    rng = np.random.default_rng(1)
    A = rng.normal(size=(nb, nb)) * 1e-7
    dP = A + A.T
    G_full = eng.fock_rhf(dP)
    eng.set_density_screening(1e-12)
    G_scr = eng.fock_rhf(dP)
    G_zero = eng.fock_rhf(np.zeros((nb, nb)))
    eng.set_density_screening(0.0)
    G_again = eng.fock_rhf(dP)
    eng.close()
    assert np.abs(G_scr - G_full).max() < 1e-10
    assert not np.any(G_zero)
    assert np.abs(G_again - G_full).max() < 1e-15


def test_device_linear_algebra_loop_matches_the_host_loop():
    """scf.rhf_device (density in HBM, eigh and DIIS on the GPU) converges to
    the host loop's energy (1e-9 Eh) within a couple of iterations of it, from
    the default guess and from a supplied density."""
    P = pfk()
    sysm = P.scf.System(water_cluster(3, seed=5), "6-31g**", basis_library())
    r_h = sysm.run()
    r_d = sysm.run(linalg="device")
    r_d2 = sysm.run(P0=r_h["P"], linalg="device")
    sysm.close()
    assert r_h["converged"] and r_d["converged"] and r_d2["converged"]
    assert abs(r_d["energy"] - r_h["energy"]) < 1e-9
    assert abs(r_d["iterations"] - r_h["iterations"]) <= 2
    assert r_d2["iterations"] <= 3 and abs(r_d2["energy"] - r_h["energy"]) < 1e-9
    assert r_d["build_seconds"] > 0


@pytest.mark.parametrize("case_id", ["ethylene_rhf_ccpvdz_auto", "water_rhf_stability_stable"])
def test_c_abi_scf_loop_matches_reference_regressions(case_id):
    """pfk_scf_rhf (the whole loop behind the C ABI: DIIS and Dsyevd on the
    device) reproduces the reference's regression energies within its 1e-9 Eh
    and its recorded iteration count within one (the DIIS solve and the
    eigensolver round differently from the host loop's)."""
    P = pfk()
    c = regression_cases()[case_id]
    sysm = P.scf.System(c["atoms"], c["basis"], basis_library(), engine=c["engine"])
    r = sysm.run(linalg="gpu", max_iter=c["max_cycles"] or 0)
    sysm.close()
    assert r["converged"]
    assert abs(r["energy"] - c["energy"]) < c["atol"]
    if "iterations" in c:
        assert abs(r["iterations"] - c["iterations"]) <= 1


def test_c_abi_scf_loops_in_threads_repeat_bitwise():
    """Three device SCF loops (pfk_scf_rhf, one context each) run at once
    from host threads -- the way guess_train.py evaluate --batch runs the
    held-out set -- give bitwise the energies, densities and iteration
    counts of the same loops run one after the other."""
    from concurrent.futures import ThreadPoolExecutor
    P = pfk()
    systems = [P.scf.System(water_cluster(n, seed=11 + n), "6-31g**", basis_library()) for n in (2, 3, 4)]
    seq = [s.run(linalg="gpu") for s in systems]
    with ThreadPoolExecutor(3) as pool:
        par = list(pool.map(lambda s: s.run(linalg="gpu"), systems))
    for s in systems:
        s.close()
    for a, b in zip(seq, par):
        assert a["converged"] and b["converged"]
        assert a["energy"] == b["energy"] and a["iterations"] == b["iterations"]
        assert np.array_equal(a["P"], b["P"])


def test_c_abi_scf_loop_matches_host_loop_and_repeats():
    """(H2O)4 / 6-31G**: the C-ABI loop takes the host loop's steps -- the same
    energy at every iteration (1e-9 Eh) while the density steps are above 1e-8
    -- and converges to its energy (1e-9 Eh); three runs repeat bitwise; a run
    from the converged density stops at once; FP32 difference builds keep the
    energy within 1e-6 Eh.  (Below ~1e-8 both loops wander at the rounding
    level until one step meets the 1e-10 tests, so their iteration counts
    differ by the luck of that tail.)"""
    P = pfk()
    sysm = P.scf.System(water_cluster(4, seed=7), "6-31g**", basis_library())
    r_h = sysm.run()
    runs = [sysm.run(linalg="gpu") for _ in range(3)]
    r_p = sysm.run(P0=r_h["P"], linalg="gpu")
    r_i = sysm.run(linalg="gpu", incremental=True)
    sysm.close()
    r = runs[0]
    assert r_h["converged"] and r["converged"] and r_p["converged"] and r_i["converged"]
    assert abs(r["energy"] - r_h["energy"]) < 1e-9
    steps = [(a, b) for a, b in zip(r_h["history"], r["history"]) if a[3] > 1e-8]
    assert len(steps) >= 10
    assert all(abs(a[1] - b[1]) < 1e-9 for a, b in steps)
    assert all(x["energy"] == r["energy"] and x["iterations"] == r["iterations"] for x in runs)
    assert np.array_equal(runs[1]["P"], r["P"])
    assert r_p["iterations"] <= 3 and abs(r_p["energy"] - r_h["energy"]) < 1e-9
    assert abs(r_i["energy"] - r["energy"]) < 1e-6 and r_i["difference_builds"] > 0
    nocc = sysm.nocc
    assert np.allclose(2.0 * r["C"][:, :nocc] @ r["C"][:, :nocc].T, r["P"], atol=1e-9)
