"""Parity of the CUDA Fock engine with the oracle (GPU tests).

Tolerances (the project's accuracy targets): integrals within 1e-10 absolute on the FP64 path;
G/J/K within 1e-10 absolute; converged energies within 1e-8 Eh of the oracle
and within the reference's own 1e-9 of its regression energies.  Screened
quartet sets must be identical (count and digest)."""
import numpy as np
import pytest

import oracle
from helpers import (WATER, alkane, basis_library, pfk, random_density, random_shells, regression_cases,
                     water_cluster)

pytestmark = pytest.mark.gpu

ETHYLENE = regression_cases()["ethylene_rhf_ccpvdz_auto"]["atoms"]


def _setup(atoms, basis, engine="os"):
    P = pfk()
    mol, shells = P.shells_for(atoms, basis, basis_library())
    eng = P.FockEngine(shells, engine=engine)
    ob = oracle.Basis(oracle.shells_for(oracle.Molecule(atoms), basis))
    return eng, ob, mol


@pytest.fixture(scope="module")
def water():
    return _setup(WATER, "6-31g**")


@pytest.fixture(scope="module")
def ethylene():
    return _setup(ETHYLENE, "cc-pvdz")


def test_schwarz_table(water, ethylene):
    for eng, ob, _ in (water, ethylene):
        Qg = eng.schwarz()
        Qo = ob.schwarz(oracle.OS)
        assert np.abs(Qg - Qo).max() < 1e-12 * max(1.0, Qo.max())


@pytest.mark.parametrize("which", ["water", "ethylene"])
def test_quartet_set_bit_exact(which, water, ethylene):
    eng, ob, _ = water if which == "water" else ethylene
    Qo = ob.schwarz(oracle.OS)
    n_o, dig_o, lst_o = ob.quartet_list(1e-10, Qo, want_list=True)
    n_g, dig_g, n_shell = eng.quartet_count()
    assert n_g == n_o
    assert dig_g == dig_o
    lst_g = eng.quartet_list()
    a = {tuple(x) for x in lst_g.tolist()}
    b = {tuple(x) for x in lst_o.tolist()}
    assert a == b


@pytest.mark.parametrize("engine", ["os", "rys"])
def test_eri_tensor_water(water, engine):
    eng, ob, _ = water
    eng.set_options(1e-10, engine)
    eri_g = eng.eri_tensor()
    eri_o, _ = ob.eri_tensor(1e-10, oracle.OS if engine == "os" else oracle.RYS)
    assert np.abs(eri_g - eri_o).max() < 1e-10
    eng.set_options(1e-10, "os")


def test_eri_tensor_ethylene(ethylene):
    eng, ob, _ = ethylene
    eri_g = eng.eri_tensor()
    eri_o, _ = ob.eri_tensor(1e-10, oracle.OS)
    assert np.abs(eri_g - eri_o).max() < 1e-10


def test_eri_tensor_random_f_shells():
    """Random shells with s..f, contraction depth up to 6 and exponents up to
    1e4 (the ERI class microbenchmark's distributions), every class present.

    (a) Against 60-digit values (tests/golden/eri_highprec.json): 1e-12
        relative to max(1, |v|), on the quartets where the reference's own
        OS and Rys engines disagree most plus a random sample.
    (b) Against the oracle on 3000 sampled canonical AO quartets: 1e-10
        relative to max(1, |v|) on at least 95% of them.  The reference
        algorithm (which the oracle restates) loses up to ~3e-7 absolute on
        this basis to cancellation in its A->B transfer with the lower-L
        centre first; the 12 sampled quartets furthest outside 1e-10 are
        re-evaluated at 60 digits, and there the CUDA value must be the
        accurate one."""
    import json
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_eri_highprec as highprec
    P = pfk()
    fx = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "eri_highprec.json")))
    shells = random_shells(fx["nshell"], lmax=3, seed=fx["seed"], box=fx["box_angstrom"])
    eng = P.FockEngine(shells)
    eri_g = eng.eri_tensor()
    worst = 0.0
    for q, v, _, _ in fx["quartets"]:
        v = float(v)
        err = abs(eri_g[tuple(q)] - v) / max(1.0, abs(v))
        worst = max(worst, err)
    assert worst < 1e-12, worst
    ob = oracle.Basis(shells)
    shell, lxyz, _ = ob.ao_info()
    rng = np.random.default_rng(5)
    pairs = rng.integers(0, ob.npairs, size=(3000, 2))
    iu = np.triu_indices(eng.nbasis)
    outside = []
    for p, q in pairs:
        p, q = int(p), int(q)
        v_os = ob.eri_pair(p, q, oracle.OS)
        i, j, k, l = (int(x) for x in (iu[0][p], iu[1][p], iu[0][q], iu[1][q]))
        if abs(eri_g[i, j, k, l] - v_os) > 1e-10 * max(1.0, abs(v_os)):
            outside.append(((i, j, k, l), v_os))
    assert len(outside) <= 150, len(outside)
    outside.sort(key=lambda e: -abs(eri_g[e[0]] - e[1]) / max(1.0, abs(e[1])))
    for (i, j, k, l), v_os in outside[:12]:
        ao = [(int(shell[x]), tuple(int(c) for c in lxyz[x])) for x in (i, j, k, l)]
        v = float(highprec.eri(shells, ao))
        assert abs(eri_g[i, j, k, l] - v) < 1e-12 * max(1.0, abs(v))
        assert abs(eri_g[i, j, k, l] - v) < abs(v_os - v)


@pytest.mark.parametrize("which", ["water", "ethylene"])
def test_fock_rhf(which, water, ethylene):
    eng, ob, _ = water if which == "water" else ethylene
    nb = eng.nbasis
    Pm = random_density(nb, seed=3)
    eri_o, _ = ob.eri_tensor(1e-10, oracle.OS)
    G_o = oracle.fock_rhf_tensor(eri_o, Pm)
    G_g = eng.fock_rhf(Pm)
    assert np.abs(G_g - G_o).max() < 1e-10
    assert np.abs(G_g - G_g.T).max() < 1e-13


def test_fock_uhf(water):
    eng, ob, _ = water
    nb = eng.nbasis
    Pa, Pb = random_density(nb, seed=4), random_density(nb, seed=5)
    eri_o, _ = ob.eri_tensor(1e-10, oracle.OS)
    Ga_o, Gb_o = oracle.fock_uhf_tensor(eri_o, Pa, Pb)
    Ga, Gb = eng.fock_uhf(Pa, Pb)
    assert np.abs(Ga - Ga_o).max() < 1e-10
    assert np.abs(Gb - Gb_o).max() < 1e-10


def test_jk_against_streaming_oracle(ethylene):
    eng, ob, _ = ethylene
    nb = eng.nbasis
    Pm = random_density(nb, seed=6)
    Pk = random_density(nb, seed=7)
    J_o, K_o, _ = ob.jk_direct(Pm, [Pk], 1e-10, oracle.OS)
    J, K = eng.jk(Pm, Pk, k_scale=0.25)
    assert np.abs(J - J_o).max() < 1e-10
    assert np.abs(K - 0.25 * K_o[0]).max() < 1e-10


def test_device_graph_path_matches_host(water):
    torch = pytest.importorskip("torch")
    eng, ob, _ = water
    nb = eng.nbasis
    Pm = random_density(nb, seed=8)
    G_host = eng.fock_rhf(Pm)
    dP = torch.tensor(Pm, device="cuda:0", dtype=torch.float64)
    dG = torch.zeros_like(dP)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        for _ in range(3):   # first call captures, later calls replay the graph
            dG.zero_()
            eng.fock_rhf_device(dP.data_ptr(), dG.data_ptr(), s.cuda_stream)
        # the context's own stream when no stream is given
        eng.fock_rhf_device(dP.data_ptr(), dG.data_ptr(), 0)
    torch.cuda.synchronize()
    assert np.abs(dG.cpu().numpy() - G_host).max() < 1e-12


def _scf(eng, mol, ob, max_iter=None):
    S, T, V = ob.one_electron(mol)
    return oracle.rhf(T + V, S, mol.nuclear_repulsion(), mol.nelectron() // 2,
                      lambda P: eng.fock_rhf(P), max_iter=max_iter)


@pytest.mark.parametrize("case_id", ["water_rhf_stability_stable", "ethylene_rhf_ccpvdz_auto"])
def test_rhf_energy_matches_reference_regressions(case_id):
    c = regression_cases()[case_id]
    eng, ob, _ = _setup(c["atoms"], c["basis"], c["engine"])
    omol = oracle.Molecule(c["atoms"])
    r = _scf(eng, omol, ob, max_iter=c["max_cycles"] or None)
    assert r["converged"]
    assert abs(r["energy"] - c["energy"]) < c["atol"]


def test_rhf_water_631gss_matches_oracle():
    """The configuration the reference runs on CPU today (water/6-31G**, DIIS,
    hcore guess, 1e-10): GPU direct SCF energy vs the oracle's within 1e-8."""
    eng, ob, _ = _setup(WATER, "6-31g**")
    omol = oracle.Molecule(WATER)
    r_g = _scf(eng, omol, ob)
    r_o = oracle.rhf_conventional(WATER, "6-31g**")
    assert r_g["converged"] and r_o["converged"]
    assert abs(r_g["energy"] - r_o["energy"]) < 1e-8


def test_larger_systems_quartet_set_and_fock():
    """Three waters and butane: quartet set identical, G against the
    streaming oracle within 1e-10."""
    for atoms, basis in ((water_cluster(3, seed=4), "6-31g**"), (alkane(4), "6-31g*")):
        eng, ob, _ = _setup(atoms, basis)
        Qo = ob.schwarz(oracle.OS)
        n_o, dig_o, _ = ob.quartet_list(1e-10, Qo)
        n_g, dig_g, _ = eng.quartet_count()
        assert (n_g, dig_g) == (n_o, dig_o)
        Pm = random_density(eng.nbasis, seed=9, scale=0.1)
        J_o, K_o, _ = ob.jk_direct(Pm, [Pm], 1e-10, oracle.OS, Q=Qo)
        G_o = J_o - 0.5 * K_o[0]
        assert np.abs(eng.fock_rhf(Pm) - G_o).max() < 1e-10


def test_rejects_asymmetric_and_nonfinite_density(water):
    """pfk_fock_rhf checks its density on the host before any device work:
    asymmetric (above 1e-10 relative) or non-finite densities fail with
    PFK_ERR_INVALID and a message; a density asymmetric at the rounding level
    is accepted."""
    P = pfk()
    eng = water[0]
    Pm = random_density(eng.nbasis, seed=3)
    G = eng.fock_rhf(Pm)
    Pn = Pm.copy()
    Pn[0, 1] += 1e-15
    assert np.abs(eng.fock_rhf(Pn) - G).max() < 1e-12
    for bad in ("asym", "nan", "inf"):
        Pb = Pm.copy()
        if bad == "asym":
            Pb[3, 7] += 1e-6
        else:
            Pb[5, 5] = np.nan if bad == "nan" else np.inf
        with pytest.raises(P.PfkError) as e:
            eng.fock_rhf(Pb)
        assert e.value.status == 1 and "not symmetric" in str(e.value)
