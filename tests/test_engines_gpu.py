"""The two device integral engines (GPU tests).

`engine os` and `engine auto` run the Obara-Saika kernels (pfk_os.cuh) for
every class with LA+LB+LC+LD <= 4 -- the classes where the reference's
per-quartet auto choice picks OS for every component quartet (rys.cpp:195-236)
-- and the Rys kernels for the larger classes; `engine rys` runs Rys for all
classes.  The two engines evaluate the same integrals by different
recurrences, so they must agree to rounding, and each must match the oracle's
restatement of the corresponding reference engine."""
import numpy as np
import pytest

import oracle
from helpers import WATER, basis_library, pfk, random_density, random_shells

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def random_basis():
    # s, p and d shells, contraction depth 1-6, exponents up to 1e4, centres
    # in a 2.5 Angstrom cube: every class up to (dd|dd) is present
    return random_shells(9, lmax=2, seed=21, box=2.5)


def test_os_and_rys_kernels_agree(random_basis):
    P = pfk()
    eng = P.FockEngine(random_basis, engine="os")
    eri_os = eng.eri_tensor()
    eng.set_options(1e-10, "rys")
    eri_rys = eng.eri_tensor()
    eng.close()
    scale = np.maximum(1.0, np.abs(eri_rys))
    assert np.max(np.abs(eri_os - eri_rys) / scale) < 1e-12


def test_os_kernels_match_oracle_os(random_basis):
    P = pfk()
    eng = P.FockEngine(random_basis, engine="os")
    eri_g = eng.eri_tensor()
    eng.close()
    ob = oracle.Basis(random_basis)
    eri_o, _ = ob.eri_tensor(1e-10, oracle.OS)
    assert np.max(np.abs(eri_g - eri_o) / np.maximum(1.0, np.abs(eri_o))) < 1e-10


def test_engine_auto_runs_the_os_kernels(random_basis):
    P = pfk()
    eng = P.FockEngine(random_basis, engine="auto")
    eri_auto = eng.eri_tensor()
    eng.set_options(1e-10, "os")
    eri_os = eng.eri_tensor()
    eng.close()
    assert np.array_equal(eri_auto, eri_os)


def test_engine_switches_between_device_builds():
    """Engine changes between captured device builds (each change drops the
    captured graphs): every build stays within 1e-10 of the oracle's G."""
    torch = pytest.importorskip("torch")
    P = pfk()
    mol, shells = P.shells_for(WATER, "cc-pvdz", basis_library())
    ob = oracle.Basis(oracle.shells_for(oracle.Molecule(WATER), "cc-pvdz"))
    eng = P.FockEngine(shells, engine="os")
    nb = eng.nbasis
    Pm = random_density(nb, seed=9)
    eri_o, _ = ob.eri_tensor(1e-10, oracle.OS)
    G_o = oracle.fock_rhf_tensor(eri_o, Pm)
    dP = torch.tensor(Pm, device="cuda:0", dtype=torch.float64)
    dG = torch.zeros_like(dP)
    stream = torch.cuda.Stream()
    for engine in ("os", "rys", "auto", "os"):
        eng.set_options(1e-10, engine)
        dG.fill_(float("nan"))
        torch.cuda.synchronize()
        eng.fock_rhf_device(dP.data_ptr(), dG.data_ptr(), stream.cuda_stream)
        stream.synchronize()
        assert np.abs(dG.cpu().numpy() - G_o).max() < 1e-10
    eng.close()


def test_uhf_and_mixed_precision_on_os_kernels():
    P = pfk()
    mol, shells = P.shells_for(WATER, "6-31g**", basis_library())
    ob = oracle.Basis(oracle.shells_for(oracle.Molecule(WATER), "6-31g**"))
    eng = P.FockEngine(shells, engine="os")
    nb = eng.nbasis
    Pa, Pb = random_density(nb, seed=4), random_density(nb, seed=5)
    eri_o, _ = ob.eri_tensor(1e-10, oracle.OS)
    Ga_o, Gb_o = oracle.fock_uhf_tensor(eri_o, Pa, Pb)
    Ga, Gb = eng.fock_uhf(Pa, Pb)
    assert np.abs(Ga - Ga_o).max() < 1e-10 and np.abs(Gb - Gb_o).max() < 1e-10
    G64 = eng.fock_rhf(Pa)
    eng.set_options(1e-10, "os", "mixed", 1e-8)
    Gmx = eng.fock_rhf(Pa)
    eng.close()
    assert np.abs(Gmx - G64).max() < 1e-7
    assert abs(0.5 * np.sum(Pa * (Gmx - G64))) < 1e-6


def test_autotune_picks_per_class_and_keeps_results(random_basis):
    """pfk_autotune times every candidate per class and keeps the fastest for
    engine auto: classes above L = 4 can only run Rys, the builds before and
    after agree to rounding, and switching engine and back keeps the choice."""
    P = pfk()
    eng = P.FockEngine(random_basis, engine="auto")
    nb = eng.nbasis
    Pm = random_density(nb, seed=12)
    G0 = eng.fock_rhf(Pm)
    res = eng.autotune()
    assert res
    for name, (choice, times) in res.items():
        L = sum("spdf".index(ch) for ch in name if ch in "spdf")
        assert choice in ("rys", "os", "os-dense")
        if L > 4:
            assert choice == "rys" and set(times) == {"rys"}
        else:
            assert set(times) == {"rys", "os", "os-dense"}
            assert times[choice] == min(times.values())
    G1 = eng.fock_rhf(Pm)
    eng.set_options(1e-10, "rys")
    eng.set_options(1e-10, "auto")
    G2 = eng.fock_rhf(Pm)
    eng.close()
    assert np.abs(G1 - G0).max() < 1e-11
    assert np.abs(G2 - G1).max() < 1e-13


def test_lanes_change_only_the_order_of_additions(random_basis):
    """Class kernels spread over 1 to 4 streams (pfk_set_lanes): captured
    device builds and host builds agree to rounding, and an out-of-range
    lane count is refused."""
    P = pfk()
    eng = P.FockEngine(random_basis, engine="auto")
    Pm = random_density(eng.nbasis, seed=21)
    eng.set_lanes(1)
    G1 = eng.fock_rhf(Pm)
    out = []
    for lanes in (4, 2, 3, 4):
        eng.set_lanes(lanes)
        out.append(eng.fock_rhf(Pm))
        out.append(eng.fock_rhf(Pm))   # the second build replays the captured graph
    with pytest.raises(Exception):
        eng.set_lanes(5)
    eng.close()
    for G in out:
        assert np.abs(G - G1).max() < 1e-12 * max(1.0, np.abs(G1).max())


def test_primitive_screening_bound_holds(random_basis):
    """pfk_set_primitive_tol: builds with the default bound (1e-16), with
    every primitive (0) and with 1e-12 agree to within what the skipped
    primitive quartets can add (each below ptol per integral), the default
    build stays within 1e-10 of the oracle, and values outside [0, 1e-10] are
    refused."""
    P = pfk()
    shells = random_basis
    ob = oracle.Basis(shells)
    eri_o, _ = ob.eri_tensor(1e-10, oracle.OS)
    eng = P.FockEngine(shells, engine="os")
    Pm = random_density(eng.nbasis, seed=23)
    G_o = oracle.fock_rhf_tensor(eri_o, Pm)
    G_def = eng.fock_rhf(Pm)
    eng.set_primitive_tol(0.0)
    G_all = eng.fock_rhf(Pm)
    eng.set_primitive_tol(1e-12)
    G_loose = eng.fock_rhf(Pm)
    for bad in (-1.0, 1e-9, float("nan")):
        with pytest.raises(Exception):
            eng.set_primitive_tol(bad)
    eng.close()
    assert np.abs(G_def - G_o).max() < 1e-10
    assert np.abs(G_def - G_all).max() < 1e-11
    assert np.abs(G_loose - G_all).max() < 1e-7
