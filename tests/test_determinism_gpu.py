"""Bitwise reproducibility of the Fock build (GPU tests).

The class kernels add every J/K contribution to fixed-point integer
accumulators (fx_add in csrc/pfk_device.cuh): integer addition is
associative, so a build's result does not depend on the order in which
threads, warps, kernels and launch streams arrive.  The reference's
digestion is a static loop over mu (os.cpp:1512-1520) and is deterministic
too; with FP64 atomics the plain FP64 SCF of C40H82 had taken anywhere from
93 to 165 iterations from one run to the next.  These tests require
bitwise-equal results across repeats, across launch-lane counts, and across
whole SCF runs."""
import numpy as np
import pytest

from helpers import basis_library, pfk, random_density, water_cluster

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cluster():
    P = pfk()
    atoms = water_cluster(8, seed=11)
    mol, shells = P.shells_for(atoms, "6-31g**", basis_library())
    return atoms, shells


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_rhf_build_bitwise_repeatable(cluster, precision):
    _, shells = cluster
    P = pfk()
    eng = P.FockEngine(shells, precision=precision)
    Pm = random_density(eng.nbasis, seed=31, scale=0.1)
    G1 = eng.fock_rhf(Pm)
    G2 = eng.fock_rhf(Pm)
    assert np.array_equal(G1, G2)
    # one launch stream instead of four: another order of arrival
    eng.set_lanes(1)
    G3 = eng.fock_rhf(Pm)
    eng.set_lanes(4)
    assert np.array_equal(G1, G3)
    # a second context on the same basis
    eng2 = P.FockEngine(shells, precision=precision)
    assert np.array_equal(G1, eng2.fock_rhf(Pm))
    eng2.close()
    eng.close()


def test_uhf_and_jk_bitwise_repeatable(cluster):
    _, shells = cluster
    eng = pfk().FockEngine(shells)
    nb = eng.nbasis
    Pa, Pb = random_density(nb, seed=32, scale=0.1), random_density(nb, seed=33, scale=0.1)
    Ga1, Gb1 = eng.fock_uhf(Pa, Pb)
    Ga2, Gb2 = eng.fock_uhf(Pa, Pb)
    assert np.array_equal(Ga1, Ga2) and np.array_equal(Gb1, Gb2)
    J1, K1 = eng.jk(Pa, Pb, k_scale=0.25)
    J2, K2 = eng.jk(Pa, Pb, k_scale=0.25)
    assert np.array_equal(J1, J2) and np.array_equal(K1, K2)
    eng.close()


def test_graph_replay_bitwise_equals_host(cluster):
    torch = pytest.importorskip("torch")
    _, shells = cluster
    eng = pfk().FockEngine(shells)
    Pm = random_density(eng.nbasis, seed=34, scale=0.1)
    G_host = eng.fock_rhf(Pm)
    dP = torch.tensor(Pm, device="cuda:0", dtype=torch.float64)
    dG = torch.zeros_like(dP)
    s = torch.cuda.Stream()
    outs = []
    with torch.cuda.stream(s):
        for _ in range(3):
            eng.fock_rhf_device(dP.data_ptr(), dG.data_ptr(), s.cuda_stream)
            outs.append(dG.clone())
    torch.cuda.synchronize()
    for o in outs:
        assert np.array_equal(o.cpu().numpy(), G_host)
    eng.close()


def test_scf_runs_repeat_exactly():
    """Three RHF runs of the same molecule: equal iteration counts and
    bitwise-equal energies (the SCF iteration count is part of the metric)."""
    P = pfk()
    atoms = water_cluster(4, seed=7)
    lib = basis_library()
    runs = []
    for _ in range(3):
        sysm = P.scf.System(atoms, "6-31g**", lib)
        r = sysm.run()
        sysm.close()
        assert r["converged"]
        runs.append((r["iterations"], r["energy"]))
    assert runs[0] == runs[1] == runs[2], runs
