"""Parity at the sizes the benchmark and the SCF measurements run (GPU tests).

(H2O)32 / 6-31G** (800 functions, the bench's molecule and seed) and
C40H82 / cc-pVDZ (1010 Cartesian functions, the time-to-energy molecule):

* the screened canonical AO quartet set (os.cpp:1458-1476) is identical to
  the oracle's: same count and same 64-bit order-independent digest, over
  2.3e9 and ~1e10 quartets;
* sampled elements of G = J - K/2 agree with the oracle's element-wise
  evaluation from the definition (orc_fock_elements: every integral of the
  element's J and K sums, screened like the reference) within 1e-10.

The full oracle build of these molecules takes minutes to hours on the host,
so G is checked element by element on a seeded sample."""
import numpy as np
import pytest

import oracle
from helpers import basis_library, pfk

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def _systems():
    W = pfk().workloads
    return {"water32": (W.water_cluster(32, seed=2026), "6-31g**"),
            "c40h82": (W.alkane(40, seed=3, noise=0.03), "cc-pvdz")}


@pytest.mark.parametrize("name", ["water32", "c40h82"])
def test_timed_quartet_set_and_sampled_fock(name):
    atoms, basis = _systems()[name]
    P = pfk()
    mol, shells = P.shells_for(atoms, basis, basis_library())
    eng = P.FockEngine(shells)
    ob = oracle.Basis(oracle.shells_for(oracle.Molecule(atoms), basis))
    nb = eng.nbasis
    assert nb == ob.nbasis == (800 if name == "water32" else 1010)
    Qo = ob.schwarz(oracle.OS)
    n_o, dig_o, _ = ob.quartet_list(1e-10, Qo)
    n_g, dig_g, _ = eng.quartet_count()
    assert (n_g, dig_g) == (n_o, dig_o)

    rng = np.random.default_rng(2026)
    A = rng.normal(size=(nb, nb)) * 0.05
    Pm = A + A.T
    G = eng.fock_rhf(Pm)
    eng.close()
    el = rng.integers(0, nb, size=(32, 2))
    g_o = ob.fock_elements(Pm, el, tol=1e-10, engine=oracle.OS, Q=Qo)
    err = np.abs(G[el[:, 0], el[:, 1]] - g_o)
    assert err.max() < 1e-10, err.max()
