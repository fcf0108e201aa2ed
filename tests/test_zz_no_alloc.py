"""The allocation-free RHF build, pfk_fock_rhf_noalloc (GPU).

Some host programs may not allocate GPU memory themselves: their device memory
belongs to another allocator or pool, or their budget is fixed before the SCF
starts.  pfk_fock_rhf_noalloc serves them by taking every buffer it needs from
one static device array inside the library.  These tests call it through the
C ABI on buffers the test owns, twice in a row on the same array (so the second
call runs on whatever the first left behind), and compare each result with the
regular entry point pfk_fock_rhf to the tolerance the other Fock tests use
(1e-10 absolute).  The file is named to run last in a full test session; it
also passes on its own in a fresh process."""
import ctypes

import numpy as np
import pytest

from helpers import WATER, basis_library, pfk, random_density, regression_cases, water_cluster

pytestmark = pytest.mark.gpu


def _desc(P, shells):
    keep = {k: np.ascontiguousarray(v) for k, v in shells.items()}
    keep["L"] = keep["L"].astype(np.int32)
    keep["nprim"] = keep["nprim"].astype(np.int32)
    for k in ("center", "expo", "coef", "norm"):
        keep[k] = keep[k].astype(np.float64)
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    d = P.BasisDesc(len(keep["L"]), ptr(keep["L"]), ptr(keep["nprim"]), ptr(keep["center"]), ptr(keep["expo"]),
                    ptr(keep["coef"]), ptr(keep["norm"]))
    return d, keep


@pytest.mark.parametrize("case", ["water_631gss", "ethylene_ccpvdz"])
def test_noalloc_matches_regular_build_twice(case):
    torch = pytest.importorskip("torch")
    P = pfk()
    lib = P.load_library()
    atoms, basis = (WATER, "6-31g**") if case == "water_631gss" else \
        (regression_cases()["ethylene_rhf_ccpvdz_auto"]["atoms"], "cc-pvdz")
    mol, shells = P.shells_for(atoms, basis, basis_library())
    eng = P.FockEngine(shells)
    nb = eng.nbasis
    desc, keep = _desc(P, shells)
    stream = torch.cuda.Stream()
    for seed in (11, 12):                      # two calls in a row on the shared array
        Pm = random_density(nb, seed=seed)
        G_ref = eng.fock_rhf(Pm)
        dP = torch.tensor(Pm, device="cuda:0", dtype=torch.float64)
        dG = torch.full_like(dP, float("nan"))
        torch.cuda.synchronize()
        st = lib.pfk_fock_rhf_noalloc(ctypes.byref(desc), ctypes.c_void_p(dP.data_ptr()),
                                      ctypes.c_void_p(dG.data_ptr()), 1e-10, ctypes.c_void_p(stream.cuda_stream))
        assert st == P.PFK_OK, lib.pfk_last_error(None).decode()
        G = dG.cpu().numpy()
        assert np.all(np.isfinite(G))
        assert np.abs(G - G_ref).max() < 1e-10
    eng.close()


def test_noalloc_rejects_a_basis_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    P = pfk()
    lib = P.load_library()
    mol, shells = P.shells_for(water_cluster(16, seed=3), "6-31g**", basis_library())
    desc, keep = _desc(P, shells)
    nb = sum((int(l) + 1) * (int(l) + 2) // 2 for l in keep["L"])
    dP = torch.zeros((nb, nb), device="cuda:0", dtype=torch.float64)
    dG = torch.zeros_like(dP)
    st = lib.pfk_fock_rhf_noalloc(ctypes.byref(desc), ctypes.c_void_p(dP.data_ptr()),
                                  ctypes.c_void_p(dG.data_ptr()), 1e-10, None)
    assert st == P.PFK_ERR_UNSUPPORTED
    assert b"limit" in lib.pfk_last_error(None)
