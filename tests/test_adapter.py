"""The C++ adapter (include/planck_fock_adapter.hpp) compiles against
Planck-shaped types and behaves like the reference's entry points
(base.h:39-93): tests/adapter_check.cpp is built with g++ against the
header and the library, with stand-ins for HartreeFock::Shell / Basis /
IntegralMethod and an Eigen-like matrix.

CPU: the shell data reach the C ABI in its layout, g shells and bad
exponents are rejected before the device is touched, and without a GPU a
context fails with PFK_ERR_CUDA instead of falling back to anything.
GPU: G through the adapter (OS and Rys, tol_eri passed through), the UHF
pair, and J/K equal the Python binding's results bitwise, and two symmetry
operations or a wrong nbasis are rejected."""
import os
import subprocess

import numpy as np
import pytest

from helpers import REPO, WATER, basis_library, pfk, random_density


def _build(tmp_path):
    lib_dir = os.path.dirname(pfk().LIB_PATH)
    exe = str(tmp_path / "adapter_check")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-I", os.path.join(REPO, "include"),
           os.path.join(REPO, "tests", "adapter_check.cpp"), "-L", lib_dir, "-lplanck_fock",
           f"-Wl,-rpath,{lib_dir}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _basis_file(tmp_path, shells):
    path = str(tmp_path / "basis.txt")
    L, nprim, center = shells["L"], shells["nprim"], shells["center"]
    expo, coef, norm = shells["expo"], shells["coef"], shells["norm"]
    off = 0
    with open(path, "w") as f:
        f.write(f"{len(L)}\n")
        for s in range(len(L)):
            c = center[s] if np.ndim(center) == 2 else center[3 * s:3 * s + 3]
            f.write(f"{int(L[s])} {int(nprim[s])} {float(c[0])!r} {float(c[1])!r} {float(c[2])!r}\n")
            for i in range(off, off + int(nprim[s])):
                f.write(f"{float(expo[i])!r} {float(coef[i])!r} {float(norm[i])!r}\n")
            off += int(nprim[s])
    return path


def _gpu_visible():
    try:
        import torch
        return torch.cuda.is_available()
    except ImportError:
        return False


def test_adapter_compiles_and_validates(tmp_path):
    P = pfk()
    P.load_library()
    mol, shells = P.shells_for(WATER, "6-31g**", basis_library())
    exe = _build(tmp_path)
    args = [exe, "cpu", _basis_file(tmp_path, shells)] + ([] if _gpu_visible() else ["nogpu"])
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ok shell_data nshell=12 nprim=" in r.stdout and "nbasis=25" in r.stdout
    assert "ok rejects_g_shell" in r.stdout and "ok rejects_bad_exponent" in r.stdout
    if not _gpu_visible():
        assert "ok no_gpu_fails_loudly" in r.stdout


@pytest.mark.gpu
def test_adapter_builds_match_python_binding(tmp_path):
    P = pfk()
    mol, shells = P.shells_for(WATER, "6-31g**", basis_library())
    exe = _build(tmp_path)
    eng = P.FockEngine(shells)
    nb = eng.nbasis
    Pm = random_density(nb, seed=51, scale=0.2)
    pfile, ofile = str(tmp_path / "P.bin"), str(tmp_path / "out.bin")
    Pm.astype(np.float64).tofile(pfile)
    r = subprocess.run([exe, "gpu", _basis_file(tmp_path, shells), pfile, ofile], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ok rejects_sym_ops_and_nbasis" in r.stdout
    G_os, G_rys, Ga, Gb, J, K, G_loose = np.fromfile(ofile).reshape(7, nb, nb)
    assert np.array_equal(G_os, eng.fock_rhf(Pm))
    Ga_p, Gb_p = eng.fock_uhf(Pm, Pm)
    assert np.array_equal(Ga, Ga_p) and np.array_equal(Gb, Gb_p)
    J_p, K_p = eng.jk(Pm, Pm, k_scale=-0.25)
    assert np.array_equal(J, J_p) and np.array_equal(K, K_p)
    eng.set_options(1e-10, "rys")
    assert np.array_equal(G_rys, eng.fock_rhf(Pm))
    n_tight = eng.quartet_count()[0]
    eng.set_options(1e-3, "os")
    assert eng.quartet_count()[0] < n_tight          # tol_eri 1e-3 drops quartets on water
    assert np.array_equal(G_loose, eng.fock_rhf(Pm))
    assert np.abs(G_loose - G_os).max() > 0.0
    eng.close()
