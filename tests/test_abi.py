"""CPU-side checks of the product boundary: the C-ABI library loads and exports
every symbol include/planck_fock.h declares, argument validation needs no GPU,
and the host-side basis construction matches the oracle's."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle
from helpers import REPO, WATER, basis_library, pfk

HEADER = os.path.join(REPO, "include", "planck_fock.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:pfk_status|int|long long|const char \*)\s*(pfk_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = pfk().load_library()
    syms = declared_symbols()
    assert len(syms) >= 14
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(pfk().EXPORTS)


def test_library_has_sm100a_code():
    so = pfk().LIB_PATH
    r = os.popen(f"/usr/local/cuda/bin/cuobjdump --list-elf {so} 2>/dev/null").read()
    assert "sm_100a" in r


def _desc(shells):
    P = pfk()
    s = {k: np.ascontiguousarray(v) for k, v in shells.items()}
    s["L"] = s["L"].astype(np.int32)
    s["nprim"] = s["nprim"].astype(np.int32)
    d = P.BasisDesc(len(s["L"]), *(a.ctypes.data_as(ctypes.c_void_p) for a in
                                   (s["L"], s["nprim"], s["center"], s["expo"], s["coef"], s["norm"])))
    return d, s


def test_create_rejects_bad_input_without_touching_the_gpu():
    P = pfk()
    lib = P.load_library()
    mol, shells = P.shells_for(WATER, "6-31g**", basis_library())
    h = ctypes.c_void_p()
    # null descriptor
    assert lib.pfk_create(None, 0, ctypes.byref(h)) == P.PFK_ERR_INVALID
    assert b"null" in lib.pfk_last_error(None)
    # g functions
    bad = dict(shells)
    bad["L"] = shells["L"].copy()
    bad["L"][0] = 4
    d, keep = _desc(bad)
    assert lib.pfk_create(ctypes.byref(d), 0, ctypes.byref(h)) == P.PFK_ERR_UNSUPPORTED
    # negative exponent
    bad = dict(shells)
    bad["expo"] = shells["expo"].copy()
    bad["expo"][3] = -1.0
    d, keep = _desc(bad)
    assert lib.pfk_create(ctypes.byref(d), 0, ctypes.byref(h)) == P.PFK_ERR_INVALID
    # NaN centre
    bad = dict(shells)
    bad["center"] = shells["center"].copy()
    bad["center"][1, 1] = np.nan
    d, keep = _desc(bad)
    assert lib.pfk_create(ctypes.byref(d), 0, ctypes.byref(h)) == P.PFK_ERR_INVALID
    # calls on a null context
    assert lib.pfk_fock_rhf(None, None, None) == P.PFK_ERR_STATE


def test_symmetry_ops_rejected_like_the_boundary_says():
    P = pfk()

    class Dummy:
        nbasis = 25
        tol_eri = 1e-10
        engine = "os"

    with pytest.raises(P.PfkError):
        P._compute_2e_fock(Dummy(), np.zeros((25, 25)), 25, "os", 1e-10, sym_ops=[1, 2])


@pytest.mark.parametrize("basis", ["sto-3g", "6-31g**", "cc-pvdz"])
def test_host_basis_matches_oracle(basis):
    P = pfk()
    mol, shells = P.shells_for(WATER, basis, basis_library())
    omol = oracle.Molecule(WATER)
    oshells = oracle.shells_for(omol, basis)
    for k in ("L", "nprim", "center", "expo"):
        assert np.array_equal(shells[k], oshells[k])
    np.testing.assert_allclose(shells["coef"], oshells["coef"], rtol=1e-15, atol=0)
    np.testing.assert_allclose(shells["norm"], oshells["norm"], rtol=1e-15, atol=0)
    assert sum((l + 1) * (l + 2) // 2 for l in shells["L"]) == {"sto-3g": 7, "6-31g**": 25, "cc-pvdz": 25}[basis]


def test_cartesian_order_and_norms_match_oracle():
    P = pfk()
    mol, shells = P.shells_for(WATER, "cc-pvdz", basis_library())
    b = oracle.Basis(oracle.shells_for(oracle.Molecule(WATER), "cc-pvdz"))
    shell, lxyz, cn = b.ao_info()
    k = 0
    for s, l in enumerate(shells["L"]):
        for (lx, ly, lz) in P.cartesian_order(int(l)):
            assert shell[k] == s and tuple(lxyz[k]) == (lx, ly, lz)
            assert abs(cn[k] - P.component_norm(lx, ly, lz)) < 1e-16
            k += 1


def _table():
    path = os.path.join(REPO, "planck-refactored_b200", "csrc", "rys_table_data.inc")
    text = open(path).read()
    body = text[text.index("kRysCheb[PFK_RYS_TABLE_SIZE] = {") + 32:]
    body = body[:body.index("};")]
    vals = [float(v) for v in re.findall(r"[-+0-9.eE]+(?=,)", re.sub(r"//[^\n]*", "", body))]
    off = [int(v) for v in re.search(r"kRysOffset\[PFK_RYS_NMAX \+ 1\] = \{([^}]*)\}", text).group(1).split(",")]
    tmax = [float(v) for v in re.search(r"kRysTmax\[PFK_RYS_NMAX \+ 1\] = \{([^}]*)\}", text).group(1).split(",")]
    def rows(name):
        m = re.search(name + r"\[PFK_RYS_NMAX \+ 1\]\[PFK_RYS_NMAX\] = \{\{0\},(.*?)\};", text, re.S)
        return [[float(x) for x in r.split(",") if x.strip()] for r in re.findall(r"\{([^}]*)\}", m.group(1))]
    return np.array(vals), off, tmax, rows("kRysAsymU"), rows("kRysAsymW")


def _cheb(c, x):
    b1 = b2 = 0.0
    for k in range(len(c) - 1, 0, -1):
        b1, b2 = c[k] + 2 * x * b1 - b2, b1
    return c[0] + x * b1 - b2


def _boys_exact(k, T):
    import mpmath
    mpmath.mp.dps = 30
    if T == 0:
        return 1.0 / (2 * k + 1)
    return float(mpmath.hyp1f1(k + 0.5, k + 1.5, -T) / (2 * k + 1))


def test_device_rys_table_reproduces_boys_moments():
    """The product's Rys table (evaluated as the device does) integrates the
    Boys moments F_k(T), k < 2n, to rounding (checked against 30-digit
    mpmath; the reference's own Boys table + 6-term Taylor is only good to
    ~1.3e-12 near the end of each 0.1-wide interval), and agrees with the
    oracle's long-double moment construction where that is well conditioned."""
    cheb, off, tmax, au, aw = _table()
    rng = np.random.default_rng(2)
    for n in range(1, 8):
        for T in list(rng.uniform(0, tmax[n], 12)) + [0.0, tmax[n] - 1e-9, tmax[n], 150.0, 2e4]:
            if T < tmax[n]:
                iv = int(T / 2.0)
                x = (T - iv * 2.0) - 1.0
                nint = int(round(tmax[n] / 2.0))
                # layout [k][root][interval][u, w]
                idx = lambda k, r: off[n] + 2 * ((k * n + r) * nint + iv)
                u = np.array([_cheb([cheb[idx(k, r)] for k in range(15)], x) for r in range(n)])
                w = np.array([_cheb([cheb[idx(k, r) + 1] for k in range(15)], x) for r in range(n)])
            else:
                u = np.array(au[n - 1]) / T
                w = np.array(aw[n - 1]) / np.sqrt(T)
            for k in range(2 * n):
                fk = _boys_exact(k, T)
                assert abs(np.sum(w * u ** k) - fk) <= 4e-16 * n * fk + 1e-300, (n, T, k)
            if n <= 3 and T < 30:
                uo, wo = oracle.rys_roots(n, T)
                np.testing.assert_allclose(u, uo, rtol=1e-12, atol=1e-15)
                np.testing.assert_allclose(w, wo, rtol=1e-12, atol=1e-15)


@pytest.mark.gpu
def test_contexts_do_not_leak_device_memory():
    """Building the screened lists allocates temporaries; 200 create/destroy
    cycles must leave the device's free memory where it was (within 8 MiB)."""
    torch = pytest.importorskip("torch")
    P = pfk()
    mol, shells = P.shells_for(WATER, "6-31g**", basis_library())
    for _ in range(5):
        P.FockEngine(shells).close()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(200):
        eng = P.FockEngine(shells)
        eng.set_options(1e-9, "os")       # a second list build
        eng.close()
    torch.cuda.synchronize()
    assert free0 - torch.cuda.mem_get_info()[0] < 8 << 20


def test_header_compiles_and_links_as_c(tmp_path):
    """A C99 caller (-pedantic -Werror) includes include/planck_fock.h, takes
    the address of every function it declares, links against the library and
    runs its argument checks: the header is plain C and every declaration
    resolves to the library's symbol of the same name."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    syms = declared_symbols()
    src = tmp_path / "abi_check.c"
    src.write_text(
        '#include <stdio.h>\n#include <string.h>\n#include "planck_fock.h"\n'
        "typedef void (*fn)(void);\n"
        "int main(void) {\n"
        "    volatile fn all[] = {" + ", ".join(f"(fn){s}" for s in syms) + "};\n"
        "    pfk_ctx *ctx = NULL;\n"
        "    size_t i;\n"
        "    for (i = 0; i < sizeof all / sizeof all[0]; ++i)\n"
        "        if (!all[i]) return 2;\n"
        "    if (pfk_create(NULL, 0, &ctx) != PFK_ERR_INVALID || ctx != NULL) return 3;\n"
        "    if (strlen(pfk_last_error(NULL)) == 0) return 4;\n"
        "    puts(pfk_last_error(NULL));\n"
        "    return 0;\n}\n")
    lib_dir = os.path.dirname(pfk().LIB_PATH)
    exe = tmp_path / "abi_check"
    r = subprocess.run(["gcc", "-std=c99", "-pedantic", "-Wall", "-Werror", "-I",
                        os.path.join(REPO, "include"), str(src), "-L", lib_dir, "-lplanck_fock",
                        "-Wl,-rpath," + lib_dir, "-Wl,-rpath-link,/usr/local/cuda/lib64", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    env = dict(os.environ, LD_LIBRARY_PATH=":".join(filter(None, ["/usr/local/cuda/lib64",
                                                                  os.environ.get("LD_LIBRARY_PATH", "")])))
    r = subprocess.run([str(exe)], capture_output=True, text=True, env=env)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert "null" in r.stdout
