"""CPU oracle for the direct-SCF Fock build -- TEST INFRASTRUCTURE ONLY.

This package restates the reference's algorithm on the CPU (oracle.c, built
into liboracle.so with gcc + OpenMP) and drives it from Python.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline / reference arm may import
it, and only to compare against: the product path never routes through it.

Pinned against (tests/test_oracle.py):
  * the reference's own Boys function (src/lookup/boys.cpp compiled unmodified,
    tests/golden/boys_ref.json);
  * the reference's RHF regression energies (tests/regression_cases.json,
    copied with their geometries into tests/golden/regression_cases.json).
"""
import ctypes
import json
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "liboracle.so")
GOLDEN = os.path.join(REPO, "tests", "golden")

OS, RYS, AUTO = 0, 1, 2
ENGINES = {"os": OS, "rys": RYS, "auto": AUTO}
ANGSTROM_TO_BOHR = 1.8897259886          # src/base/tables.h:8
ZNUC = {"H": 1, "He": 2, "C": 6, "N": 7, "O": 8}

_lock = threading.Lock()
_lib = None


def build():
    """Compile liboracle.so (gcc, OpenMP)."""
    src = os.path.join(HERE, "oracle.c")
    subprocess.check_call(["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-Wall",
                           "-Wno-unused-function", src, "-o", LIB_PATH, "-lm"])


def lib():
    global _lib
    with _lock:
        if _lib is None:
            src = os.path.join(HERE, "oracle.c")
            if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
                build()
            L = ctypes.CDLL(LIB_PATH)
            c_int, c_dbl, vp = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
            L.orc_boys_init.restype = None
            L.orc_boys.restype = c_dbl
            L.orc_boys.argtypes = [c_int, c_dbl]
            L.orc_normalize_shell.argtypes = [c_int, c_int, vp, vp, vp, vp]
            L.orc_basis_create.restype = vp
            L.orc_basis_create.argtypes = [c_int, vp, vp, vp, vp, vp, vp]
            L.orc_basis_destroy.argtypes = [vp]
            L.orc_nbasis.argtypes = [vp]
            L.orc_npairs.argtypes = [vp]
            L.orc_ao_info.argtypes = [vp, vp, vp, vp]
            L.orc_rys_roots.argtypes = [c_int, c_dbl, vp, vp]
            L.orc_eri_pair.restype = c_dbl
            L.orc_eri_pair.argtypes = [vp, c_int, c_int, c_int]
            L.orc_schwarz.argtypes = [vp, c_int, vp]
            L.orc_eri_tensor.restype = ctypes.c_longlong
            L.orc_eri_tensor.argtypes = [vp, c_dbl, c_int, vp, vp]
            L.orc_fock_rhf_from_tensor.argtypes = [ctypes.c_size_t, vp, vp, vp]
            L.orc_fock_uhf_from_tensor.argtypes = [ctypes.c_size_t, vp, vp, vp, vp, vp]
            L.orc_shell_block.restype = None
            L.orc_shell_block.argtypes = [vp, c_int, c_int, c_int, c_int, c_int, vp]
            L.orc_fock_elements.restype = None
            L.orc_fock_elements.argtypes = [vp, c_dbl, c_int, vp, vp, vp, c_int, vp]
            L.orc_jk_direct.restype = ctypes.c_longlong
            L.orc_jk_direct.argtypes = [vp, c_dbl, c_int, vp, c_int, vp, vp, vp, vp, c_int, c_int]
            L.orc_jk_direct_rows.restype = ctypes.c_longlong
            L.orc_jk_direct_rows.argtypes = [vp, c_dbl, c_int, vp, c_int, vp, vp, vp, vp, vp, c_int]
            L.orc_row_count.restype = ctypes.c_longlong
            L.orc_row_count.argtypes = [vp, c_dbl, vp, c_int]
            L.orc_quartet_list.restype = ctypes.c_longlong
            L.orc_quartet_list.argtypes = [vp, c_dbl, vp, vp, vp, ctypes.c_longlong]
            L.orc_one_electron.argtypes = [vp, c_int, vp, vp, vp, vp]
            L.orc_num_threads.restype = c_int
            L.orc_boys_init()
            _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def boys(n, x):
    return lib().orc_boys(int(n), float(x))


def rys_roots(n, T):
    r = np.zeros(n)
    w = np.zeros(n)
    lib().orc_rys_roots(n, float(T), _p(r), _p(w))
    return r, w


def load_basis_library():
    with open(os.path.join(REPO, "planck-refactored_b200", "data", "basis_sets.json")) as f:
        return json.load(f)["basis"]


def normalize_shell(L, expo, raw):
    expo = np.ascontiguousarray(expo, dtype=np.float64)
    raw = np.ascontiguousarray(raw, dtype=np.float64)
    coef = np.zeros_like(raw)
    norm = np.zeros_like(raw)
    lib().orc_normalize_shell(int(L), len(expo), _p(expo), _p(raw), _p(coef), _p(norm))
    return coef, norm


class Molecule:
    """Atoms in Bohr (converted from Angstrom with the reference's constant)."""

    def __init__(self, atoms, charge=0, units="angstrom"):
        self.symbols = [a[0] for a in atoms]
        xyz = np.array([[a[1], a[2], a[3]] for a in atoms], dtype=np.float64)
        self.coords = xyz * ANGSTROM_TO_BOHR if units == "angstrom" else xyz
        self.Z = np.array([ZNUC[s] for s in self.symbols], dtype=np.float64)
        self.charge = charge

    def nuclear_repulsion(self):
        """types.h:934-964"""
        e = 0.0
        n = len(self.Z)
        for a in range(n):
            for b in range(a + 1, n):
                d = self.coords[a] - self.coords[b]
                e += self.Z[a] * self.Z[b] / np.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
        return e

    def nelectron(self):
        return int(self.Z.sum()) - self.charge


def shells_for(mol, basis_name, library=None):
    """Shell arrays in the reference's order (gaussian.cpp:230-298): atoms in
    input order, shells in file order, coefficients Nc-folded, primitive
    norms per primitive.  Returns dict of numpy arrays."""
    library = library or load_basis_library()
    data = library[basis_name]
    L, nprim, center, expo, coef, norm = [], [], [], [], [], []
    for sym, xyz in zip(mol.symbols, mol.coords):
        for l, prims in data[sym]:
            e = np.array([p[0] for p in prims])
            c_raw = np.array([p[1] for p in prims])
            c, nrm = normalize_shell(l, e, c_raw)
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


class Basis:
    """Owns an orc_basis (AO pairs with primitive-pair data)."""

    def __init__(self, shells):
        self.shells = {k: np.ascontiguousarray(v) for k, v in shells.items()}
        s = self.shells
        self.h = lib().orc_basis_create(len(s["L"]), _p(s["L"]), _p(s["nprim"]), _p(s["center"]),
                                        _p(s["expo"]), _p(s["coef"]), _p(s["norm"]))
        self.nbasis = lib().orc_nbasis(self.h)
        self.npairs = lib().orc_npairs(self.h)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_basis_destroy(self.h)
            self.h = None

    def ao_info(self):
        nb = self.nbasis
        shell = np.zeros(nb, dtype=np.int32)
        lxyz = np.zeros((nb, 3), dtype=np.int32)
        cn = np.zeros(nb)
        lib().orc_ao_info(self.h, _p(shell), _p(lxyz), _p(cn))
        return shell, lxyz, cn

    def schwarz(self, engine=OS):
        Q = np.zeros((self.nbasis, self.nbasis))
        lib().orc_schwarz(self.h, engine, _p(Q))
        return Q

    def eri_tensor(self, tol=1e-10, engine=OS, Q=None):
        if Q is None:
            Q = self.schwarz(engine)
        nb = self.nbasis
        eri = np.zeros((nb, nb, nb, nb))
        n = lib().orc_eri_tensor(self.h, tol, engine, _p(Q), _p(eri))
        return eri, n

    def quartet_list(self, tol, Q, want_list=False):
        import ctypes as ct
        digest = ct.c_uint64(0)
        if want_list:
            cnt = lib().orc_quartet_list(self.h, tol, _p(Q), ct.byref(digest), None, 0)
            out = np.zeros((cnt, 4), dtype=np.int32)
            lib().orc_quartet_list(self.h, tol, _p(Q), ct.byref(digest), _p(out), cnt)
            return cnt, digest.value, out
        cnt = lib().orc_quartet_list(self.h, tol, _p(Q), ct.byref(digest), None, 0)
        return cnt, digest.value, None

    def jk_direct(self, Pj, Pk_list, tol=1e-10, engine=OS, Q=None, pair_range=(0, -1)):
        """Streaming J(Pj) and K(Pk) for each Pk (no nb^4 tensor)."""
        if Q is None:
            Q = self.schwarz(engine)
        nb = self.nbasis
        Pj = np.ascontiguousarray(Pj, dtype=np.float64)
        Pk = np.ascontiguousarray(np.stack(Pk_list), dtype=np.float64)
        J = np.zeros((nb, nb))
        K = np.zeros((len(Pk_list), nb, nb))
        n = lib().orc_jk_direct(self.h, tol, engine, _p(Q), len(Pk_list), _p(Pj), _p(Pk),
                                _p(J), _p(K), pair_range[0], pair_range[1])
        return J, K, n

    def jk_direct_rows(self, Pj, Pk_list, rows, tol=1e-10, engine=OS, Q=None):
        """Streaming J/K restricted to the given bra AO-pair rows."""
        if Q is None:
            Q = self.schwarz(engine)
        nb = self.nbasis
        Pj = np.ascontiguousarray(Pj, dtype=np.float64)
        Pk = np.ascontiguousarray(np.stack(Pk_list), dtype=np.float64)
        rows = np.ascontiguousarray(rows, dtype=np.int32)
        J = np.zeros((nb, nb))
        K = np.zeros((len(Pk_list), nb, nb))
        n = lib().orc_jk_direct_rows(self.h, tol, engine, _p(Q), len(Pk_list), _p(Pj), _p(Pk),
                                     _p(J), _p(K), _p(rows), len(rows))
        return J, K, n

    def shell_block(self, sa, sb, sc, sd, engine=OS):
        """Cartesian block (sa sb|sc sd), components ((ia*NB+ib)*NC+ic)*ND+id."""
        L = self.shells["L"]
        n = [(int(L[x]) + 1) * (int(L[x]) + 2) // 2 for x in (sa, sb, sc, sd)]
        out = np.zeros(n[0] * n[1] * n[2] * n[3])
        lib().orc_shell_block(self.h, int(sa), int(sb), int(sc), int(sd), engine, _p(out))
        return out

    def fock_elements(self, P, elems, tol=1e-10, engine=OS, Q=None):
        """G(m, n) = J - K/2 of the RHF build for the (m, n) pairs in elems,
        from the definition (O(nb^2) integrals per element)."""
        if Q is None:
            Q = self.schwarz(engine)
        P = np.ascontiguousarray(P, dtype=np.float64)
        el = np.ascontiguousarray(np.asarray(elems, dtype=np.int32).reshape(-1, 2))
        out = np.zeros(len(el))
        lib().orc_fock_elements(self.h, tol, engine, _p(Q), _p(P), _p(el), len(el), _p(out))
        return out

    def row_count(self, p, tol, Q):
        return lib().orc_row_count(self.h, tol, _p(Q), int(p))

    def eri_pair(self, p, q, engine=OS):
        return lib().orc_eri_pair(self.h, p, q, engine)

    def one_electron(self, mol):
        nb = self.nbasis
        S = np.zeros((nb, nb))
        T = np.zeros((nb, nb))
        V = np.zeros((nb, nb))
        ch = np.ascontiguousarray(np.hstack([mol.coords, mol.Z[:, None]]))
        lib().orc_one_electron(self.h, len(mol.Z), _p(ch), _p(S), _p(T), _p(V))
        return S, T, V


def fock_rhf_tensor(eri, P):
    nb = P.shape[0]
    G = np.zeros((nb, nb))
    lib().orc_fock_rhf_from_tensor(nb, _p(eri), _p(np.ascontiguousarray(P)), _p(G))
    return G


def fock_uhf_tensor(eri, Pa, Pb):
    nb = Pa.shape[0]
    Ga = np.zeros((nb, nb))
    Gb = np.zeros((nb, nb))
    lib().orc_fock_uhf_from_tensor(nb, _p(eri), _p(np.ascontiguousarray(Pa)),
                                   _p(np.ascontiguousarray(Pb)), _p(Ga), _p(Gb))
    return Ga, Gb


# ---------------------------------------------------------------------------
# SCF (restates src/scf/scf.cpp:15-45 orthogonaliser + hcore guess,
# :89-135 metrics/convergence, :175-441 RHF loop; DIIS src/base/types.h:759-837)
# ---------------------------------------------------------------------------
def _colpiv_qr_solve(A, b):
    """Least-squares solve by column-pivoted Householder QR with the rank
    cut-off Eigen's ColPivHouseholderQR uses (|R_kk| > n * eps * |R_00|),
    as the reference's DIIS does (types.h:813)."""
    import scipy.linalg as sl
    Q, R, piv = sl.qr(A, pivoting=True)
    d = np.abs(np.diag(R))
    rank = int((d > np.finfo(float).eps * len(d) * d[0]).sum())
    y = Q.T @ b
    z = np.zeros(A.shape[1])
    if rank:
        z[:rank] = sl.solve_triangular(R[:rank, :rank], y[:rank])
    x = np.zeros(A.shape[1])
    x[piv] = z
    return x


class DIIS:
    def __init__(self, max_vecs=8):
        self.F, self.E, self.max_vecs = [], [], max_vecs

    def push(self, F, e):
        self.F.append(F.copy())
        self.E.append(e.copy())
        if len(self.F) > self.max_vecs:
            self.F.pop(0)
            self.E.pop(0)

    def ready(self):
        return len(self.F) >= 2

    def extrapolate(self):
        m = len(self.F)
        B = np.zeros((m + 1, m + 1))
        for i in range(m):
            for j in range(i, m):
                B[i, j] = B[j, i] = float((self.E[i] * self.E[j]).sum())
            B[i, m] = B[m, i] = -1.0
        rhs = np.zeros(m + 1)
        rhs[m] = -1.0
        c = _colpiv_qr_solve(B, rhs)
        return sum(c[i] * self.F[i] for i in range(m))

    def error_norm(self):
        e = self.E[-1]
        return float(np.sqrt((e * e).sum() / e.size))


def orthogonalizer(S):
    s, U = np.linalg.eigh(S)
    return U @ np.diag(1.0 / np.sqrt(s)) @ U.T


def hcore_guess(H, X, nocc):
    _, Cp = np.linalg.eigh(X.T @ H @ X)
    C = X @ Cp
    Co = C[:, :nocc]
    return 2.0 * Co @ Co.T


def max_cycles_for(nb):
    """types.h:356-363"""
    return 300 if nb > 1000 else 200 if nb > 500 else 100 if nb > 250 else 50


def rhf(H, S, enuc, nocc, fock_builder, P0=None, max_iter=None, tol_e=1e-10, tol_d=1e-10,
        diis_dim=8, callback=None):
    """Run the reference's RHF loop.  fock_builder(P) -> G = J - K/2.
    Returns dict(energy, iterations, converged, P, F, eps, C, history)."""
    nb = H.shape[0]
    X = orthogonalizer(S)
    P = hcore_guess(H, X, nocc) if P0 is None else P0.copy()
    max_iter = max_iter or max_cycles_for(nb)
    diis = DIIS(diis_dim)
    E_prev = 0.0
    hist = []
    for it in range(1, max_iter + 1):
        G = fock_builder(P)
        F = H + G
        E = 0.5 * float((P * (H + F)).sum()) + enuc
        e = X.T @ (F @ P @ S - S @ P @ F) @ X
        diis.push(F, e)
        Fd = diis.extrapolate() if diis.ready() else F
        eps, Cp = np.linalg.eigh(X.T @ Fd @ X)
        C = X @ Cp
        Co = C[:, :nocc]
        Pn = 2.0 * Co @ Co.T
        dP = Pn - P
        dE = abs(E - E_prev)
        dmax = float(np.abs(dP).max())
        drms = float(np.sqrt((dP * dP).sum() / dP.size))
        hist.append((it, E, dE, drms, dmax))
        if callback:
            callback(it, E, P)
        P = Pn
        E_prev = E
        if it > 1 and dE < tol_e and drms < tol_d and dmax < tol_d:
            return {"energy": E, "iterations": it, "converged": True, "P": P, "F": F,
                    "eps": eps, "C": C, "history": hist}
    return {"energy": E_prev, "iterations": max_iter, "converged": False, "P": P, "F": F,
            "eps": eps, "C": C, "history": hist}


def setup(atoms, basis_name, charge=0, units="angstrom"):
    mol = Molecule(atoms, charge=charge, units=units)
    shells = shells_for(mol, basis_name)
    bas = Basis(shells)
    S, T, V = bas.one_electron(mol)
    return mol, shells, bas, S, T + V


def rhf_conventional(atoms, basis_name, engine=OS, tol_eri=1e-10, charge=0, max_iter=None):
    """Conventional RHF as the reference's default scf_mode does (scf.cpp:248-264)."""
    mol, shells, bas, S, H = setup(atoms, basis_name, charge)
    eri, _ = bas.eri_tensor(tol_eri, engine)
    res = rhf(H, S, mol.nuclear_repulsion(), mol.nelectron() // 2,
              lambda P: fock_rhf_tensor(eri, P), max_iter=max_iter)
    res.update(mol=mol, shells=shells, basis=bas, S=S, H=H)
    return res
