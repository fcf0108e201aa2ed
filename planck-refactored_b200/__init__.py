"""planck-refactored_b200: B200-native direct-SCF Fock build for Planck.

Python host mirror of the reference's two-electron interface
(src/integrals/base.h:39-93) over the C ABI in include/planck_fock.h.
The compute path is the CUDA library libplanck_fock.so built in-tree by
build.py; there is no CPU fallback -- importing works without a GPU, but
every compute call fails loudly if the library or the device is missing.

Typical use (mirrors scf.cpp:281-284):

    eng = FockEngine(shells)                 # once per geometry
    G = _compute_2e_fock(eng, P, nbasis, "os", 1e-10)
"""
import ctypes
import os

import numpy as np

from . import shard, workloads  # noqa: F401
from .basis import (ANGSTROM_TO_BOHR, Molecule, cartesian_order, component_norm,  # noqa: F401
                    read_gbs_basis, shells_for)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libplanck_fock.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include", "planck_fock.h")

PFK_OK, PFK_ERR_INVALID, PFK_ERR_UNSUPPORTED, PFK_ERR_CUDA, PFK_ERR_NOMEM, PFK_ERR_STATE = range(6)
ENGINES = {"os": 0, "rys": 1, "auto": 2}
PRECISIONS = {"fp64": 0, "mixed": 1}
EXPORTS = ["pfk_create", "pfk_destroy", "pfk_set_options", "pfk_nbasis", "pfk_last_error", "pfk_schwarz",
           "pfk_quartet_count", "pfk_quartet_list", "pfk_fock_rhf", "pfk_fock_uhf", "pfk_jk",
           "pfk_fock_rhf_device", "pfk_eri_tensor", "pfk_class_stats", "pfk_set_shard", "pfk_measure_fma_peak",
           "pfk_fock_rhf_noalloc", "pfk_one_electron", "pfk_set_density_screening", "pfk_set_lanes", "pfk_set_primitive_tol", "pfk_autotune", "pfk_mlp_create", "pfk_mlp_destroy", "pfk_mlp_last_error",
           "pfk_mlp_param_count", "pfk_mlp_set_params", "pfk_mlp_get_params", "pfk_mlp_forward", "pfk_mlp_gradients",
           "pfk_mlp_train_step", "pfk_checkpoint_write", "pfk_checkpoint_read_density",
           "pfk_checkpoint_last_error", "pfk_mo_transform",
           "pfk_mo_transform_times", "pfk_rmp2_energy",
           "pfk_ump2_energy", "pfk_eri_batch_create", "pfk_eri_batch_destroy", "pfk_eri_batch_last_error",
           "pfk_eri_batch_set_quartets", "pfk_eri_batch_run", "pfk_precision_stats", "pfk_scf_rhf"]

_lib = None


class PfkError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"pfk status {status}: {msg}")
        self.status = status


class ScfOptions(ctypes.Structure):
    _fields_ = [("max_iter", ctypes.c_int), ("tol_energy", ctypes.c_double), ("tol_density", ctypes.c_double),
                ("diis_depth", ctypes.c_int), ("incremental", ctypes.c_void_p),
                ("incremental_below", ctypes.c_double), ("incremental_floor", ctypes.c_double),
                ("full_every", ctypes.c_int), ("history", ctypes.c_void_p)]


class ScfResult(ctypes.Structure):
    _fields_ = [("energy", ctypes.c_double), ("first_energy", ctypes.c_double), ("iterations", ctypes.c_int),
                ("converged", ctypes.c_int), ("full_builds", ctypes.c_int), ("difference_builds", ctypes.c_int),
                ("build_ms", ctypes.c_double), ("total_ms", ctypes.c_double)]


class BasisDesc(ctypes.Structure):
    _fields_ = [("nshell", ctypes.c_int), ("L", ctypes.c_void_p), ("nprim", ctypes.c_void_p),
                ("center", ctypes.c_void_p), ("expo", ctypes.c_void_p), ("coef", ctypes.c_void_p),
                ("norm", ctypes.c_void_p)]


def load_library(path=LIB_PATH):
    """Load libplanck_fock.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python build.py` (nvcc, sm_100a)")
    L = ctypes.CDLL(path)
    vp, c_int, c_dbl, c_ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_longlong
    for name in EXPORTS:
        getattr(L, name).restype = c_int
    L.pfk_create.argtypes = [ctypes.POINTER(BasisDesc), c_int, ctypes.POINTER(vp)]
    L.pfk_destroy.argtypes = [vp]
    L.pfk_set_options.argtypes = [vp, c_dbl, c_int, c_int, c_dbl]
    L.pfk_nbasis.argtypes = [vp]
    L.pfk_last_error.restype = ctypes.c_char_p
    L.pfk_checkpoint_last_error.restype = ctypes.c_char_p
    L.pfk_checkpoint_last_error.argtypes = []
    L.pfk_last_error.argtypes = [vp]
    L.pfk_schwarz.argtypes = [vp, vp]
    L.pfk_quartet_count.argtypes = [vp, ctypes.POINTER(c_ll), ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(c_ll)]
    L.pfk_quartet_list.argtypes = [vp, vp, c_ll, ctypes.POINTER(c_ll)]
    L.pfk_fock_rhf.argtypes = [vp, vp, vp]
    L.pfk_fock_uhf.argtypes = [vp, vp, vp, vp, vp]
    L.pfk_jk.argtypes = [vp, vp, vp, vp, vp, c_dbl]
    L.pfk_fock_rhf_device.argtypes = [vp, vp, vp, vp]
    L.pfk_eri_tensor.argtypes = [vp, vp]
    L.pfk_class_stats.argtypes = [vp, vp, vp, vp]
    L.pfk_set_shard.argtypes = [vp, c_int, c_int]
    L.pfk_measure_fma_peak.argtypes = [c_int, ctypes.POINTER(c_dbl), ctypes.POINTER(c_dbl)]
    L.pfk_fock_rhf_noalloc.argtypes = [ctypes.POINTER(BasisDesc), vp, vp, c_dbl, vp]
    L.pfk_one_electron.argtypes = [ctypes.POINTER(BasisDesc), c_int, vp, vp, vp, vp, c_int]
    L.pfk_set_density_screening.argtypes = [vp, c_dbl]
    L.pfk_set_lanes.argtypes = [vp, c_int]
    L.pfk_mo_transform.argtypes = [vp, vp, c_int, vp, c_int, vp, c_int, vp, c_int, vp]
    L.pfk_mo_transform_times.argtypes = [vp, vp]
    L.pfk_rmp2_energy.argtypes = [vp, vp, vp, c_int, ctypes.POINTER(c_dbl)]
    L.pfk_ump2_energy.argtypes = [vp, vp, vp, vp, vp, c_int, c_int, ctypes.POINTER(c_dbl)]
    L.pfk_set_primitive_tol.argtypes = [vp, c_dbl]
    L.pfk_autotune.argtypes = [vp, vp, vp]
    L.pfk_precision_stats.argtypes = [vp, vp, vp]
    L.pfk_scf_rhf.argtypes = [vp, vp, vp, c_dbl, c_int, vp, vp, ctypes.POINTER(ScfOptions),
                              ctypes.POINTER(ScfResult), vp, vp, vp]
    L.pfk_eri_batch_create.argtypes = [ctypes.POINTER(BasisDesc), c_int, vp, c_int, ctypes.POINTER(vp)]
    L.pfk_eri_batch_destroy.argtypes = [vp]
    L.pfk_eri_batch_last_error.restype = ctypes.c_char_p
    L.pfk_eri_batch_last_error.argtypes = [vp]
    L.pfk_eri_batch_set_quartets.argtypes = [vp, vp, c_ll, ctypes.POINTER(c_int), ctypes.POINTER(c_int)]
    L.pfk_eri_batch_run.argtypes = [vp, c_ll, c_ll, c_int, c_int, vp, vp]
    _lib = L
    return L


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


CLASS_NAMES = []
for _x in range(10):
    for _y in range(_x + 1):
        _pc = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2), (3, 0), (3, 1), (3, 2), (3, 3)]
        _s = "spdf"
        CLASS_NAMES.append(f"({_s[_pc[_x][0]]}{_s[_pc[_x][1]]}|{_s[_pc[_y][0]]}{_s[_pc[_y][1]]})")


class FockEngine:
    """One molecule/basis on one GPU: owns a pfk_ctx (device data, screened
    quartet lists, captured graphs)."""

    def __init__(self, shells, device=0, tol_eri=1e-10, engine="os", precision="fp64", fp32_bound=1e-8):
        self.lib = load_library()
        self._keep = {k: np.ascontiguousarray(v) for k, v in shells.items()}
        s = self._keep
        s["L"] = np.ascontiguousarray(s["L"], dtype=np.int32)
        s["nprim"] = np.ascontiguousarray(s["nprim"], dtype=np.int32)
        for k in ("center", "expo", "coef", "norm"):
            s[k] = _f64(s[k])
        desc = BasisDesc(len(s["L"]), _p(s["L"]), _p(s["nprim"]), _p(s["center"]), _p(s["expo"]),
                         _p(s["coef"]), _p(s["norm"]))
        h = ctypes.c_void_p()
        st = self.lib.pfk_create(ctypes.byref(desc), int(device), ctypes.byref(h))
        if st != PFK_OK:
            raise PfkError(st, self.lib.pfk_last_error(None).decode())
        self.h = h
        self.nbasis = self.lib.pfk_nbasis(h)
        self.device = int(device)
        self.tol_eri, self.engine, self.precision, self.fp32_bound = 1e-10, "os", "fp64", fp32_bound
        self.set_options(tol_eri, engine, precision, fp32_bound)

    def _check(self, st):
        if st != PFK_OK:
            raise PfkError(st, self.lib.pfk_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.pfk_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_options(self, tol_eri=1e-10, engine="os", precision="fp64", fp32_bound=1e-8):
        self._check(self.lib.pfk_set_options(self.h, float(tol_eri), ENGINES[engine], PRECISIONS[precision],
                                             float(fp32_bound)))
        self.tol_eri, self.engine, self.precision, self.fp32_bound = tol_eri, engine, precision, fp32_bound

    def schwarz(self):
        Q = np.zeros((self.nbasis, self.nbasis))
        self._check(self.lib.pfk_schwarz(self.h, _p(Q)))
        return Q

    def quartet_count(self):
        n = ctypes.c_longlong()
        d = ctypes.c_uint64()
        ns = ctypes.c_longlong()
        self._check(self.lib.pfk_quartet_count(self.h, ctypes.byref(n), ctypes.byref(d), ctypes.byref(ns)))
        return n.value, d.value, ns.value

    def quartet_list(self):
        n_ao, _, _ = self.quartet_count()
        out = np.zeros((max(n_ao, 1), 4), dtype=np.int32)
        n = ctypes.c_longlong()
        self._check(self.lib.pfk_quartet_list(self.h, _p(out), n_ao, ctypes.byref(n)))
        return out[:n.value]

    def fock_rhf(self, P, out=None):
        """G = J(P) - K(P)/2 from host buffers (pfk_fock_rhf).  out: an
        optional C-contiguous float64 host array for G (pinned memory makes
        the device-to-host copy a single DMA); a new array otherwise."""
        P = _f64(P)
        if out is None:
            out = np.empty_like(P)   # every element is written
        elif out.dtype != np.float64 or out.shape != P.shape or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a C-contiguous float64 array shaped like P")
        self._check(self.lib.pfk_fock_rhf(self.h, _p(P), _p(out)))
        return out

    def fock_uhf(self, Pa, Pb):
        Pa, Pb = _f64(Pa), _f64(Pb)
        Ga, Gb = np.zeros_like(Pa), np.zeros_like(Pb)
        self._check(self.lib.pfk_fock_uhf(self.h, _p(Pa), _p(Pb), _p(Ga), _p(Gb)))
        return Ga, Gb

    def jk(self, P, Pk=None, k_scale=1.0, want_k=True):
        P = _f64(P)
        Pk = P if Pk is None else _f64(Pk)
        J = np.zeros_like(P)
        K = np.zeros_like(P) if want_k else None
        self._check(self.lib.pfk_jk(self.h, _p(P), _p(Pk), _p(J), _p(K) if want_k else None, float(k_scale)))
        return J, K

    def fock_rhf_device(self, dP_ptr, dG_ptr, stream_ptr=0):
        self._check(self.lib.pfk_fock_rhf_device(self.h, ctypes.c_void_p(dP_ptr), ctypes.c_void_p(dG_ptr),
                                                 ctypes.c_void_p(stream_ptr or None)))

    def eri_tensor(self):
        nb = self.nbasis
        eri = np.zeros((nb, nb, nb, nb))
        self._check(self.lib.pfk_eri_tensor(self.h, _p(eri)))
        return eri

    def mo_transform(self, C1, C2, C3, C4):
        """(C1 C2 | C3 C4) MO integrals, shape (n1, n2, n3, n4), from the
        device-resident AO tensor (pfk_mo_transform; nbasis <= 180).  C_k are
        nbasis x n_k arrays of MO coefficients."""
        Cs = [np.asarray(C, dtype=np.float64).reshape(self.nbasis, -1) for C in (C1, C2, C3, C4)]
        cm = [np.ascontiguousarray(C.T) for C in Cs]   # column-major storage
        n = [C.shape[1] for C in Cs]
        out = np.zeros(n)
        self._check(self.lib.pfk_mo_transform(self.h, _p(cm[0]), n[0], _p(cm[1]), n[1], _p(cm[2]), n[2],
                                              _p(cm[3]), n[3], _p(out)))
        return out

    def rmp2_energy(self, C, eps, nocc):
        """RMP2 correlation energy with the (ov|ov) block kept on the device
        (pfk_rmp2_energy).  C: nbasis x nbasis MO coefficients, occupied first."""
        cm = np.ascontiguousarray(np.asarray(C, dtype=np.float64).T)   # column-major storage
        e = _f64(np.asarray(eps, dtype=np.float64).reshape(-1))
        out = ctypes.c_double(0.0)
        self._check(self.lib.pfk_rmp2_energy(self.h, _p(cm), _p(e), int(nocc), ctypes.byref(out)))
        return out.value

    def ump2_energy(self, Ca, eps_a, Cb, eps_b, n_alpha, n_beta):
        """UMP2 correlation energy with the three (ov|ov) blocks kept on the
        device (pfk_ump2_energy).  Ca, Cb: MO coefficients, occupied first."""
        ca = np.ascontiguousarray(np.asarray(Ca, dtype=np.float64).T)
        cb = np.ascontiguousarray(np.asarray(Cb, dtype=np.float64).T)
        ea = _f64(np.asarray(eps_a, dtype=np.float64).reshape(-1))
        eb = _f64(np.asarray(eps_b, dtype=np.float64).reshape(-1))
        out = ctypes.c_double(0.0)
        self._check(self.lib.pfk_ump2_energy(self.h, _p(ca), _p(ea), _p(cb), _p(eb), int(n_alpha), int(n_beta),
                                             ctypes.byref(out)))
        return out.value

    def mo_transform_times(self):
        """(AO tensor, quarter-transform GEMMs, copy-out) device ms of the last mo_transform."""
        t = np.zeros(3)
        self._check(self.lib.pfk_mo_transform_times(self.h, _p(t)))
        return tuple(float(x) for x in t)

    def class_stats(self, timed=True):
        """{class name: (shell quartets, primitive quartets, ms)} for non-empty classes."""
        q = np.zeros(55, dtype=np.int64)
        k = np.zeros(55, dtype=np.int64)
        ms = np.zeros(55)
        self._check(self.lib.pfk_class_stats(self.h, _p(q), _p(k), _p(ms) if timed else None))
        return {CLASS_NAMES[c]: (int(q[c]), int(k[c]), float(ms[c])) for c in range(55) if q[c]}

    def precision_stats(self):
        """{class name: (FP32 shell quartets, FP32 primitive quartets)} for the
        classes with a non-empty FP32 list (mixed precision)."""
        q = np.zeros(55, dtype=np.int64)
        k = np.zeros(55, dtype=np.int64)
        self._check(self.lib.pfk_precision_stats(self.h, _p(q), _p(k)))
        return {CLASS_NAMES[c]: (int(q[c]), int(k[c])) for c in range(55) if q[c]}

    def set_shard(self, rank, nranks):
        self._check(self.lib.pfk_set_shard(self.h, int(rank), int(nranks)))

    def scf_rhf(self, H, S, enuc, nocc, P0=None, G0=None, max_iter=0, tol_energy=1e-10, tol_density=1e-10,
                diis_depth=8, incremental=None, incremental_below=1e-4, incremental_floor=1e-8, full_every=8):
        """RHF to convergence on the device (pfk_scf_rhf).  incremental: an
        optional second FockEngine for the difference-density builds.
        Returns scf.rhf()'s dict keys (energy, iterations, converged, P, C,
        eps, first_energy) plus the build counts and times."""
        nb = self.nbasis
        H, S = _f64(H), _f64(S)
        P0 = None if P0 is None else _f64(P0)
        G0 = None if G0 is None else _f64(G0)
        mi = int(max_iter or 0) or (300 if nb > 1000 else 200 if nb > 500 else 100 if nb > 250 else 50)
        hist = np.zeros((mi, 6))
        opt = ScfOptions(mi, tol_energy, tol_density, int(diis_depth),
                         incremental.h if incremental is not None else None, incremental_below, incremental_floor,
                         int(full_every), _p(hist))
        res = ScfResult()
        Pout, Cout, eps = np.zeros((nb, nb)), np.zeros((nb, nb)), np.zeros(nb)
        self._check(self.lib.pfk_scf_rhf(self.h, _p(H), _p(S), float(enuc), int(nocc),
                                         None if P0 is None else _p(P0), None if G0 is None else _p(G0),
                                         ctypes.byref(opt), ctypes.byref(res), _p(Pout), _p(Cout), _p(eps)))
        return {"energy": res.energy, "first_energy": res.first_energy, "iterations": res.iterations,
                "converged": bool(res.converged), "P": Pout, "C": Cout.T.copy(), "eps": eps,
                "full_builds": res.full_builds, "difference_builds": res.difference_builds,
                "build_seconds": res.build_ms * 1e-3, "seconds": res.total_ms * 1e-3,
                "history": [tuple(h) for h in hist[:res.iterations]]}

    def autotune(self):
        """Measure the candidate kernels per class (pfk_autotune) and keep the
        fastest for engine auto.  Returns {class: (choice, {candidate: ms})}
        for the classes with work; choice is "rys", "os" or "os-dense"."""
        choice = np.zeros(55, dtype=np.int32)
        ms = np.zeros(55 * 3)
        self._check(self.lib.pfk_autotune(self.h, _p(choice), _p(ms)))
        names = {0: "rys", 2: "os", 6: "os-dense"}
        out = {}
        for c in range(55):
            t = {names[k]: float(ms[3 * c + v]) for v, k in enumerate((0, 2, 6)) if ms[3 * c + v] > 0}
            if t:
                out[CLASS_NAMES[c]] = (names[int(choice[c])], t)
        return out

    def set_primitive_tol(self, ptol):
        """Skip primitive quartets whose Cauchy-Schwarz bound is below ptol
        (default 1e-16; 0 evaluates them all)."""
        self._check(self.lib.pfk_set_primitive_tol(self.h, float(ptol)))

    def set_lanes(self, lanes):
        """Streams the class kernels of a build are spread over (1 to 4)."""
        self._check(self.lib.pfk_set_lanes(self.h, int(lanes)))

    def set_density_screening(self, dtol):
        """Skip shell quartets whose Schwarz bound times the largest density
        block they touch is below dtol (for difference-density builds; 0 off)."""
        self._check(self.lib.pfk_set_density_screening(self.h, float(dtol)))


def _basis_desc(shells):
    """(BasisDesc, arrays it points into) for a shells dict."""
    keep = {k: np.ascontiguousarray(v) for k, v in shells.items()}
    keep["L"] = np.ascontiguousarray(keep["L"], dtype=np.int32)
    keep["nprim"] = np.ascontiguousarray(keep["nprim"], dtype=np.int32)
    for k in ("center", "expo", "coef", "norm"):
        keep[k] = _f64(keep[k])
    desc = BasisDesc(len(keep["L"]), _p(keep["L"]), _p(keep["nprim"]), _p(keep["center"]), _p(keep["expo"]),
                     _p(keep["coef"]), _p(keep["norm"]))
    return desc, keep


class EriBatch:
    """Cartesian blocks of listed shell quartets (pfk_eri_batch_*).

    shells: a shells dict; pairs: (npairs, 2) shell indices with L(first) >=
    L(second); quartets: (n, 2) pair ids, all of one class (bra class >= ket
    class).  run() writes blocks into a device buffer given by pointer."""

    def __init__(self, shells, pairs, quartets, device=0):
        self.lib = load_library()
        desc, keep = _basis_desc(shells)
        pr = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
        self.h = ctypes.c_void_p()
        st = self.lib.pfk_eri_batch_create(ctypes.byref(desc), len(pr), _p(pr), int(device), ctypes.byref(self.h))
        if st != PFK_OK:
            raise PfkError(st, self.lib.pfk_eri_batch_last_error(None).decode())
        q = np.ascontiguousarray(quartets, dtype=np.int32).reshape(-1, 2)
        cls, nc = ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.pfk_eri_batch_set_quartets(self.h, _p(q), len(q), ctypes.byref(cls), ctypes.byref(nc)))
        self.n, self.cls, self.ncomp = len(q), cls.value, nc.value
        self.name = CLASS_NAMES[self.cls]

    def _check(self, st):
        if st != PFK_OK:
            raise PfkError(st, self.lib.pfk_eri_batch_last_error(self.h).decode())

    def run(self, first, count, engine, precision, out_ptr, stream_ptr=0):
        """Blocks of quartets first..first+count-1 into the device buffer at
        out_ptr (count * ncomp doubles); asynchronous on the stream."""
        self._check(self.lib.pfk_eri_batch_run(self.h, int(first), int(count), ENGINES[engine],
                                               PRECISIONS[precision], ctypes.c_void_p(out_ptr),
                                               ctypes.c_void_p(stream_ptr)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.pfk_eri_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def one_electron(shells, coords, charges, device=0):
    """Overlap S, kinetic T and nuclear attraction V (nb x nb) on the GPU for
    point nuclei at `coords` (Bohr, natom x 3) with `charges` (pfk_one_electron)."""
    L = load_library()
    desc, keep = _basis_desc(shells)
    nb = int(sum((int(l) + 1) * (int(l) + 2) // 2 for l in keep["L"]))
    nuc = _f64(np.hstack([np.asarray(coords, dtype=np.float64).reshape(-1, 3),
                          np.asarray(charges, dtype=np.float64).reshape(-1, 1)]))
    S, T, V = (np.zeros((nb, nb)) for _ in range(3))
    st = L.pfk_one_electron(ctypes.byref(desc), len(nuc), _p(nuc), _p(S), _p(T), _p(V), int(device))
    if st != PFK_OK:
        raise PfkError(st, L.pfk_last_error(None).decode())
    return S, T, V


def measure_fma_peak(device=0):
    """(FP64, FP32) FMA throughput of the device in TFLOP/s."""
    L = load_library()
    a, b = ctypes.c_double(), ctypes.c_double()
    st = L.pfk_measure_fma_peak(int(device), ctypes.byref(a), ctypes.byref(b))
    if st != PFK_OK:
        raise PfkError(st, L.pfk_last_error(None).decode())
    return a.value, b.value


def class_flops(name, prim_quartets):
    """Algorithmic FP64 work of a class: K * n_r * [12 (e+1)(f+1) +
    6 (la+1)(lb+1)(lc+1)(ld+1) + 3 N] + 40 K (K = primitive quartets,
    e = la+lb, f = lc+ld, n_r = (e+f)//2 + 1, N = Cartesian block size)."""
    l = {"s": 0, "p": 1, "d": 2, "f": 3}
    la, lb, lc, ld = l[name[1]], l[name[2]], l[name[4]], l[name[5]]
    e, f = la + lb, lc + ld
    nr = (e + f) // 2 + 1
    nc = lambda x: (x + 1) * (x + 2) // 2
    N = nc(la) * nc(lb) * nc(lc) * nc(ld)
    return prim_quartets * nr * (12 * (e + 1) * (f + 1) + 6 * (la + 1) * (lb + 1) * (lc + 1) * (ld + 1) + 3 * N) \
        + 40 * prim_quartets


# ---------------------------------------------------------------------------
# Reference-shaped entry points (src/integrals/base.h:39-93).  The first
# argument is the FockEngine that stands in for the shell-pair vector.
# ---------------------------------------------------------------------------
def _prepare(eng, nbasis, engine, tol_eri, sym_ops):
    if sym_ops is not None and len(sym_ops) > 1:
        raise PfkError(PFK_ERR_UNSUPPORTED, "integral symmetry operations are not supported; pass None")
    if nbasis != eng.nbasis:
        raise PfkError(PFK_ERR_INVALID, f"nbasis {nbasis} does not match the engine ({eng.nbasis})")
    if tol_eri != eng.tol_eri or engine != eng.engine:
        eng.set_options(tol_eri, engine, eng.precision, eng.fp32_bound)


def _compute_2e(eng, nbasis, engine="os", tol_eri=1e-10, sym_ops=None):
    """Dense nb^4 tensor, row-major (base.h:39-55)."""
    _prepare(eng, nbasis, engine, tol_eri, sym_ops)
    return eng.eri_tensor().reshape(-1)


def _compute_2e_fock(eng, density, nbasis, engine="os", tol_eri=1e-10, sym_ops=None):
    """G = J - K/2 (base.h:57-73)."""
    _prepare(eng, nbasis, engine, tol_eri, sym_ops)
    return eng.fock_rhf(density)


def _compute_2e_fock_uhf(eng, Pa, Pb, nbasis, engine="os", tol_eri=1e-10, sym_ops=None):
    """(G_alpha, G_beta) (base.h:75-93)."""
    _prepare(eng, nbasis, engine, tol_eri, sym_ops)
    return eng.fock_uhf(Pa, Pb)
from . import checkpoint, guess, mlp, mp2, scf  # noqa: E402,F401  (RHF driver and learned guess; import this package lazily)
