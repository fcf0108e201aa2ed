"""Planck checkpoint files (.hfchk) through the C ABI (pfk_checkpoint_*).

The reference restarts an SCF from a checkpoint with `guess density`
(src/io/checkpoint.h:11-72, load() at src/io/checkpoint.cpp:491-663): it
takes the stored density as the first iteration's density.  This module
writes such files for densities made here -- the learned guess
(save_guess) or a converged GPU SCF (write) -- and reads the density back
from any version 2-6 checkpoint (read_density), so the GPU driver can
restart from the reference's files too.  File writing and reading are host
code in the library (csrc/pfk_checkpoint.cu) and need no GPU.
"""
import ctypes

import numpy as np


class PfkCheckpointMeta(ctypes.Structure):
    _fields_ = [("natoms", ctypes.c_int), ("atomic_numbers", ctypes.c_void_p), ("coords_bohr", ctypes.c_void_p),
                ("charge", ctypes.c_int), ("multiplicity", ctypes.c_uint), ("basis_name", ctypes.c_char_p),
                ("total_energy", ctypes.c_double), ("nuclear_repulsion", ctypes.c_double),
                ("converged", ctypes.c_int), ("has_opt_coords", ctypes.c_int)]


class PfkSpinChannel(ctypes.Structure):
    _fields_ = [("density", ctypes.c_void_p), ("fock", ctypes.c_void_p), ("mo_energies", ctypes.c_void_p),
                ("mo_coefficients", ctypes.c_void_p)]


def _lib():
    from . import load_library
    L = load_library()
    if not getattr(L, "_chk_ready", False):
        vp, c_int = ctypes.c_void_p, ctypes.c_int
        L.pfk_checkpoint_write.argtypes = [ctypes.c_char_p, ctypes.POINTER(PfkCheckpointMeta), vp, vp, vp,
                                           ctypes.POINTER(PfkSpinChannel), ctypes.POINTER(PfkSpinChannel)]
        L.pfk_checkpoint_read_density.argtypes = [ctypes.c_char_p, c_int, c_int, c_int, c_int, vp, vp,
                                                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(c_int)]
        L.pfk_checkpoint_last_error.restype = ctypes.c_char_p
        L.pfk_checkpoint_last_error.argtypes = []
        L._chk_ready = True
    return L


class CheckpointError(RuntimeError):
    pass


def _colmajor(M):
    """Column-major bytes of a matrix (the layout the C ABI and the file use)."""
    return np.ascontiguousarray(np.asarray(M, dtype=np.float64).T)


def natural_orbitals(P, S):
    """MO coefficients C (S-orthonormal columns, occupation descending) and
    occupations n of a closed-shell density P: the eigenvectors V of
    S^1/2 P S^1/2 / 2, C = S^-1/2 V."""
    s, U = np.linalg.eigh(S)
    Sh = (U * np.sqrt(s)) @ U.T
    Smh = (U / np.sqrt(s)) @ U.T
    w, V = np.linalg.eigh(0.5 * Sh @ P @ Sh)
    order = np.argsort(-w, kind="stable")
    return Smh @ V[:, order], w[order]


def write(path, system, P, F=None, energy=0.0, converged=False, Pb=None, Fb=None, multiplicity=1,
          has_opt_coords=False):
    """Write `system`'s checkpoint with closed-shell density P (or spin
    densities P, Pb for an open-shell file) and Fock matrices F (Fb).  MO
    coefficients are P's natural orbitals, occupied first, so a UHF or ROHF
    reader of an RHF file finds its occupied orbitals in the leading
    columns; orbital energies are their Rayleigh quotients with F.  F
    defaults to the core Hamiltonian."""
    L = _lib()
    from . import _basis_desc
    desc, keep = _basis_desc(system.shells)
    mol = system.mol
    Z = np.ascontiguousarray(np.rint(mol.Z).astype(np.int32))
    xyz = np.ascontiguousarray(np.asarray(mol.coords, dtype=np.float64).reshape(-1))
    name = getattr(system, "basis_name", "").encode()
    meta = PfkCheckpointMeta(len(Z), Z.ctypes.data, xyz.ctypes.data, int(getattr(mol, "charge", 0)),
                             int(multiplicity), name,
                             float(energy), float(system.enuc), 1 if converged else 0, 1 if has_opt_coords else 0)
    hold = [Z, xyz]

    def channel(Pm, Fm, factor):
        C, _ = natural_orbitals(Pm * (2.0 / factor), system.S)
        Fm = system.H if Fm is None else Fm
        eps = np.sum(C * (Fm @ C), axis=0)   # C_j^T F C_j
        arrays = [_colmajor(Pm), _colmajor(Fm), np.ascontiguousarray(eps), _colmajor(C)]
        hold.extend(arrays)
        return PfkSpinChannel(*[a.ctypes.data for a in arrays])

    S, H = _colmajor(system.S), _colmajor(system.H)
    if Pb is None:
        a, b = channel(P, F, 2.0), None
    else:
        a, b = channel(P, F, 1.0), channel(Pb, Fb, 1.0)
    st = L.pfk_checkpoint_write(str(path).encode(), ctypes.byref(meta), ctypes.addressof(desc), S.ctypes.data,
                                H.ctypes.data, ctypes.byref(a), ctypes.byref(b) if b is not None else None)
    if st != 0:
        raise CheckpointError(L.pfk_checkpoint_last_error().decode())


def read_density(path, nbasis, uhf=False, n_alpha=0, n_beta=0):
    """(Pa, Pb, total_energy, file_is_spin_resolved) for a restart with
    `guess density`: Pa is the closed-shell density for an RHF target (Pb
    None), else the two spin densities (an RHF file's from its first
    n_alpha / n_beta MO columns)."""
    L = _lib()
    Pa = np.zeros((nbasis, nbasis))
    Pb = np.zeros((nbasis, nbasis)) if uhf else None
    e = ctypes.c_double(0.0)
    fu = ctypes.c_int(0)
    st = L.pfk_checkpoint_read_density(str(path).encode(), int(nbasis), 1 if uhf else 0, int(n_alpha), int(n_beta),
                                       Pa.ctypes.data, Pb.ctypes.data if uhf else None, ctypes.byref(e),
                                       ctypes.byref(fu))
    if st != 0:
        raise CheckpointError(L.pfk_checkpoint_last_error().decode())
    # the file is column-major; the densities are symmetric, but return them
    # in logical layout regardless
    return Pa.T.copy(), (Pb.T.copy() if uhf else None), e.value, bool(fu.value)


def save_guess(path, model, system):
    """Run the learned-guess hook (guess.choose) on `system` and write its
    density to `path` for the reference's `guess density` restart, with the
    first-iteration energy and Fock matrix H + G.  Returns what the hook
    returns, (P0, G0, info)."""
    from . import guess
    from .scf import first_energy
    P0, G0, info = guess.choose(model, system)
    write(path, system, P0, F=system.H + G0, energy=first_energy(system.H, system.enuc, P0, G0), converged=False)
    return P0, G0, info
