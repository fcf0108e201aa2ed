"""CPU restatement of the reference's checkpoint format (test infrastructure).

The tests compare the library's .hfchk writer and density reader with it
(planck-refactored_b200/csrc/pfk_checkpoint.cu); nothing in the product
imports it.  It follows the reference's src/io/checkpoint.cpp:
  save()                      checkpoint.cpp:347-489
  load(load_1e_matrices=0)    checkpoint.cpp:491-663
  read_* helpers and limits   checkpoint.cpp:26-225
  adapt_restart_spin_state    checkpoint.cpp:294-336 (density_from_mos 272-292)

Parity unpinned: the reference's checkpoint code needs Eigen, which this
machine lacks, so it cannot be compiled and run here, and the reference ships
no .hfchk fixture.  The byte layout below is restated from the code above and
the format comment in src/io/checkpoint.h:11-72; the tests compare the
library with this restatement byte for byte and message for message.
"""
import struct

import numpy as np

MAGIC = b"PLNKCHK\0"
VERSION = 6
MAX_STRING = 4096
MAX_ATOMS = 1_000_000


class CheckpointError(Exception):
    pass


def _dfact(n):
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def _matrix(m):
    """int64 rows, int64 cols, column-major doubles (write_matrix, checkpoint.cpp:114-122)."""
    m = np.asarray(m, dtype=np.float64)
    if m.ndim == 1:
        m = m.reshape(-1, 1)
    return struct.pack("<qq", *m.shape) + np.asfortranarray(m).tobytes(order="F")


def save(meta, shells, S, H, alpha, beta=None):
    """Bytes of the checkpoint Checkpoint::save writes.  meta: dict with
    natoms-length 'Z' and 'coords' (Bohr), 'charge', 'multiplicity',
    'basis_name', 'total_energy', 'nuclear_repulsion', 'converged',
    'has_opt_coords'.  alpha/beta: dicts with density, fock, mo_energies,
    mo_coefficients (numpy matrices, logical layout)."""
    L, nprim = shells["L"], shells["nprim"]
    nb = int(sum((l + 1) * (l + 2) // 2 for l in L))
    out = bytearray()
    out += MAGIC
    out += struct.pack("<IQBBIdd", VERSION, nb, 1 if beta is not None else 0, 1 if meta["converged"] else 0, 0,
                       meta["total_energy"], meta["nuclear_repulsion"])
    Z = list(meta["Z"])
    out += struct.pack("<QiI", len(Z), meta["charge"], meta["multiplicity"])
    out += struct.pack(f"<{len(Z)}i", *[int(z) for z in Z])
    out += np.asarray(meta["coords"], dtype=np.float64).reshape(-1).tobytes()
    name = meta["basis_name"].encode()
    out += struct.pack("<I", len(name)) + name
    out += struct.pack("<B", 1 if meta["has_opt_coords"] else 0)
    out += _matrix(S) + _matrix(H)
    for ch in (alpha, beta):
        if ch is None:
            continue
        out += _matrix(ch["density"]) + _matrix(ch["fock"]) + _matrix(ch["mo_energies"])
        out += _matrix(ch["mo_coefficients"])
    out += struct.pack("<B", 0)                 # has_casscf_mos
    out += struct.pack("<BQ", 1, len(L))        # has_basis, nshells
    p0 = 0
    for s, l in enumerate(L):
        n = int(nprim[s])
        out += struct.pack("<iI", int(l), n) + np.asarray(shells["center"][s], dtype=np.float64).tobytes()
        for key in ("expo", "coef", "norm"):
            out += np.asarray(shells[key][p0:p0 + n], dtype=np.float64).tobytes()
        p0 += n
    out += struct.pack("<Q", nb)
    for s, l in enumerate(L):
        l = int(l)
        for lx in range(l, -1, -1):             # _cartesian_shell_order: lx, then ly descending
            for ly in range(l - lx, -1, -1):
                lz = l - lx - ly
                df = _dfact(2 * lx - 1) * _dfact(2 * ly - 1) * _dfact(2 * lz - 1)
                out += struct.pack("<Qiiid", s, lx, ly, lz, 1.0 / np.sqrt(float(df)))
    out += struct.pack("<BB", 0, 0)             # v5, v6 flags
    return bytes(out)


class _In:
    def __init__(self, data):
        self.d, self.o = data, 0

    def exact(self, n, label):
        if self.o + n > len(self.d):
            raise CheckpointError(f"Checkpoint truncated while reading {label}")
        b = self.d[self.o:self.o + n]
        self.o += n
        return b

    def pod(self, fmt):
        n = struct.calcsize("<" + fmt)
        if self.o + n > len(self.d):
            raise CheckpointError(f"Checkpoint truncated while reading {n} bytes")
        v = struct.unpack_from("<" + fmt, self.d, self.o)[0]
        self.o += n
        return v

    def string(self):
        n = struct.unpack("<I", self.exact(4, "string length"))[0]
        if n > MAX_STRING:
            raise CheckpointError(f"Checkpoint string length {n} exceeds supported limit {MAX_STRING}")
        return self.exact(n, "string data").decode() if n else ""

    def matrix(self, max_dim, label, vector=False):
        rows = struct.unpack("<q", self.exact(8, f"{label} row count"))[0]
        cols = struct.unpack("<q", self.exact(8, f"{label} column count"))[0]
        if vector and cols != 1:
            raise CheckpointError(f"Checkpoint {label} is not stored as an n x 1 vector")
        if rows < 0 or cols < 0:
            raise CheckpointError(f"Checkpoint {label} has negative dimensions")
        if rows > max_dim or cols > max_dim:
            raise CheckpointError(f"Checkpoint {label} dimensions {rows}x{cols} exceed supported limit {max_dim}")
        n = rows * cols
        data = self.exact(8 * n, f"{label} data") if n else b""
        return np.frombuffer(data, dtype=np.float64).reshape((cols, rows)).T.copy() if n else np.zeros((rows, cols))


def load_density(data, nbasis, target_uhf=False, n_alpha=0, n_beta=0):
    """(Pa, Pb, total_energy, file_uhf) as Checkpoint::load(calc, path, false)
    leaves them, adapted to the target; raises CheckpointError with the
    reference's message."""
    r = _In(data)
    if r.exact(8, "magic") != MAGIC:
        raise CheckpointError("Not a valid Planck checkpoint file (bad magic)")
    version = r.pod("I")
    if version < 2 or version > VERSION:
        raise CheckpointError(f"Checkpoint version mismatch: file={version}, expected={VERSION}")
    nb = r.pod("Q")
    uhf = r.pod("B")
    r.pod("B")
    r.pod("I")
    etot = r.pod("d")
    r.pod("d")
    natoms = r.pod("Q")
    if natoms > MAX_ATOMS:
        raise CheckpointError(f"Checkpoint geometry block atom count {natoms} exceeds supported limit {MAX_ATOMS}")
    r.pod("i")
    r.pod("I")
    for _ in range(natoms):
        r.pod("i")
    for _ in range(3 * natoms):
        r.pod("d")
    r.string()
    r.pod("B")
    if nb != nbasis:
        raise CheckpointError(f"Checkpoint nbasis ({nb}) does not match current nbasis ({nbasis}); "
                              "use the same basis set or remove the checkpoint file.")
    r.matrix(nb, "overlap matrix")
    r.matrix(nb, "core Hamiltonian")
    chans = []
    for label in (("alpha", "beta") if uhf else ("alpha",)):
        D = r.matrix(nb, f"{label} density")
        r.matrix(nb, f"{label} fock")
        r.matrix(nb, f"{label} orbital energies", vector=True)
        C = r.matrix(nb, f"{label} MO coefficients")
        chans.append((D, C))
    if version >= 3 and r.pod("B"):
        r.matrix(nb, "CASSCF MO coefficients")
    if uhf:
        if target_uhf:
            return chans[0][0], chans[1][0], etot, True
        return chans[0][0] + chans[1][0], None, etot, True
    if not target_uhf:
        return chans[0][0], None, etot, False
    C = chans[0][1]
    out = []
    for nocc in (n_alpha, n_beta):
        if nocc <= 0 or C.size == 0:
            out.append(np.zeros((C.shape[0], C.shape[0])))
            continue
        if nocc > C.shape[1]:
            raise CheckpointError(f"Checkpoint orbital block has {C.shape[1]} columns but {nocc} occupied "
                                  "orbitals are required")
        occ = C[:, :nocc]
        out.append(occ @ occ.T)
    return out[0], out[1], etot, False
