"""Checkpoint files (.hfchk) written and read by the library's C ABI
(pfk_checkpoint_write / pfk_checkpoint_read_density, host code), checked
against the oracle's restatement of the reference's Checkpoint::save and
Checkpoint::load (src/io/checkpoint.cpp:347-663): identical bytes, identical
densities after the reference's spin adaptation, and the reference's error
messages on damaged files.  No GPU is needed."""
import struct
import types

import numpy as np
import pytest

from helpers import WATER, alkane, basis_library, pfk

from oracle import checkpoint_ref as ref


def _system(atoms=WATER, basis="6-31g**", seed=0):
    """A stand-in for scf.System with seeded S, H (the file format does not
    care where they came from)."""
    P = pfk()
    mol, shells = P.shells_for(atoms, basis, basis_library())
    nb = int(sum((int(l) + 1) * (int(l) + 2) // 2 for l in shells["L"]))
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(nb, nb))
    S = A @ A.T / nb + np.eye(nb)
    B = rng.normal(size=(nb, nb))
    return types.SimpleNamespace(mol=mol, shells=shells, S=S, H=B + B.T, enuc=9.1875, basis_name=basis), nb


def _closed_shell_density(S, nocc, seed):
    rng = np.random.default_rng(seed)
    nb = S.shape[0]
    s, U = np.linalg.eigh(S)
    Smh = (U / np.sqrt(s)) @ U.T
    Q, _ = np.linalg.qr(rng.normal(size=(nb, nb)))
    C = Smh @ Q[:, :nocc]
    return 2.0 * C @ C.T


def _oracle_bytes(sysm, P, F, energy, Pb=None, Fb=None, multiplicity=1):
    C = pfk().checkpoint
    meta = {"Z": np.rint(sysm.mol.Z).astype(int), "coords": sysm.mol.coords, "charge": sysm.mol.charge,
            "multiplicity": multiplicity, "basis_name": sysm.basis_name, "total_energy": energy,
            "nuclear_repulsion": sysm.enuc, "converged": False, "has_opt_coords": False}

    def chan(Pm, Fm, factor):
        Cm, _ = C.natural_orbitals(Pm * (2.0 / factor), sysm.S)
        return {"density": Pm, "fock": Fm, "mo_energies": np.sum(Cm * (Fm @ Cm), axis=0),
                "mo_coefficients": Cm}

    if Pb is None:
        return ref.save(meta, sysm.shells, sysm.S, sysm.H, chan(P, F, 2.0))
    return ref.save(meta, sysm.shells, sysm.S, sysm.H, chan(P, F, 1.0), chan(Pb, Fb, 1.0))


@pytest.mark.parametrize("case", ["water_631gss", "butane_ccpvdz"])
def test_writer_matches_oracle_bytes(tmp_path, case):
    atoms, basis = (WATER, "6-31g**") if case == "water_631gss" else (alkane(4), "cc-pvdz")
    sysm, nb = _system(atoms, basis, seed=3)
    P = _closed_shell_density(sysm.S, 5, seed=4)
    F = sysm.H + 0.1 * np.eye(nb)
    path = tmp_path / "g.hfchk"
    pfk().checkpoint.write(path, sysm, P, F=F, energy=-76.0123)
    got = path.read_bytes()
    want = _oracle_bytes(sysm, P, F, -76.0123)
    assert len(got) == len(want)
    assert got == want
    Pa, Pb, e, uhf = ref.load_density(got, nb)
    assert np.array_equal(Pa, P) and Pb is None and e == -76.0123 and not uhf


def test_uhf_writer_matches_oracle_bytes(tmp_path):
    sysm, nb = _system(seed=5)
    Pa = 0.5 * _closed_shell_density(sysm.S, 5, seed=6)
    Pb = 0.5 * _closed_shell_density(sysm.S, 4, seed=7)
    path = tmp_path / "u.hfchk"
    pfk().checkpoint.write(path, sysm, Pa, F=sysm.H, Pb=Pb, Fb=sysm.H, energy=-75.5, multiplicity=2)
    assert path.read_bytes() == _oracle_bytes(sysm, Pa, sysm.H, -75.5, Pb=Pb, Fb=sysm.H, multiplicity=2)


@pytest.mark.parametrize("file_uhf,target_uhf", [(False, False), (False, True), (True, False), (True, True)])
def test_read_density_adapts_spin_like_the_reference(tmp_path, file_uhf, target_uhf):
    """The four cases of adapt_restart_spin_state (checkpoint.cpp:294-336)."""
    sysm, nb = _system(seed=8)
    Pa = _closed_shell_density(sysm.S, 5, seed=9)
    path = tmp_path / "x.hfchk"
    if file_uhf:
        Pb = 0.5 * _closed_shell_density(sysm.S, 4, seed=10)
        pfk().checkpoint.write(path, sysm, 0.5 * Pa, Pb=Pb, energy=-1.0, multiplicity=2)
    else:
        pfk().checkpoint.write(path, sysm, Pa, energy=-1.0)
    data = path.read_bytes()
    oa, ob, oe, ou = ref.load_density(data, nb, target_uhf, 5, 4)
    ga, gb, ge, gu = pfk().checkpoint.read_density(path, nb, target_uhf, 5, 4)
    assert ge == oe and gu == ou == file_uhf
    if file_uhf or not target_uhf:   # stored densities, or their sum: exact
        assert np.array_equal(ga, oa)
        assert (gb is None and ob is None) or np.array_equal(gb, ob)
    else:                            # C_occ C_occ^T in another summation order
        assert np.abs(ga - oa).max() < 1e-13 and np.abs(gb - ob).max() < 1e-13
        # the natural orbitals of an idempotent P reproduce it: its 5
        # occupied ones give the alpha density P/2
        assert np.abs(ga - 0.5 * Pa).max() < 1e-10


def _damaged(data, nb):
    """(name, bytes) pairs for damaged files: every header field truncated,
    a bad magic, versions out of range, a too-long basis name, a vector
    stored with two columns, negative and oversized matrix dimensions, an
    nbasis mismatch, and a version 2 file (no CASSCF flag), which is valid."""
    out = [("empty", b""), ("magic", b"PLNKCHX\0" + data[8:])]
    for v in (1, 7):
        out.append((f"version{v}", data[:8] + struct.pack("<I", v) + data[12:]))
    for cut in (5, 10, 15, 18, 21, 30, 40, 60, 80, 100, 200, 1000, len(data) // 2, len(data) - 3):
        out.append((f"cut{cut}", data[:cut]))
    off = 8 + 4 + 8 + 1 + 1 + 4 + 8 + 8
    natoms = struct.unpack_from("<Q", data, off)[0]
    name_off = off + 8 + 4 + 4 + 4 * natoms + 24 * natoms
    out.append(("longname", data[:name_off] + struct.pack("<I", 5000) + data[name_off + 4:]))
    out.append(("bignatoms", data[:off] + struct.pack("<Q", 2_000_000) + data[off + 8:]))
    mat0 = name_off + 4 + struct.unpack_from("<I", data, name_off)[0] + 1
    out.append(("negdim", data[:mat0] + struct.pack("<q", -1) + data[mat0 + 8:]))
    out.append(("bigdim", data[:mat0] + struct.pack("<q", nb + 1) + data[mat0 + 8:]))
    # the alpha orbital-energy vector: after S, H, density and Fock
    vec = mat0 + 4 * (16 + 8 * nb * nb)
    out.append(("vec2cols", data[:vec + 8] + struct.pack("<q", 2) + data[vec + 16:]))
    v2_end = vec + 16 + 8 * nb + 16 + 8 * nb * nb
    out.append(("version2", data[:8] + struct.pack("<I", 2) + data[12:v2_end]))
    return out


def test_damaged_files_fail_with_the_references_messages(tmp_path):
    sysm, nb = _system(seed=11)
    P = _closed_shell_density(sysm.S, 5, seed=12)
    good = tmp_path / "good.hfchk"
    pfk().checkpoint.write(good, sysm, P, energy=-2.0)
    data = good.read_bytes()
    for name, blob in _damaged(data, nb):
        path = tmp_path / f"{name}.hfchk"
        path.write_bytes(blob)
        try:
            want = ref.load_density(blob, nb)
            want_err = None
        except ref.CheckpointError as e:
            want_err = str(e)
        if want_err is None:
            got = pfk().checkpoint.read_density(path, nb)
            assert np.array_equal(got[0], want[0]), name
        else:
            with pytest.raises(pfk().checkpoint.CheckpointError) as ei:
                pfk().checkpoint.read_density(path, nb)
            assert str(ei.value) == want_err, name
    # nbasis mismatch and a missing file
    with pytest.raises(pfk().checkpoint.CheckpointError, match=r"Checkpoint nbasis \(25\) does not match current"):
        pfk().checkpoint.read_density(good, nb + 1)
    with pytest.raises(pfk().checkpoint.CheckpointError, match="Cannot open checkpoint file"):
        pfk().checkpoint.read_density(tmp_path / "missing.hfchk", nb)
