"""The oracle's restatement of the AO -> MO transform and MP2 energies
(oracle/mo_ref.py) checked on the CPU: the quarter transforms in the
reference's order against the one-shot definition, and UMP2 of a
closed-shell reference against RMP2."""
import numpy as np

from oracle import mo_ref


def _sym_tensor(nb, seed):
    """A random AO tensor with the 8-fold permutational symmetry of (mn|ls)."""
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(nb, nb, nb, nb))
    A = A + A.transpose(1, 0, 2, 3)
    A = A + A.transpose(0, 1, 3, 2)
    return A + A.transpose(2, 3, 0, 1)


def test_quarter_transforms_match_the_definition():
    nb = 7
    eri = _sym_tensor(nb, 1)
    rng = np.random.default_rng(2)
    C = [rng.normal(size=(nb, n)) for n in (2, 5, 3, 4)]
    want = np.einsum("mnls,mi,na,lj,sb->iajb", eri, *C, optimize=True)
    got = mo_ref.transform_eri(eri.reshape(-1), *C)
    assert got.shape == (2, 5, 3, 4)
    assert np.abs(got - want).max() < 1e-11 * np.abs(want).max()


def test_ump2_of_a_closed_shell_is_rmp2():
    nb, nocc = 8, 3
    eri = _sym_tensor(nb, 3) * 0.01
    rng = np.random.default_rng(4)
    C, _ = np.linalg.qr(rng.normal(size=(nb, nb)))
    eps = np.sort(rng.normal(size=nb))
    eps[nocc:] += 2.0   # a gap, so every denominator is negative
    e_r = mo_ref.rmp2_energy(eri, C, eps, nocc)
    e_u = mo_ref.ump2_energy(eri, C, eps, C, eps, nocc, nocc)
    assert e_r < 0 and abs(e_u - e_r) < 1e-12 * abs(e_r)


def test_oracle_rmp2_reproduces_the_reference_regression():
    """The oracle's RHF and RMP2 on water / STO-3G give the reference's
    recorded energies (tests/regression_cases.json:39-50) within its 1e-9."""
    import oracle
    from helpers import regression_cases
    c = regression_cases()["water_rmp2_sto3g"]
    mol = oracle.Molecule(c["atoms"])
    eri, _ = oracle.Basis(oracle.shells_for(mol, c["basis"])).eri_tensor(1e-10, oracle.OS)
    r = oracle.rhf_conventional(c["atoms"], c["basis"])
    e_corr = mo_ref.rmp2_energy(eri, r["C"], r["eps"], mol.nelectron() // 2)
    assert abs(r["energy"] - c["energy"]) < c["atol"]
    assert abs(r["energy"] + e_corr - c["mp2_energy"]) < c["mp2_atol"]
