"""CPU restatement of the reference's AO -> MO transform and MP2 energies
(test infrastructure: the tests compare pfk_mo_transform and
planck-refactored_b200/mp2.py with it; nothing in the product imports it).

  transform_eri  src/post_hf/integrals.cpp:63-134 -- four quarter
                 transforms over a row-major nb^4 AO tensor, each a
                 contraction over one AO index, in the reference's order
                 (mu, then nu, then lambda, then sigma);
  rmp2_energy    src/post_hf/mp2.cpp:25-35 with tau from
                 src/post_hf/mp2_gradient.cpp:216-230;
  ump2_energy    src/post_hf/mp2.cpp:93-142.
Pinned through the reference's UMP2 regression energy (water radical
cation / STO-3G, tests/regression_cases.json) in the GPU tests, and here
against the one-shot definition sum C C C C (mu nu|lam sig).
"""
import numpy as np


def transform_eri(eri, C1, C2, C3, C4):
    nb = C1.shape[0]
    E = eri.reshape(nb, nb, nb, nb)
    T1 = np.tensordot(C1, E, axes=([0], [0]))                       # [i, nu, lam, sig]
    T2 = np.tensordot(T1, C2, axes=([1], [0])).transpose(0, 3, 1, 2)  # [i, a, lam, sig]
    T3 = np.tensordot(T2, C3, axes=([2], [0])).transpose(0, 1, 3, 2)  # [i, a, j, sig]
    return np.tensordot(T3, C4, axes=([3], [0]))                    # [i, a, j, b]


def _den(eo1, ev1, eo2, ev2):
    return eo1[:, None, None, None] - ev1[None, :, None, None] + eo2[None, None, :, None] - ev2[None, None, None, :]


def rmp2_energy(eri, C, eps, nocc):
    Co, Cv = C[:, :nocc], C[:, nocc:]
    iajb = transform_eri(eri, Co, Cv, Co, Cv)
    tau = (2.0 * iajb - iajb.transpose(0, 3, 2, 1)) / _den(eps[:nocc], eps[nocc:], eps[:nocc], eps[nocc:])
    return float(np.sum(iajb * tau))


def ump2_energy(eri, Ca, eps_a, Cb, eps_b, na, nb_):
    e = 0.0
    for C, eps, n in ((Ca, eps_a, na), (Cb, eps_b, nb_)):
        g = transform_eri(eri, C[:, :n], C[:, n:], C[:, :n], C[:, n:])
        anti = g - g.transpose(0, 3, 2, 1)
        e += 0.25 * float(np.sum(anti * anti / _den(eps[:n], eps[n:], eps[:n], eps[n:])))
    g = transform_eri(eri, Ca[:, :na], Ca[:, na:], Cb[:, :nb_], Cb[:, nb_:])
    return e + float(np.sum(g * g / _den(eps_a[:na], eps_a[na:], eps_b[:nb_], eps_b[nb_:])))
