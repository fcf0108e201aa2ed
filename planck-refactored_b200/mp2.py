"""MP2 correlation energies on the device AO -> MO transform.

The MO integrals come from FockEngine.mo_transform (pfk_mo_transform: the
AO tensor built by the class kernels and the four quarter transforms as FP64
GEMMs, all on the GPU); the energy sums follow the reference:
  rmp2  run_rmp2 (src/post_hf/mp2.cpp:10-38) with the amplitudes of
        build_rmp2_amplitudes (src/post_hf/mp2_gradient.cpp:203-232):
        E = sum_{iajb} (ia|jb) [2 (ia|jb) - (ib|ja)] / (e_i + e_j - e_a - e_b)
  ump2  run_ump2 (src/post_hf/mp2.cpp:43-143): the alpha-alpha and beta-beta
        terms 1/4 sum [(ia|jb) - (ib|ja)]^2 / D and the alpha-beta term
        sum (ia|jb)^2 / D, from three transforms.
"""
import numpy as np


def _denominator(eo1, ev1, eo2, ev2):
    return (eo1[:, None, None, None] - ev1[None, :, None, None] + eo2[None, None, :, None]
            - ev2[None, None, None, :])


def rmp2(engine, C, eps, nocc):
    """RMP2 correlation energy of a converged RHF (MO coefficients C, orbital
    energies eps, nocc doubly occupied orbitals)."""
    nb = C.shape[0]
    if nocc <= 0 or nocc >= nb:
        raise ValueError("rmp2: no occupied or virtual orbitals")
    Co, Cv = C[:, :nocc], C[:, nocc:]
    iajb = engine.mo_transform(Co, Cv, Co, Cv)
    ibja = iajb.transpose(0, 3, 2, 1)
    D = _denominator(eps[:nocc], eps[nocc:], eps[:nocc], eps[nocc:])
    return float(np.sum(iajb * (2.0 * iajb - ibja) / D))


def ump2(engine, Ca, eps_a, Cb, eps_b, n_alpha, n_beta):
    """UMP2 correlation energy of a converged UHF."""
    nb = Ca.shape[0]
    if n_alpha == 0 or n_alpha >= nb or n_beta == 0 or n_beta >= nb:
        raise ValueError("ump2: no occupied or virtual orbitals in a spin channel")
    Cao, Cav, Cbo, Cbv = Ca[:, :n_alpha], Ca[:, n_alpha:], Cb[:, :n_beta], Cb[:, n_beta:]
    e = 0.0
    for Co, Cv, eo, ev in ((Cao, Cav, eps_a[:n_alpha], eps_a[n_alpha:]), (Cbo, Cbv, eps_b[:n_beta], eps_b[n_beta:])):
        g = engine.mo_transform(Co, Cv, Co, Cv)
        anti = g - g.transpose(0, 3, 2, 1)
        e += 0.25 * float(np.sum(anti * anti / _denominator(eo, ev, eo, ev)))
    g = engine.mo_transform(Cao, Cav, Cbo, Cbv)
    e += float(np.sum(g * g / _denominator(eps_a[:n_alpha], eps_a[n_alpha:], eps_b[:n_beta], eps_b[n_beta:])))
    return e
