"""The Boys-function scheme of the Obara-Saika kernels (CPU test).

boys_fm<M> in csrc/pfk_os.cuh evaluates F_0..F_M (M <= 6) as follows:
  * T below TS (1 for M <= 1, 2 for M <= 4, 3 above): the Taylor series of
    F_M, sum_k (-T)^k / (k! (2M+2k+1)), with 18, 25 or 32 terms, then the
    downward recursion F_m = (2T F_{m+1} + e^-T) / (2m+1);
  * up to TA (34, 38, 42, 44, 46 for M = 0..4, 60 above) F_0 =
    sqrt(pi)/2 erf(sqrt T)/sqrt T,
    with erf(sqrt T) = 1 - e^-T erfcx(sqrt T), and the upward recursion
    F_{m+1} = ((2m+1) F_m - e^-T) / (2T);
  * above TA the large-T limit F_0 = sqrt(pi/4T), F_{m+1} = (2m+1) F_m / (2T).
This test restates that scheme in double precision with the C library's exp
and scipy's erfcx and checks it against 40-digit Boys values.  The scheme's parameters
(thresholds, term counts) are what the device code uses.  The device's erfcx
and exp differ from the C library's by a few ulp, which the GPU integral tests
cover."""
import math

import numpy as np
import pytest
from scipy.special import erfcx

mpmath = pytest.importorskip("mpmath")


def _coef(M, k):
    return (-1) ** k / (math.factorial(k) * (2 * M + 2 * k + 1))


TA = {0: 34.0, 1: 38.0, 2: 42.0, 3: 44.0, 4: 46.0, 5: 60.0, 6: 60.0}


def boys_scheme(M, T):
    TS, NT = (1.0, 18) if M <= 1 else (2.0, 25) if M <= 4 else (3.0, 32)
    F = [0.0] * (M + 1)
    if T < TS:
        s = _coef(M, NT - 1)
        for k in range(NT - 2, -1, -1):
            s = s * T + _coef(M, k)
        F[M] = s
        e = math.exp(-T)
        for m in range(M - 1, -1, -1):
            F[m] = (2.0 * T * F[m + 1] + e) * (1.0 / (2 * m + 1))
    elif T < TA[M]:
        ist = 1.0 / math.sqrt(T)
        e = math.exp(-T)
        F[0] = 0.88622692545275801365 * (1.0 - e * erfcx(T * ist)) * ist
        h = 0.5 * ist * ist
        for m in range(M):
            F[m + 1] = ((2 * m + 1) * F[m] - e) * h
    else:
        ist = 1.0 / math.sqrt(T)
        F[0] = 0.88622692545275801365 * ist
        h = 0.5 * ist * ist
        for m in range(M):
            F[m + 1] = (2 * m + 1) * h * F[m]
    return F


def boys_exact(m, T):
    with mpmath.workdps(40):
        T = mpmath.mpf(T)
        if T == 0:
            return mpmath.mpf(1) / (2 * m + 1)
        return mpmath.gammainc(m + mpmath.mpf(1) / 2, 0, T) / (2 * T ** (m + mpmath.mpf(1) / 2))


@pytest.mark.parametrize("M,bound", [(0, 1e-15), (1, 2e-15), (2, 4e-15), (3, 8e-15), (4, 2e-14), (5, 2e-14),
                                     (6, 4e-14)])
def test_boys_scheme_relative_error(M, bound):
    rng = np.random.default_rng(M)
    Ts = np.concatenate([rng.uniform(0, 3, 150), rng.uniform(0, 80, 150), rng.uniform(45, 65, 60),
                         np.logspace(-14, 3, 40),
                         [0.0, 0.999999999, 1.0, 1.000000001, 1.999999999, 2.0, 2.000000001, 49.999999, 50.0,
                          59.999999, 60.0],
                         [TA[M] * (1 - 1e-9), TA[M], TA[M] * (1 + 1e-9)], rng.uniform(30, 50, 60)])
    worst = 0.0
    for T in Ts:
        F = boys_scheme(M, float(T))
        for m in range(M + 1):
            ref = boys_exact(m, T)
            worst = max(worst, float(abs((F[m] - ref) / ref)))
    assert worst < bound, worst
