"""60-digit reference values of contracted ERIs for a random s..f basis.

The basis is the one the ERI class microbenchmark draws from (tests/helpers.py
random_shells: exponents log-uniform in [0.05, 1e4], contraction depth 1..6,
coefficients in (0, 1], reference normalisation): 9 shells, seed 21, centres
in a 3 Angstrom cube.  For it the reference algorithm itself (restated in the
oracle) is not accurate to 1e-10: its OS and Rys engines disagree by up to
1e-6 absolute, from cancellation in the A->B transfer with the lower-L centre
first.  These values decide such elements.

Each value is computed independently of the oracle and of the CUDA code:
Rys quadrature with roots/weights from the exact Boys moments
(Stieltjes + symmetric eigensolve at 60 digits) and the transfer relations
expanded as binomial sums, all in mpmath at 60 digits.

Selection: the 60 AO quartets where the oracle's OS and Rys tensors differ
most, plus 40 seeded random quartets with |value| > 1e-4.  Writes
eri_highprec.json next to this script.  Runtime: a few minutes on 8 cores.

    python tests/golden/make_eri_highprec.py
"""
import json
import multiprocessing as mproc
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

SEED, NSHELL, BOX = 21, 9, 3.0


def _mp():
    import mpmath
    mpmath.mp.dps = 60
    return mpmath


def boys(m, k, T):
    if T == 0:
        return m.mpf(1) / (2 * k + 1)
    return m.hyp1f1(k + m.mpf(1) / 2, k + m.mpf(3) / 2, -T) / (2 * k + 1)


def gauss(m, mom, n):
    polys = [[1 / m.sqrt(mom[0])]]
    al, be = [], []

    def inner(a, b):
        return m.fsum(x * y * mom[i + j] for i, x in enumerate(a) for j, y in enumerate(b))

    for k in range(n):
        xp = [m.mpf(0)] + polys[k]
        a = inner(xp, polys[k])
        al.append(a)
        if k == n - 1:
            break
        q = list(xp)
        for i, c in enumerate(polys[k]):
            q[i] -= a * c
        if k > 0:
            for i, c in enumerate(polys[k - 1]):
                q[i] -= be[k - 1] * c
        b = m.sqrt(inner(q, q))
        be.append(b)
        polys.append([c / b for c in q])
    J = m.matrix(n, n)
    for i in range(n):
        J[i, i] = al[i]
        if i + 1 < n:
            J[i, i + 1] = J[i + 1, i] = be[i]
    E, Q = m.eigsy(J)
    return [E[i] for i in range(n)], [mom[0] * Q[0, i] ** 2 for i in range(n)]


def axis(m, la, lb, lc, ld, C00, D00, B00, B10, B01, AB, CD):
    E, F = la + lb, lc + ld
    I = [[m.mpf(0)] * (F + 1) for _ in range(E + 1)]
    I[0][0] = m.mpf(1)
    for a in range(E):
        I[a + 1][0] = C00 * I[a][0] + (a * B10 * I[a - 1][0] if a > 0 else 0)
    for c in range(F):
        for a in range(E + 1):
            v = D00 * I[a][c]
            if c > 0:
                v += c * B01 * I[a][c - 1]
            if a > 0:
                v += a * B00 * I[a - 1][c]
            I[a][c + 1] = v

    def ab(a, b, c):
        return m.fsum(m.binomial(b, t) * AB ** (b - t) * I[a + t][c] for t in range(b + 1))

    return m.fsum(m.binomial(ld, t) * CD ** (ld - t) * ab(la, lb, lc + t) for t in range(ld + 1))


def dfact(n):
    r = 1
    while n > 0:
        r *= n
        n -= 2
    return r


def eri(shells, ao):
    """ao: four (shell, (lx, ly, lz)) tuples."""
    m = _mp()
    off = np.concatenate([[0], np.cumsum(shells["nprim"])])
    cen = [[m.mpf(float(x)) for x in shells["center"][s]] for s, _ in ao]
    prims = [[(m.mpf(float(shells["expo"][p])), m.mpf(float(shells["coef"][p])) * m.mpf(float(shells["norm"][p])))
              for p in range(off[s], off[s + 1])] for s, _ in ao]
    ls = [l for _, l in ao]
    n = sum(sum(l) for l in ls) // 2 + 1
    A, B, C, D = cen
    d2 = lambda X, Y: sum((X[i] - Y[i]) ** 2 for i in range(3))
    tot = m.mpf(0)
    for a, ca in prims[0]:
        for b, cb in prims[1]:
            z = a + b
            P = [(a * A[i] + b * B[i]) / z for i in range(3)]
            Kab = (m.pi / z) ** 1.5 * m.exp(-a * b / z * d2(A, B)) * ca * cb
            for c, cc in prims[2]:
                for d, cd in prims[3]:
                    e = c + d
                    Q = [(c * C[i] + d * D[i]) / e for i in range(3)]
                    Kcd = (m.pi / e) ** 1.5 * m.exp(-c * d / e * d2(C, D)) * cc * cd
                    rho = z * e / (z + e)
                    T = rho * d2(P, Q)
                    pref = 2 * m.sqrt(rho / m.pi) * Kab * Kcd
                    us, ws = gauss(m, [boys(m, k, T) for k in range(2 * n + 1)], n)
                    W = [(z * P[i] + e * Q[i]) / (z + e) for i in range(3)]
                    for u, w in zip(us, ws):
                        B00 = u / (2 * (z + e))
                        B10 = (1 - rho / z * u) / (2 * z)
                        B01 = (1 - rho / e * u) / (2 * e)
                        val = w * pref
                        for x in range(3):
                            val *= axis(m, ls[0][x], ls[1][x], ls[2][x], ls[3][x],
                                        (P[x] - A[x]) + u * (W[x] - P[x]), (Q[x] - C[x]) + u * (W[x] - Q[x]),
                                        B00, B10, B01, A[x] - B[x], C[x] - D[x])
                        tot += val
    cn = m.mpf(1)
    for l in ls:
        cn /= m.sqrt(dfact(2 * l[0] - 1) * dfact(2 * l[1] - 1) * dfact(2 * l[2] - 1))
    return tot * cn


def _job(args):
    shells, ao = args
    return str(eri(shells, ao))


def main():
    import oracle
    from helpers import random_shells
    shells = random_shells(NSHELL, lmax=3, seed=SEED, box=BOX)
    ob = oracle.Basis(shells)
    shell, lxyz, _ = ob.ao_info()
    e_os, _ = ob.eri_tensor(1e-10, oracle.OS)
    e_ry, _ = ob.eri_tensor(1e-10, oracle.RYS)
    diff = np.abs(e_os - e_ry)
    picks, seen = [], set()

    def add(flat):
        idx = np.unravel_index(flat, e_os.shape)
        i, j, k, l = (int(x) for x in idx)
        key = tuple(sorted([tuple(sorted((i, j))), tuple(sorted((k, l)))]))
        if key not in seen:
            seen.add(key)
            picks.append((i, j, k, l))

    for f in np.argsort(diff.ravel())[::-1]:
        if len(picks) >= 60:
            break
        add(int(f))
    rng = np.random.default_rng(SEED)
    cand = np.flatnonzero(np.abs(e_os.ravel()) > 1e-4)
    for f in rng.choice(cand, 200, replace=False):
        if len(picks) >= 100:
            break
        add(int(f))
    jobs = [(shells, [(int(shell[x]), tuple(int(v) for v in lxyz[x])) for x in q]) for q in picks]
    with mproc.get_context("spawn").Pool(os.cpu_count()) as pool:
        vals = pool.map(_job, jobs, chunksize=1)
    out = {"seed": SEED, "nshell": NSHELL, "box_angstrom": BOX,
           "note": "60-digit values; oracle OS/Rys max disagreement %.3e" % diff.max(),
           "oracle_os_rys_max_diff": float(diff.max()),
           "quartets": [[list(q), v, float(e_os[q]), float(e_ry[q])] for q, v in zip(picks, vals)]}
    with open(os.path.join(HERE, "eri_highprec.json"), "w") as f:
        json.dump(out, f, indent=0)
    worst_os = max(abs(float(v) - e_os[q]) for q, v in zip(picks, vals))
    print("wrote", len(picks), "values; oracle OS worst error vs 60 digits %.3e" % worst_os)


if __name__ == "__main__":
    main()
