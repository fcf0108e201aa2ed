"""40-digit nuclear-attraction matrix of a random s..f basis.

The basis and nuclei are those of the one-electron GPU test
(tests/test_scf_gpu.py, case random_f): workloads.random_shells(10, lmax=3,
seed=31, box=3.0) -- exponents log-uniform in [0.05, 1e4], contraction depth
1..6, reference normalisation -- and four point charges (Z = 1, 6, 8, 7) at
seeded positions in the same 3 Angstrom cube.  On this basis the reference's
own one-electron code (os.cpp:294-602, restated in the oracle) is not
accurate to 1e-10: its diagonal (ff|V|ff) elements are off by up to 7e-9,
which the Boys values it uses at high order explain.  These values decide
such elements.

Each value is computed independently of the oracle and of the CUDA code, in
mpmath at 40 digits: Boys values from the confluent hypergeometric function,
the Obara-Saika vertical recurrence on centre A over every nucleus and
primitive pair, then the horizontal transfer to centre B.  At 40 digits the
transfer's cancellation costs nothing.  Writes onee_highprec.json next to
this script (the upper triangle of V, Cartesian order, component norms
applied).  Runtime: about a minute on 8 cores.

    python tests/golden/make_onee_highprec.py
"""
import importlib
import json
import multiprocessing as mproc
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

SEED, NSHELL, BOX, NUC_SEED = 31, 10, 3.0, 2
Z = [1.0, 6.0, 8.0, 7.0]


def inputs():
    P = importlib.import_module("planck-refactored_b200")
    shells = P.workloads.random_shells(NSHELL, lmax=3, seed=SEED, box=BOX)
    rng = np.random.default_rng(NUC_SEED)
    coords = rng.uniform(0, BOX * P.basis.ANGSTROM_TO_BOHR, (len(Z), 3))
    return shells, coords


def carts(L):
    return [(L - yz, yz - z, z) for yz in range(L + 1) for z in range(yz + 1)]


def dfact(n):
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def pair_block(args):
    """V block of shells (a, b), L(a) >= L(b): {(i, j): 40-digit string}."""
    a, b = args
    import mpmath as m
    m.mp.dps = 40
    shells, coords = inputs()
    L, npr = shells["L"], shells["nprim"]
    off = np.concatenate([[0], np.cumsum(npr)])
    ao = np.concatenate([[0], np.cumsum([(int(l) + 1) * (int(l) + 2) // 2 for l in L])])
    LA, LB = int(L[a]), int(L[b])
    E = LA + LB
    mp = lambda x: m.mpf(float(x))
    A = [mp(x) for x in shells["center"][a]]
    B = [mp(x) for x in shells["center"][b]]
    AB = [A[d] - B[d] for d in range(3)]
    AB2 = m.fsum(x * x for x in AB)
    acc = {c: m.mpf(0) for la in range(LA, E + 1) for c in carts(la)}
    for i in range(int(npr[a])):
        al = mp(shells["expo"][off[a] + i])
        ca = mp(shells["coef"][off[a] + i]) * mp(shells["norm"][off[a] + i])
        for j in range(int(npr[b])):
            be = mp(shells["expo"][off[b] + j])
            cb = mp(shells["coef"][off[b] + j]) * mp(shells["norm"][off[b] + j])
            zeta = al + be
            iz = 1 / zeta
            K = ca * cb * m.exp(-al * be * iz * AB2)
            Pc = [(al * A[d] + be * B[d]) * iz for d in range(3)]
            PA = [Pc[d] - A[d] for d in range(3)]
            for c, Zc in enumerate(Z):
                C = [mp(x) for x in coords[c]]
                PC = [Pc[d] - C[d] for d in range(3)]
                T = zeta * m.fsum(x * x for x in PC)
                pre = -mp(Zc) * 2 * m.pi * iz * K
                V = {(0, 0, 0): [pre * m.hyp1f1(k + m.mpf(1) / 2, k + m.mpf(3) / 2, -T) / (2 * k + 1)
                                 for k in range(E + 1)]}
                for la in range(1, E + 1):
                    for t in carts(la):
                        d = 0 if t[0] else 1 if t[1] else 2
                        s = list(t)
                        s[d] -= 1
                        s = tuple(s)
                        x = [PA[d] * V[s][k] - PC[d] * V[s][k + 1] for k in range(E - la + 1)]
                        if s[d]:
                            g = list(s)
                            g[d] -= 1
                            g = tuple(g)
                            x = [x[k] + s[d] * iz / 2 * (V[g][k] - V[g][k + 1]) for k in range(E - la + 1)]
                        V[t] = x
                for t in acc:
                    acc[t] += V[t][0]
    H = {(t, (0, 0, 0)): acc[t] for t in acc}
    for lb in range(1, LB + 1):
        for la in range(LA, E - lb + 1):
            for t in carts(la):
                for u in carts(lb):
                    d = 0 if u[0] else 1 if u[1] else 2
                    um = list(u)
                    um[d] -= 1
                    tu = list(t)
                    tu[d] += 1
                    H[(t, u)] = H[(tuple(tu), tuple(um))] + AB[d] * H[(t, tuple(um))]
    out = {}
    for ia, t in enumerate(carts(LA)):
        for ib, u in enumerate(carts(LB)):
            nrm = 1 / m.sqrt(m.mpf(dfact(2 * t[0] - 1) * dfact(2 * t[1] - 1) * dfact(2 * t[2] - 1) *
                                   dfact(2 * u[0] - 1) * dfact(2 * u[1] - 1) * dfact(2 * u[2] - 1)))
            i, j = int(ao[a] + ia), int(ao[b] + ib)
            out[(min(i, j), max(i, j))] = m.nstr(H[(t, u)] * nrm, 25)
    return out


def main():
    shells, coords = inputs()
    L = shells["L"]
    jobs = []
    for s1 in range(NSHELL):
        for s2 in range(s1, NSHELL):
            jobs.append((s1, s2) if L[s1] >= L[s2] else (s2, s1))
    with mproc.get_context("spawn").Pool(os.cpu_count()) as pool:
        blocks = pool.map(pair_block, jobs)
    vals = {}
    for b in blocks:
        vals.update(b)
    nb = int(sum((int(l) + 1) * (int(l) + 2) // 2 for l in L))
    out = {"basis": {"random_shells": {"nshell": NSHELL, "lmax": 3, "seed": SEED, "box": BOX}},
           "nuclei": {"Z": Z, "seed": NUC_SEED, "coords_bohr": coords.tolist()},
           "nbasis": nb, "digits": 40,
           "V_upper": [[i, j, v] for (i, j), v in sorted(vals.items())]}
    with open(os.path.join(HERE, "onee_highprec.json"), "w") as f:
        json.dump(out, f, indent=0)
    print(f"wrote {len(vals)} elements of V (nbasis {nb})")


if __name__ == "__main__":
    main()
