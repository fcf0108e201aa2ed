"""Generate the Rys root/weight interpolation table used by the device kernels.

Rys quadrature for an ERI of total angular momentum L uses n = L//2 + 1 nodes
u_i = t_i^2 in (0, 1) and weights w_i of the measure

    d mu_T(u) = exp(-T u) u^(-1/2) / 2 du   on [0, 1],

whose moments are the Boys functions F_k(T) (the same measure the reference
builds from Boys moments in src/integrals/rys_roots.cpp:88-219).  That
construction (Hankel moments -> Stieltjes -> Jacobi eigensolve) is
ill-conditioned in double precision, so this script runs it once, offline, in
80-digit arithmetic (mpmath), and stores piecewise Chebyshev interpolants:

  * T in [0, TMAX[n]) : intervals of width H, degree DEG Chebyshev series for
    each of u_1..u_n, w_1..w_n (Clenshaw evaluation on the device);
  * T >= TMAX[n]      : the large-T limit, where the measure becomes the
    half-range Gaussian on [0, inf): u_i = x_i^2 / T, w_i = W_i / sqrt(T) with
    (x_i, W_i) the Gauss nodes/weights of exp(-x^2) on [0, inf).  TMAX[n] is
    the smallest tabulated T at which this limit agrees with the exact rule
    to better than 1e-15 relative (checked below).

Output: csrc/rys_table_data.inc (C initialisers, committed; regenerate with
`python gen_rys_table.py`).  The includer defines PFK_RYS_CONST_STORAGE and
PFK_RYS_TABLE_STORAGE (e.g. `static __constant__ const` and
`static __device__ const`) so every translation unit gets statically
initialised device copies.  Layout: per n, per coefficient degree k, per
root r, the (u_r, w_r) coefficient pair of every interval in turn.  The
device reads one (u, w) pair per 16-byte load, and the lanes of a warp,
whose T fall in different intervals, read neighbouring pairs of the same
(k, r) slab, which keeps each load within a few cache lines.  The script also prints the measured maximum
interpolation error at random T against fresh 80-digit evaluations.
"""
import multiprocessing as mproc
import os
import random
import sys

import mpmath

mp = mpmath.mp
mp.dps = 80

NMAX = 7                     # (ff|ff): L = 12 -> 7 roots
H = 2.0                      # interval width in T
DEG = 14                     # Chebyshev degree per interval
TMAX = [None, 40.0, 46.0, 60.0, 60.0, 70.0, 70.0, 80.0]


def boys(k, T):
    T = mp.mpf(T)
    if T == 0:
        return mp.mpf(1) / (2 * k + 1)
    return mp.hyp1f1(k + mp.mpf(1) / 2, k + mp.mpf(3) / 2, -T) / (2 * k + 1)


def gauss_from_moments(mom, n):
    """Gauss rule from 2n+1 moments (Stieltjes on monomial moments + eigsy)."""
    polys = [[mp.mpf(1) / mp.sqrt(mom[0])]]
    al, be = [], []

    def inner(a, b):
        s = mp.mpf(0)
        for i, x in enumerate(a):
            for j, y in enumerate(b):
                s += x * y * mom[i + j]
        return s

    for k in range(n):
        xp = [mp.mpf(0)] + polys[k]
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
        b = mp.sqrt(inner(q, q))
        be.append(b)
        polys.append([c / b for c in q])
    J = mp.matrix(n, n)
    for i in range(n):
        J[i, i] = al[i]
        if i + 1 < n:
            J[i, i + 1] = be[i]
            J[i + 1, i] = be[i]
    E, Q = mp.eigsy(J)
    idx = sorted(range(n), key=lambda i: E[i])
    return [E[i] for i in idx], [mom[0] * Q[0, i] ** 2 for i in idx]


def rys_exact(n, T):
    return gauss_from_moments([boys(k, T) for k in range(2 * n + 1)], n)


def half_hermite(n):
    """Nodes x_i^2 and weights of exp(-x^2) on [0, inf), as a rule in u = x^2."""
    mom = [mp.gamma(k + mp.mpf(1) / 2) / 2 for k in range(2 * n + 1)]
    return gauss_from_moments(mom, n)


def rys_asym(n, T):
    x2, W = half_hermite(n)
    T = mp.mpf(T)
    return [x / T for x in x2], [w / mp.sqrt(T) for w in W]


def _node_values(args):
    n, t = args
    u, w = rys_exact(n, mp.mpf(t))
    return [str(x) for x in u] + [str(x) for x in w]


def fit_interval(n, a, values_at_nodes):
    N = DEG + 1
    coefs = []
    for v in range(2 * n):
        vals = [mp.mpf(values_at_nodes[j][v]) for j in range(N)]
        row = []
        for k in range(N):
            s = mp.fsum(vals[j] * mp.cos(mp.pi * k * (j + mp.mpf(1) / 2) / N) for j in range(N))
            row.append(s / N if k == 0 else 2 * s / N)
        coefs.append([float(c) for c in row])
    return coefs


def cheb_eval(c, x):
    b1 = b2 = 0.0
    for k in range(len(c) - 1, 0, -1):
        b1, b2 = c[k] + 2 * x * b1 - b2, b1
    return c[0] + x * b1 - b2


def main():
    here = os.path.dirname(os.path.abspath(__file__))
    out_path = os.path.join(here, "csrc", "rys_table_data.inc")
    N = DEG + 1
    jobs = []
    layout = []
    for n in range(1, NMAX + 1):
        nint = int(round(TMAX[n] / H))
        layout.append(nint)
        for i in range(nint):
            a = i * H
            for j in range(N):
                t = a + H / 2 + H / 2 * mpmath.cos(mp.pi * (j + mp.mpf(1) / 2) / N)
                jobs.append((n, str(t)))
    with mproc.get_context("spawn").Pool(os.cpu_count()) as pool:
        vals = pool.map(_node_values, jobs, chunksize=8)
    tables = {}
    pos = 0
    for n in range(1, NMAX + 1):
        rows = []
        for i in range(layout[n - 1]):
            rows.append(fit_interval(n, i * H, vals[pos:pos + N]))
            pos += N
        tables[n] = rows

    # accuracy check at random T (interpolated and asymptotic ranges)
    rng = random.Random(12345)
    worst = {}
    for n in range(1, NMAX + 1):
        err = 0.0
        for _ in range(40):
            t = rng.uniform(0.0, TMAX[n] + 40.0)
            u, w = rys_exact(n, mp.mpf(t))
            if t < TMAX[n]:
                i = int(t / H)
                x = 2.0 * (t - i * H) / H - 1.0
                ua = [cheb_eval(tables[n][i][v], x) for v in range(n)]
                wa = [cheb_eval(tables[n][i][n + v], x) for v in range(n)]
            else:
                uu, ww = rys_asym(n, t)
                ua = [float(x) for x in uu]
                wa = [float(x) for x in ww]
            wsum = float(mp.fsum(w))
            for v in range(n):
                err = max(err, abs(ua[v] - float(u[v])) / float(u[v]),
                          abs(wa[v] - float(w[v])) / wsum)
        worst[n] = err
    x2, _ = None, None

    with open(out_path, "w") as f:
        f.write("// Generated by gen_rys_table.py (80-digit mpmath); do not edit.\n")
        f.write(f"// Chebyshev interval width {H}, degree {DEG}; n = 1..{NMAX}.\n")
        f.write("// Max relative error at 40 random T per n (roots; weights relative to sum w):\n")
        for n in range(1, NMAX + 1):
            f.write(f"//   n={n}: {worst[n]:.3e}\n")
        f.write(f"#define PFK_RYS_NMAX {NMAX}\n#define PFK_RYS_DEG {DEG}\n")
        f.write(f"#define PFK_RYS_H {H!r}\n")
        f.write("PFK_RYS_CONST_STORAGE double kRysTmax[PFK_RYS_NMAX + 1] = {0.0, " +
                ", ".join(repr(TMAX[n]) for n in range(1, NMAX + 1)) + "};\n")
        off = 0
        offs = [0]
        for n in range(1, NMAX + 1):
            offs.append(off)
            off += layout[n - 1] * 2 * n * N
        f.write("PFK_RYS_CONST_STORAGE int kRysOffset[PFK_RYS_NMAX + 1] = {" + ", ".join(str(o) for o in offs) + "};\n")
        f.write(f"#define PFK_RYS_TABLE_SIZE {off}\n")
        f.write("PFK_RYS_CONST_STORAGE int kRysNint[PFK_RYS_NMAX + 1] = {0, " +
                ", ".join(str(layout[n - 1]) for n in range(1, NMAX + 1)) + "};\n")
        f.write("PFK_RYS_TABLE_STORAGE double __align__(16) kRysCheb[PFK_RYS_TABLE_SIZE] = {\n")
        for n in range(1, NMAX + 1):
            f.write(f"// n = {n}: {N} coefficients x {n} roots x {layout[n-1]} intervals x (u, w)\n")
            for k in range(N):
                for r in range(n):
                    f.write(",".join(f"{tables[n][i][r][k]:.17g},{tables[n][i][n + r][k]:.17g}"
                                     for i in range(layout[n - 1])) + ",\n")
        f.write("};\n")
        # large-T limit constants: x_i^2 and W_i for each n
        f.write("PFK_RYS_CONST_STORAGE double kRysAsymU[PFK_RYS_NMAX + 1][PFK_RYS_NMAX] = {{0},\n")
        asym_w = []
        for n in range(1, NMAX + 1):
            x2, W = half_hermite(n)
            f.write("  {" + ", ".join(f"{float(x):.17g}" for x in x2) + "},\n")
            asym_w.append(W)
        f.write("};\n")
        f.write("PFK_RYS_CONST_STORAGE double kRysAsymW[PFK_RYS_NMAX + 1][PFK_RYS_NMAX] = {{0},\n")
        for W in asym_w:
            f.write("  {" + ", ".join(f"{float(x):.17g}" for x in W) + "},\n")
        f.write("};\n")
    for n in range(1, NMAX + 1):
        print(f"n={n} max rel err {worst[n]:.3e}")
    print("wrote", out_path, "size", off)


if __name__ == "__main__":
    sys.exit(main())
