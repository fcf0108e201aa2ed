"""Seeded synthetic workloads with the shapes the benchmarks are quoted on.

  * water_cluster: (H2O)_n on a grid (4x4x2 for n = 32) at 3.0 Angstrom with
    seeded rigid rotations and +-0.2 Angstrom jitter of the experimental
    monomer (O (0,0,0.1173), H (0,+-0.7572,-0.4692) Angstrom);
  * alkane: all-trans CnH2n+2 with seeded noise;
  * random_shells: shells drawn like the ERI class microbenchmark
    (exponents log-uniform in [0.05, 1e4], contraction depth 1..6,
    coefficients uniform in (0, 1], reference normalisation).
No public dataset is involved; these stand in for the benchmark molecules.
"""
import numpy as np

WATER = [["O", 0.0, 0.0, 0.1173], ["H", 0.0, 0.7572, -0.4692], ["H", 0.0, -0.7572, -0.4692]]


def water_cluster(n, seed=1, spacing=3.0, jitter=0.2):
    """n waters on a grid (4x4x2 for n=32) at `spacing` Angstrom with seeded
    rigid rotations and +-jitter Angstrom displacements of the monomer."""
    rng = np.random.default_rng(seed)
    mono = np.array([a[1:] for a in WATER])
    mono = mono - mono[0]
    dims = (4, 4, 2) if n == 32 else (int(np.ceil(n ** (1 / 3))),) * 3
    atoms = []
    k = 0
    for ix in range(dims[0]):
        for iy in range(dims[1]):
            for iz in range(dims[2]):
                if k == n:
                    break
                q = rng.normal(size=4)
                q /= np.linalg.norm(q)
                a, b, c, d = q
                R = np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                              [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                              [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])
                shift = np.array([ix, iy, iz]) * spacing + rng.uniform(-jitter, jitter, 3)
                for sym, xyz in zip(["O", "H", "H"], mono @ R.T + shift):
                    atoms.append([sym, *map(float, xyz)])
                k += 1
    return atoms


def alkane(nc, seed=3, noise=0.03):
    """All-trans linear CnH2n+2 (C-C 1.53, C-H 1.09 Angstrom, tetrahedral) with
    seeded +-noise Angstrom displacements."""
    rng = np.random.default_rng(seed)
    cc, ch = 1.53, 1.09
    half = np.deg2rad(109.471 / 2)
    dx, dy = cc * np.sin(half), cc * np.cos(half)
    carbons = [np.array([i * dx, (i % 2) * dy, 0.0]) for i in range(nc)]
    atoms = [["C", *c] for c in carbons]
    for i, c in enumerate(carbons):
        up = 1.0 if i % 2 else -1.0
        # two H in the plane perpendicular to the chain
        for s in (1.0, -1.0):
            v = np.array([0.0, up * np.cos(np.deg2rad(54.75)), s * np.sin(np.deg2rad(54.75))])
            atoms.append(["H", *(c + ch * v / np.linalg.norm(v))])
    atoms.append(["H", *(carbons[0] + ch * np.array([-np.sin(half), -np.cos(half), 0.0]))])
    sgn = 1.0 if (nc - 1) % 2 else -1.0
    atoms.append(["H", *(carbons[-1] + ch * np.array([np.sin(half), sgn * np.cos(half), 0.0]))])
    out = []
    for a in atoms:
        out.append([a[0], *(np.array(a[1:], dtype=float) + rng.uniform(-noise, noise, 3))])
    return out


def random_shells(nshell, lmax=3, seed=11, box=10.0):
    """Random shells like the ERI class microbenchmark: centres uniform in a
    `box` Angstrom cube, exponents log-uniform in [0.05, 1e4], contraction
    depth 1..6, coefficients uniform in (0, 1], reference normalisation."""
    from . import basis
    rng = np.random.default_rng(seed)
    L, nprim, center, expo, coef, norm = [], [], [], [], [], []
    for s in range(nshell):
        l = int(rng.integers(0, lmax + 1))
        k = int(rng.integers(1, 7))
        e = np.exp(rng.uniform(np.log(0.05), np.log(1e4), k))
        c_raw = rng.uniform(1e-6, 1.0, k)
        c, nrm = basis.normalize(l, e, c_raw)
        L.append(l)
        nprim.append(k)
        center.append(rng.uniform(0, box, 3) * basis.ANGSTROM_TO_BOHR)
        expo.extend(e)
        coef.extend(c)
        norm.extend(nrm)
    return {"L": np.array(L, dtype=np.int32), "nprim": np.array(nprim, dtype=np.int32),
            "center": np.array(center), "expo": np.array(expo), "coef": np.array(coef), "norm": np.array(norm)}
