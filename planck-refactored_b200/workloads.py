"""Seeded synthetic workloads with the shapes the benchmarks are quoted on.

  * water_cluster: (H2O)_n on a grid (4x4x2 for n = 32) at 3.0 Angstrom with
    seeded rigid rotations and +-0.2 Angstrom jitter of the experimental
    monomer (O (0,0,0.1173), H (0,+-0.7572,-0.4692) Angstrom);
  * alkane: all-trans CnH2n+2 with seeded noise;
  * alkane_conformer: seeded linear or branched CnH2n+2 conformers with
    bond, angle and torsion noise (the learned-guess training and
    evaluation sets);
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


def _unit(v):
    return v / np.linalg.norm(v)


def _rotate(v, axis, ang):
    """Rodrigues rotation of v about unit `axis` by `ang` radians."""
    return v * np.cos(ang) + np.cross(axis, v) * np.sin(ang) + axis * np.dot(axis, v) * (1.0 - np.cos(ang))


def alkane_conformer(nc, seed, branched=None, bond_noise=0.05, angle_noise_deg=5.0):
    """A seeded conformer of an acyclic alkane CnH2n+2, as [symbol, x, y, z]
    rows in Angstrom.

    Skeleton: linear when `branched` is False; otherwise every new carbon
    bonds to a random earlier carbon with fewer than three carbon neighbours
    (or four for a quaternary centre, with small probability), so both linear
    and branched isomers occur (branched=None draws the choice).  Geometry:
    C-C 1.53 and C-H 1.09 Angstrom each with uniform +-bond_noise, bond
    angles tetrahedral with uniform +-angle_noise_deg, and a random torsion
    about every C-C bond: the substituents take the three staggered
    positions (60, 180, 300 degrees from a substituent of the neighbouring
    carbon, all shifted by one uniform +-20 degrees) in random order, so each
    bond is a random trans/gauche rotamer.  Conformers whose non-bonded atoms
    come closer than 1.7 Angstrom (C-C), 1.4 (C-H) or 1.2 (H-H) are redrawn."""
    rng = np.random.default_rng(seed)
    if branched is None:
        branched = bool(rng.integers(0, 2)) and nc >= 4
    tet = np.deg2rad(109.4712)

    def too_close(x, sym, placed, skip):
        for k, (s2, y) in enumerate(placed):
            if k in skip:
                continue
            lim = 1.7 if sym == s2 == "C" else 1.2 if sym == s2 == "H" else 1.4
            if np.linalg.norm(x - y) < lim:
                return True
        return False

    for _attempt in range(100):
        parent = [-1]
        nbr = [[] for _ in range(nc)]
        for c in range(1, nc):
            if not branched:
                p = c - 1
            else:
                cands = [q for q in range(c) if len(nbr[q]) < (4 if rng.random() < 0.1 else 3)]
                p = int(rng.choice(cands)) if cands else c - 1
            parent.append(p)
            nbr[p].append(c)
            nbr[c].append(p)
        # placed atoms as (symbol, position); carbons keep their index c in slot[c]
        placed, slot, hydrogens = [("C", np.zeros(3))], {0: 0}, []
        dirs = {}
        order = [0]
        ok = True
        while order and ok:
            c = order.pop(0)
            children = [x for x in nbr[c] if x != parent[c]]
            for _try in range(40):
                if c == 0:
                    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
                    cand = [_unit(q @ v) for v in (np.array([1, 1, 1.0]), np.array([1, -1, -1.0]),
                                                   np.array([-1, 1, -1.0]), np.array([-1, -1, 1.0]))]
                    cand = [cand[k] for k in rng.permutation(4)]
                else:
                    pc = placed[slot[c]][1]
                    u = _unit(placed[slot[parent[c]]][1] - pc)   # towards the parent
                    # dihedrals are measured from another substituent of the parent
                    ref = next(d for d in dirs[parent[c]] if np.dot(d, -u) < 0.9)
                    r = _unit(ref - np.dot(ref, u) * u)
                    w = np.cross(u, r)
                    # staggered positions (60, 180, 300 degrees, all +-20) in
                    # random order: which substituent is trans or gauche is random
                    phi0 = np.deg2rad(60.0 + rng.uniform(-20.0, 20.0))
                    cand = []
                    for k in rng.permutation(3):
                        ang = tet + np.deg2rad(rng.uniform(-angle_noise_deg, angle_noise_deg))
                        phi = phi0 + 2 * np.pi * k / 3
                        cand.append(_unit(np.cos(ang) * u + np.sin(ang) * (np.cos(phi) * r + np.sin(phi) * w)))
                pc = placed[slot[c]][1]
                new = []
                for k, d in enumerate(cand):
                    sym = "C" if k < len(children) else "H"
                    new.append((sym, pc + d * ((1.53 if sym == "C" else 1.09) + rng.uniform(-bond_noise, bond_noise))))
                # new substituents against every placed atom except this carbon
                # and its parent (bonded or geminal by construction)
                skip = {slot[c]} | ({slot[parent[c]]} if c else set())
                if not any(too_close(x, sym, placed, skip) for sym, x in new):
                    break
            else:
                ok = False
                break
            dirs[c] = cand
            for k, (sym, x) in enumerate(new):
                placed.append((sym, x))
                if sym == "C":
                    slot[children[k]] = len(placed) - 1
                    order.append(children[k])
                else:
                    hydrogens.append(x)
        if ok:
            return [["C", *map(float, placed[slot[c]][1])] for c in range(nc)] + \
                   [["H", *map(float, x)] for x in hydrogens]
    raise RuntimeError(f"no clash-free conformer for C{nc} (seed {seed})")


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


def _normalize_many(L, expo, raw):
    """basis.normalize over many shells of one angular momentum and one
    contraction depth (rows of expo / raw), with the same operation order,
    so every row equals the scalar routine's result."""
    from . import basis
    pi = np.pi
    prefactor = 2.0 ** (2.0 * L + 1.5) / pi ** 1.5
    norm = np.sqrt(expo ** (L + 1.5) * prefactor)
    k = expo.shape[1]
    total = np.zeros(expo.shape[0])
    for j in range(k):
        for i in range(k):
            sij = (pi ** 1.5 / 2.0 ** L) / (expo[:, i] + expo[:, j]) ** (L + 1.5)
            total += raw[:, i] * raw[:, j] * norm[:, i] * norm[:, j] * sij
    del basis
    return raw * (1.0 / np.sqrt(total))[:, None], norm


def eri_class_quartets(la, lb, lc, ld, n, seed=0, box=10.0):
    """The ERI class microbenchmark's inputs for class (la lb|lc ld):
    n independent shell quartets, each of four fresh shells with centres
    uniform in a `box` Angstrom cube, contraction depth uniform in 1..6,
    exponents log-uniform in [0.05, 1e4] and coefficients uniform in (0, 1],
    normalised as the reference does (basis.cpp:39-75).  Shells 4t..4t+3
    belong to quartet t; pair 2t is (4t, 4t+1), pair 2t+1 is (4t+2, 4t+3).
    Requires la >= lb, lc >= ld and (la, lb) >= (lc, ld) in pair-class order.
    Returns (shells, pairs (2n x 2), quartets (n x 2))."""
    from . import basis
    rng = np.random.default_rng([seed, la, lb, lc, ld])
    ns = 4 * n
    Ls = np.tile(np.array([la, lb, lc, ld], dtype=np.int32), n)
    depth = rng.integers(1, 7, size=ns).astype(np.int32)
    center = rng.uniform(0.0, box, size=(ns, 3)) * basis.ANGSTROM_TO_BOHR
    E = np.exp(rng.uniform(np.log(0.05), np.log(1e4), size=(ns, 6)))
    # coefficients in (0, 1]: 1 - U[0, 1) never gives 0
    Rw = 1.0 - rng.uniform(0.0, 1.0, size=(ns, 6))
    coef = np.zeros((ns, 6))
    norm = np.zeros((ns, 6))
    for L in sorted(set(int(x) for x in (la, lb, lc, ld))):
        for k in range(1, 7):
            rows = np.nonzero((Ls == L) & (depth == k))[0]
            if len(rows) == 0:
                continue
            c, nm = _normalize_many(L, E[rows, :k], Rw[rows, :k])
            coef[rows, :k] = c
            norm[rows, :k] = nm
    mask = np.arange(6)[None, :] < depth[:, None]
    shells = {"L": Ls, "nprim": depth, "center": center, "expo": E[mask], "coef": coef[mask],
              "norm": norm[mask]}
    pairs = np.arange(ns, dtype=np.int32).reshape(-1, 2)
    quartets = np.arange(2 * n, dtype=np.int32).reshape(-1, 2)
    return shells, pairs, quartets
