"""Learned initial guess: atom-pair density blocks from local geometry.

The SCF's guess hook (Planck selects its guess in scf.cpp:206-240; a density
supplied from outside enters like its ReadDensity guess, scf.cpp:213-216)
gets a density built here instead of the default core-Hamiltonian one:

  1. every atom pair (A, B) closer than PAIR_CUTOFF gets a local frame: z
     along A->B (for A = B, towards the nearest neighbour), x towards the
     nearest other atom, orthogonalised;
  2. invariant features of the pair's surroundings are computed in that
     frame: radial Gaussians times (1, x/r, y/r, z/r) of every neighbour,
     per element and per pair centre, with a smooth cutoff, and Gaussians
     of the A-B distance;
  3. one network per pair type (C-C, C-H, H-H, C-C on-site, H-H on-site)
     predicts the block of the density in the local frame, standardised
     per output; the networks are the library's BF16 tensor-core MLP
     (pfk_mlp_*) trained on the GPU (train());
  4. the blocks are rotated back to the molecule's frame (Cartesian shells
     transform by D(R): s -> 1, p -> R, d -> the symmetric product of R with
     the component norms), assembled, and projected to an idempotent density
     with the right electron count: the nocc leading eigenvectors of
     S^1/2 P S^1/2 / 2;
  5. choose() keeps it only if its first-iteration energy is not above the
     default guess's; the SCF then runs to convergence with the plain
     method, so the guess changes the iteration count, never the answer.

Training data are converged densities of seed-generated alkane conformers
from the plain GPU SCF (scf.py on the GPU Fock build).  A model is tied to
the basis set it was trained in (H and C; 6-31G* and cc-pVDZ are shipped).
"""
import json
import time

import numpy as np

from .basis import ANGSTROM_TO_BOHR

PAIR_CUTOFF = 5.5                 # Angstrom; blocks of farther pairs are zero
ENV_CUTOFF = 4.5                  # Angstrom; neighbours entering the features
RAD_MU = np.linspace(0.9, 4.0, 6)
RAD_SIGMA = 0.35
DIST_MU = np.linspace(0.0, 5.5, 8)
DIST_SIGMA = 0.4
ELEMENTS = ("H", "C")
NFEAT = 112                       # 2 centres x 2 elements x 6 radial x 4 angular + 8 + 1, padded to 112
TYPES = ("CC", "CH", "HH", "C", "H")
HIDDEN = 256


def _pad8(n):
    return (n + 7) // 8 * 8


# ---------------------------------------------------------------------------
# Basis layout and the rotation of Cartesian shells
# ---------------------------------------------------------------------------
def atom_layout(mol, shells):
    """Per atom: (first AO, [L of its shells]); shells are grouped by atom in
    atom order (the reference's basis order)."""
    centers = np.asarray(shells["center"]).reshape(-1, 3)
    Ls = np.asarray(shells["L"])
    out, s, ao = [], 0, 0
    for a in range(len(mol.symbols)):
        first = ao
        lst = []
        while s < len(Ls) and np.allclose(centers[s], mol.coords[a]):
            lst.append(int(Ls[s]))
            ao += (Ls[s] + 1) * (Ls[s] + 2) // 2
            s += 1
        out.append((first, lst))
    assert s == len(Ls), "shells are not grouped by atom in atom order"
    return out


def _cart(L):
    return [(lx, ly, L - lx - ly) for lx in range(L, -1, -1) for ly in range(L - lx, -1, -1)]


def _dfact(n):
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def _cnorm(e):
    return 1.0 / np.sqrt(_dfact(2 * e[0] - 1) * _dfact(2 * e[1] - 1) * _dfact(2 * e[2] - 1))


def shell_rotation(L, R):
    """D (ncart x ncart, batched over R of shape (..., 3, 3)) with
    chi_local = D chi_global for a Cartesian shell of angular momentum L,
    where local coordinates are R (x - centre)."""
    R = np.asarray(R)
    if L == 0:
        return np.ones(R.shape[:-2] + (1, 1))
    comps = _cart(L)
    index = {c: i for i, c in enumerate(comps)}
    D = np.zeros(R.shape[:-2] + (len(comps), len(comps)))
    for a, ea in enumerate(comps):
        axes = [0] * ea[0] + [1] * ea[1] + [2] * ea[2]      # local axes multiplied
        # expand prod_k (sum_c R[axes[k], c] x_c) into global monomials
        terms = {(0, 0, 0): np.ones(R.shape[:-2])}
        for ax in axes:
            nxt = {}
            for e, coef in terms.items():
                for c in range(3):
                    e2 = tuple(e[i] + (1 if i == c else 0) for i in range(3))
                    nxt[e2] = nxt.get(e2, 0.0) + coef * R[..., ax, c]
            terms = nxt
        for e, coef in terms.items():
            D[..., a, index[e]] = coef * (_cnorm(ea) / _cnorm(e))
    return D


def atom_rotation(Ls, R):
    """Block-diagonal D of one atom's shells, batched over R."""
    blocks = [shell_rotation(L, R) for L in Ls]
    n = sum(b.shape[-1] for b in blocks)
    D = np.zeros(R.shape[:-2] + (n, n))
    o = 0
    for b in blocks:
        k = b.shape[-1]
        D[..., o:o + k, o:o + k] = b
        o += k
    return D


# ---------------------------------------------------------------------------
# Pairs, frames and features (positions in Angstrom)
# ---------------------------------------------------------------------------
def molecule_pairs(symbols, pos):
    """{type: int array (npair, 2)}: C-C (A < B), C-H (A carbon), H-H (A < B),
    and the on-site pairs C and H, for atom pairs closer than PAIR_CUTOFF."""
    d = np.linalg.norm(pos[:, None] - pos[None], axis=-1)
    out = {t: [] for t in TYPES}
    n = len(symbols)
    for a in range(n):
        out[symbols[a]].append((a, a))
        for b in range(a + 1, n):
            if d[a, b] >= PAIR_CUTOFF:
                continue
            sa, sb = symbols[a], symbols[b]
            if sa == sb:
                out[sa + sb].append((a, b))
            elif sa == "C":
                out["CH"].append((a, b))
            else:
                out["CH"].append((b, a))
    return {t: np.array(v, dtype=np.int64).reshape(-1, 2) for t, v in out.items()}


def frames(pos, pairs):
    """Rotation matrices (npair, 3, 3) whose rows are the local x, y, z axes."""
    d = np.linalg.norm(pos[:, None] - pos[None], axis=-1)
    Rs = np.zeros((len(pairs), 3, 3))
    for k, (a, b) in enumerate(pairs):
        order = [x for x in np.argsort(d[a]) if x != a]
        if a != b:
            ez = pos[b] - pos[a]
            cands = [x for x in order if x != b] + [x for x in np.argsort(d[b]) if x not in (a, b)]
        else:
            ez = pos[order[0]] - pos[a] if order else np.array([0.0, 0.0, 1.0])
            cands = order[1:]
        ez = ez / np.linalg.norm(ez)
        ex = None
        for x in cands:
            v = pos[x] - pos[a]
            v = v - np.dot(v, ez) * ez
            if np.linalg.norm(v) > 0.3:
                ex = v / np.linalg.norm(v)
                break
        if ex is None:   # linear arrangement: any perpendicular
            t = np.array([1.0, 0.0, 0.0]) if abs(ez[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
            ex = t - np.dot(t, ez) * ez
            ex /= np.linalg.norm(ex)
        Rs[k] = np.stack([ex, np.cross(ez, ex), ez])
    return Rs


def features(symbols, pos, pairs, Rs):
    """(npair, NFEAT) float32 features in each pair's frame."""
    elem = np.array([ELEMENTS.index(s) for s in symbols])
    npair, n = len(pairs), len(pos)
    F = np.zeros((npair, NFEAT), dtype=np.float64)
    if npair == 0:
        return F.astype(np.float32)
    A, B = pairs[:, 0], pairs[:, 1]
    col = 0
    for centre in (A, B):
        rel = pos[None, :, :] - pos[centre][:, None, :]                 # (npair, n, 3)
        v = np.einsum("pij,pnj->pni", Rs, rel)                          # in the frame
        r = np.linalg.norm(v, axis=-1)
        mask = (r < ENV_CUTOFF) & (np.arange(n)[None] != A[:, None]) & (np.arange(n)[None] != B[:, None])
        fc = np.where(mask, 0.5 * (np.cos(np.pi * np.minimum(r, ENV_CUTOFF) / ENV_CUTOFF) + 1.0), 0.0)
        rs = np.where(r > 1e-8, r, 1.0)
        ang = np.concatenate([np.ones_like(r)[..., None], v / rs[..., None]], axis=-1)   # (npair, n, 4)
        rad = np.exp(-((r[..., None] - RAD_MU) ** 2) / (2 * RAD_SIGMA ** 2)) * fc[..., None]   # (npair, n, 6)
        for e in range(2):
            sel = (elem == e)[None, :, None]
            blk = np.einsum("pnj,pna->pja", rad * sel, ang)               # (npair, 6, 4)
            F[:, col:col + 24] = blk.reshape(npair, 24)
            col += 24
    rab = np.linalg.norm(pos[B] - pos[A], axis=-1)
    F[:, col:col + 8] = np.exp(-((rab[:, None] - DIST_MU) ** 2) / (2 * DIST_SIGMA ** 2))
    col += 8
    F[:, col] = 1.0
    return F.astype(np.float32)


def _block_index(layout, a):
    first, Ls = layout[a]
    return first, first + sum((L + 1) * (L + 2) // 2 for L in Ls)


def local_blocks(P, layout, pairs, Rs):
    """Density blocks of the pairs in their local frames, flattened (npair, nA*nB):
    P_loc = D(R^T)^T P_AB D(R^T)."""
    if len(pairs) == 0:
        return np.zeros((0, 0))
    LA, LB = layout[pairs[0, 0]][1], layout[pairs[0, 1]][1]
    DA, DB = atom_rotation(LA, np.swapaxes(Rs, 1, 2)), atom_rotation(LB, np.swapaxes(Rs, 1, 2))
    blocks = []
    for k, (a, b) in enumerate(pairs):
        a0, a1 = _block_index(layout, a)
        b0, b1 = _block_index(layout, b)
        blocks.append((DA[k].T @ P[a0:a1, b0:b1] @ DB[k]).ravel())
    return np.array(blocks)


def assemble(nb, layout, pair_sets, blocks):
    """Global density from local-frame blocks: P_AB = D(R)^T P_loc D(R)."""
    P = np.zeros((nb, nb))
    for t, (pairs, Rs) in pair_sets.items():
        if len(pairs) == 0:
            continue
        LA, LB = layout[pairs[0, 0]][1], layout[pairs[0, 1]][1]
        DA, DB = atom_rotation(LA, Rs), atom_rotation(LB, Rs)
        nA, nB = DA.shape[-1], DB.shape[-1]
        for k, (a, b) in enumerate(pairs):
            a0, a1 = _block_index(layout, a)
            b0, b1 = _block_index(layout, b)
            blk = DA[k].T @ blocks[t][k, :nA * nB].reshape(nA, nB) @ DB[k]
            P[a0:a1, b0:b1] = blk
            if a != b:
                P[b0:b1, a0:a1] = blk.T
    return 0.5 * (P + P.T)


def purify(P, S, nocc):
    """Idempotent density with trace nocc*2: the nocc leading eigenvectors of
    S^1/2 P S^1/2 / 2, mapped back with S^-1/2."""
    s, U = np.linalg.eigh(S)
    Sh = (U * np.sqrt(s)) @ U.T
    Smh = (U / np.sqrt(s)) @ U.T
    w, V = np.linalg.eigh(0.5 * Sh @ P @ Sh)
    C = Smh @ V[:, ::-1][:, :nocc]
    return 2.0 * C @ C.T


# ---------------------------------------------------------------------------
# Model
# ---------------------------------------------------------------------------
def element_nao(basis_name, library=None):
    """Cartesian functions per element (H, C) in a basis set."""
    from .basis import load_library
    lib = library or load_library()
    return {e: int(sum((int(L) + 1) * (int(L) + 2) // 2 for L, _ in lib[basis_name][e])) for e in ("H", "C")}


class GuessModel:
    """Five networks (one per pair type) and their output standardisation."""

    def __init__(self, basis_name="6-31g*", nao=None, device=0, max_batch=8192, seed=0, params=None, stats=None):
        from .mlp import MLP
        self.basis_name, self.device = basis_name, device
        self.nao = nao or element_nao(basis_name)
        self.out = {"CC": self.nao["C"] ** 2, "CH": self.nao["C"] * self.nao["H"], "HH": self.nao["H"] ** 2,
                    "C": self.nao["C"] ** 2, "H": self.nao["H"] ** 2}
        self.nets, self.stats = {}, stats or {}
        for i, t in enumerate(TYPES):
            dims = [NFEAT, HIDDEN, HIDDEN, _pad8(self.out[t])]
            self.nets[t] = MLP(dims, max_batch, device=device, seed=seed + i,
                               params=None if params is None else params[t])

    def close(self):
        for n in self.nets.values():
            n.close()

    def save(self, path):
        arrays = {f"params_{t}": self.nets[t].params() for t in TYPES}
        for t in TYPES:
            arrays[f"mean_{t}"], arrays[f"std_{t}"] = self.stats[t]
        meta = {"basis": self.basis_name, "nao": self.nao, "pair_cutoff": PAIR_CUTOFF, "env_cutoff": ENV_CUTOFF,
                "nfeat": NFEAT, "hidden": HIDDEN}
        np.savez_compressed(path, meta=json.dumps(meta), **arrays)

    @classmethod
    def load(cls, path, device=0, max_batch=8192):
        z = np.load(path)
        meta = json.loads(str(z["meta"]))
        params = {t: z[f"params_{t}"] for t in TYPES}
        stats = {t: (z[f"mean_{t}"], z[f"std_{t}"]) for t in TYPES}
        return cls(meta["basis"], meta["nao"], device=device, max_batch=max_batch, params=params, stats=stats)

    def predict_blocks(self, feats):
        """{type: (npair, out) float64} local-frame blocks from features."""
        import torch
        out = {}
        for t in TYPES:
            X = feats[t]
            if len(X) == 0:
                out[t] = np.zeros((0, self.out[t]))
                continue
            ys = []
            for s in range(0, len(X), self.nets[t].max_batch):
                Xd = torch.from_numpy(np.ascontiguousarray(X[s:s + self.nets[t].max_batch])).to(f"cuda:{self.device}")
                ys.append(self.nets[t].forward(Xd).cpu().numpy()[:, :self.out[t]])
            mean, std = self.stats[t]
            out[t] = np.concatenate(ys).astype(np.float64) * std + mean
        return out


def pair_data(mol):
    """(pairs, frames, features) per type for a molecule (positions in Angstrom)."""
    pos = mol.coords / ANGSTROM_TO_BOHR
    sets = molecule_pairs(mol.symbols, pos)
    out = {}
    for t, pairs in sets.items():
        Rs = frames(pos, pairs) if len(pairs) else np.zeros((0, 3, 3))
        out[t] = (pairs, Rs, features(mol.symbols, pos, pairs, Rs))
    return out


def predict_density(model, system):
    """Purified learned density for an scf.System."""
    data = pair_data(system.mol)
    blocks = model.predict_blocks({t: v[2] for t, v in data.items()})
    layout = atom_layout(system.mol, system.shells)
    P = assemble(system.H.shape[0], layout, {t: (v[0], v[1]) for t, v in data.items()}, blocks)
    return purify(P, system.S, system.nocc)


def choose(model, system):
    """The guess hook: (P0, G0, info).  Builds the learned density and the
    default core-Hamiltonian one, runs one Fock build on each, and keeps the
    learned one only if its energy is not above the default's (the first
    iteration's energy); G0 is that build, reused as the SCF's first."""
    from .scf import first_energy, hcore_density, orthogonaliser
    t0 = time.perf_counter()
    P_l = predict_density(model, system)
    t_pred = time.perf_counter() - t0
    P_d = hcore_density(system.H, orthogonaliser(system.S), system.nocc)
    G_l = system.engine.fock_rhf(P_l)
    G_d = system.engine.fock_rhf(P_d)
    E_l = first_energy(system.H, system.enuc, P_l, G_l)
    E_d = first_energy(system.H, system.enuc, P_d, G_d)
    accepted = E_l <= E_d
    info = {"accepted": bool(accepted), "E_first_learned": E_l, "E_first_default": E_d,
            "predict_s": t_pred}
    return (P_l, G_l, info) if accepted else (P_d, G_d, info)


# ---------------------------------------------------------------------------
# Training data and training
# ---------------------------------------------------------------------------
def training_samples(system, result):
    """Features and local-frame target blocks of a converged SCF."""
    data = pair_data(system.mol)
    layout = atom_layout(system.mol, system.shells)
    out = {}
    for t, (pairs, Rs, F) in data.items():
        out[t] = (F, local_blocks(result["P"], layout, pairs, Rs) if len(pairs) else np.zeros((0, 0)))
    return out


def train(model, samples, epochs=30, lr=1e-3, batch=2048, seed=0, log=None):
    """Fit every network on {type: (X (n, NFEAT), Y (n, out))} with Adam on
    the GPU (pfk_mlp_train_step); targets are standardised per output.
    Returns the final mean loss per type."""
    import torch
    rng = np.random.default_rng(seed)
    losses = {}
    for t in TYPES:
        X, Y = samples[t]
        if len(X) == 0:
            continue
        out = model.out[t]
        mean, std = Y.mean(axis=0), Y.std(axis=0) + 1e-6
        model.stats[t] = (mean, std)
        Yp = np.zeros((len(Y), _pad8(out)), dtype=np.float32)
        Yp[:, :out] = (Y - mean) / std
        dev = f"cuda:{model.device}"
        Xd = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float32)).to(dev)
        Yd = torch.from_numpy(Yp).to(dev)
        net = model.nets[t]
        bs = min(batch, net.max_batch)
        steps_per_epoch = max(1, len(X) // bs)
        total = epochs * steps_per_epoch
        step = 0
        for ep in range(epochs):
            perm = torch.from_numpy(rng.permutation(len(X))).to(dev)
            acc = 0.0
            for s in range(steps_per_epoch):
                idx = perm[s * bs:(s + 1) * bs]
                xb, yb = Xd.index_select(0, idx).contiguous(), Yd.index_select(0, idx).contiguous()
                cur = lr * 0.5 * (1.0 + np.cos(np.pi * step / total))    # cosine decay
                acc += net.train_step(xb, yb, cur)
                step += 1
            losses[t] = acc / steps_per_epoch
            if log:
                log(f"{t} epoch {ep + 1}/{epochs} loss {losses[t]:.5f}")
    return losses
