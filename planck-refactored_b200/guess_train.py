"""Train and evaluate the learned initial guess on the GPU.

    python planck-refactored_b200/guess_train.py train --n 4096 --model guess_model.npz
    python planck-refactored_b200/guess_train.py evaluate --model guess_model.npz --n 512 --out eval.json

train: seed-generated alkane conformers (C1-C12, linear and branched, bond
+-0.05 Angstrom, angles +-5 degrees, random torsions; seeds 0..n-1) are
converged with the plain GPU RHF (6-31G*, or --basis cc-pvdz; scf.py on the
GPU Fock build); the
atom-pair features and local-frame density blocks of every converged
density train the five networks with Adam on the GPU (guess.train).

evaluate: held-out conformers of C8-C20 of uneven sizes (seeds from
1_000_000, disjoint from training) run as a batch of SCFs, once from the
default core-Hamiltonian guess and once through the guess hook
(guess.choose: learned density, kept only if its first-iteration energy is
not above the default's).  Reported: iterations and wall time to
convergence per guess, the fraction of learned guesses kept, and the
largest converged-energy difference between the two runs.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def _pkg():
    import importlib
    return importlib.import_module("planck-refactored_b200")


def conformer(i, lo, hi, seed_base):
    P = _pkg()
    rng = np.random.default_rng(seed_base + i)
    nc = int(rng.integers(lo, hi + 1))
    seed = seed_base + i
    for k in range(20):   # a skeleton with no clash-free conformer draws the next seed
        try:
            return nc, P.workloads.alkane_conformer(nc, seed + 7919 * k)
        except RuntimeError:
            continue
    raise RuntimeError(f"no conformer for C{nc}")


def generate(n, device=0, log=print, basis="6-31g*"):
    P = _pkg()
    G = P.guess
    lib = P.basis.load_library()
    samples = {t: ([], []) for t in G.TYPES}
    iters, t0 = [], time.perf_counter()
    for i in range(n):
        nc, atoms = conformer(i, 1, 12, 0)
        sysm = P.scf.System(atoms, basis, lib, device=device)
        r = sysm.run()
        if not r["converged"]:
            sysm.close()
            continue
        iters.append(r["iterations"])
        for t, (F, Y) in G.training_samples(sysm, r).items():
            if len(F):
                samples[t][0].append(F)
                samples[t][1].append(Y.astype(np.float32))
        sysm.close()
        if log and (i + 1) % 256 == 0:
            log(f"generated {i + 1}/{n} ({time.perf_counter() - t0:.0f} s)")
    out = {t: (np.concatenate(x) if x else np.zeros((0, G.NFEAT), np.float32),
               np.concatenate(y) if y else np.zeros((0, 0), np.float32)) for t, (x, y) in samples.items()}
    return out, {"molecules": len(iters), "mean_iterations_default": float(np.mean(iters)),
                 "seconds": time.perf_counter() - t0, "samples": {t: int(len(v[0])) for t, v in out.items()}}


def cmd_train(args):
    P = _pkg()
    G = P.guess
    samples, info = generate(args.n, args.device, basis=args.basis)
    print(json.dumps({"data": info}), flush=True)
    model = G.GuessModel(args.basis, device=args.device, seed=args.seed)
    t0 = time.perf_counter()
    losses = G.train(model, samples, epochs=args.epochs, lr=args.lr, batch=args.batch, seed=args.seed,
                     log=(lambda s: print(s, flush=True)) if args.verbose else None)
    model.save(args.model)
    print(json.dumps({"train_seconds": time.perf_counter() - t0, "final_loss": losses}), flush=True)


def evaluate(model_path, n, device=0, lo=8, hi=20, log=None, linalg="host", batch=1):
    """Default against learned guess on n held-out conformers.  batch > 1:
    the molecules go in groups of `batch` SCF runs at once (one context and
    one device SCF loop per molecule, host threads; linalg "gpu"), the
    learned guesses of a group predicted one after another (the network is
    shared); the times are then the groups' wall times."""
    P = _pkg()
    G = P.guess
    lib = P.basis.load_library()
    model = G.GuessModel.load(model_path, device=device)
    basis = model.basis_name
    if batch > 1:
        return _evaluate_batched(P, G, lib, model, basis, n, device, lo, hi, log, linalg, batch)
    rows = []
    for i in range(n):
        nc, atoms = conformer(i, lo, hi, 1_000_000)
        sysm = P.scf.System(atoms, basis, lib, device=device)
        t0 = time.perf_counter()
        r_d = sysm.run(linalg=linalg)
        t_d = time.perf_counter() - t0
        t0 = time.perf_counter()
        P0, G0, info = G.choose(model, sysm)
        r_l = sysm.run(P0=P0, G0=G0, linalg=linalg)
        t_l = time.perf_counter() - t0
        sysm.close()
        # builds: the learned path also pays the default guess's first build
        rows.append({"nc": nc, "nbasis": int(sysm.H.shape[0]), "it_default": r_d["iterations"],
                     "it_learned": r_l["iterations"], "builds_default": r_d["iterations"],
                     "builds_learned": r_l["iterations"] + 1, "t_default": t_d, "t_learned": t_l,
                     "accepted": info["accepted"], "dE": abs(r_l["energy"] - r_d["energy"]),
                     "converged": bool(r_d["converged"] and r_l["converged"])})
        if log and (i + 1) % 64 == 0:
            log(f"evaluated {i + 1}/{n}")
    model.close()
    return _summary(rows, n, basis, lo, hi)


def _summary(rows, n, basis, lo, hi, extra=None):
    it_d = np.array([r["it_default"] for r in rows])
    it_l = np.array([r["it_learned"] for r in rows])
    return {"molecules": n, "basis": basis, "sizes": f"C{lo}-C{hi}",
            "mean_iterations_default": float(it_d.mean()), "mean_iterations_learned": float(it_l.mean()),
            "iterations_ratio": float(it_l.sum() / it_d.sum()),
            "fock_builds_ratio": float(sum(r["builds_learned"] for r in rows) / sum(r["builds_default"] for r in rows)),
            "seconds_default": float(sum(r["t_default"] or 0.0 for r in rows)),
            "seconds_learned": float(sum(r["t_learned"] or 0.0 for r in rows)),
            "accepted_fraction": float(np.mean([r["accepted"] for r in rows])),
            "max_abs_dE_Eh": float(max(r["dE"] for r in rows)),
            "all_converged": bool(all(r["converged"] for r in rows)), **(extra or {}), "per_molecule": rows}


def _evaluate_batched(P, G, lib, model, basis, n, device, lo, hi, log, linalg, batch):
    from concurrent.futures import ThreadPoolExecutor
    rows, t_setup, t_def, t_lrn = [], 0.0, 0.0, 0.0
    with ThreadPoolExecutor(batch) as pool:
        for g0 in range(0, n, batch):
            idx = list(range(g0, min(n, g0 + batch)))
            t0 = time.perf_counter()
            mols = [conformer(i, lo, hi, 1_000_000) for i in idx]
            systems = [P.scf.System(atoms, basis, lib, device=device) for _, atoms in mols]
            t_setup += time.perf_counter() - t0
            t0 = time.perf_counter()
            r_d = list(pool.map(lambda s: s.run(linalg=linalg), systems))
            t_def += time.perf_counter() - t0
            t0 = time.perf_counter()
            picks = [G.choose(model, s) for s in systems]
            r_l = list(pool.map(lambda a: a[0].run(P0=a[1][0], G0=a[1][1], linalg=linalg), zip(systems, picks)))
            t_lrn += time.perf_counter() - t0
            for (nc, _), s, rd, rl, pk in zip(mols, systems, r_d, r_l, picks):
                rows.append({"nc": nc, "nbasis": int(s.H.shape[0]), "it_default": rd["iterations"],
                             "it_learned": rl["iterations"], "builds_default": rd["iterations"],
                             "builds_learned": rl["iterations"] + 1, "t_default": None, "t_learned": None,
                             "accepted": pk[2]["accepted"], "dE": abs(rl["energy"] - rd["energy"]),
                             "converged": bool(rd["converged"] and rl["converged"])})
                s.close()
            if log and len(rows) % 64 == 0:
                log(f"evaluated {len(rows)}/{n}")
    model.close()
    out = _summary(rows, n, basis, lo, hi, {"batch": batch, "linalg": linalg, "setup_seconds": t_setup})
    out["seconds_default"], out["seconds_learned"] = t_def, t_lrn
    return out


def cmd_evaluate(args):
    res = evaluate(args.model, args.n, args.device, log=lambda s: print(s, flush=True), linalg=args.linalg,
                   batch=args.batch)
    with open(args.out, "w") as f:
        json.dump(res, f)
    print(json.dumps({k: v for k, v in res.items() if k != "per_molecule"}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--n", type=int, default=4096)
    t.add_argument("--basis", default="6-31g*", choices=["6-31g*", "cc-pvdz"])
    t.add_argument("--model", default=os.path.join(HERE, "data", "guess_model_631gs.npz"))
    t.add_argument("--epochs", type=int, default=40)
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--batch", type=int, default=2048)
    t.add_argument("--seed", type=int, default=0)
    t.add_argument("--device", type=int, default=0)
    t.add_argument("--verbose", action="store_true")
    e = sub.add_parser("evaluate")
    e.add_argument("--model", default=os.path.join(HERE, "data", "guess_model_631gs.npz"))
    e.add_argument("--n", type=int, default=512)
    e.add_argument("--out", default="guess_eval.json")
    e.add_argument("--device", type=int, default=0)
    e.add_argument("--linalg", default="host", choices=["host", "gpu"],
                   help="SCF loop: numpy on the host, or pfk_scf_rhf on the device")
    e.add_argument("--batch", type=int, default=1, help="SCF runs at once (host threads, one context each)")
    args = ap.parse_args()
    {"train": cmd_train, "evaluate": cmd_evaluate}[args.cmd](args)


if __name__ == "__main__":
    main()
