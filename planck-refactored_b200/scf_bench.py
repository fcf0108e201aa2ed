"""Time to converged energy of whole RHF runs on the GPU builds.

    python planck-refactored_b200/scf_bench.py --molecule c40h82 [--out result.json]
    python planck-refactored_b200/scf_bench.py --molecule water32

Runs the same molecule several ways and reports, for each, the wall time to
convergence, the SCF iterations, the Fock-build share of that time, and the
converged energy:
  * fp64:        all-FP64 builds (the plain GPU path);
  * mixed:       FP32 for quartets whose Schwarz bound is below 1e-8;
  * mixed+dP:    mixed, with screened FP32 builds on the difference density
                 between full builds;
  * fp64+guess, mixed+guess (with --guess-model): the learned guess hook
                 (guess.choose) instead of the core-Hamiltonian guess.
Energies are compared with the FP64 run (the north star's |dE| <= 1e-6 Eh
for mixed precision).  Molecules: linear C40H82 (all-trans, C-C 1.53,
C-H 1.09 Angstrom, tetrahedral, +-0.03 Angstrom seeded noise) in cc-pVDZ
(1010 Cartesian functions; 970 spherical), and the 32-water cluster in
6-31G** (800).
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


def molecule(name):
    P = _pkg()
    if name == "c40h82":
        return P.workloads.alkane(40, seed=3, noise=0.03), "cc-pvdz"
    if name == "water32":
        return P.workloads.water_cluster(32, seed=2026), "6-31g**"
    raise ValueError(name)


class _Timed:
    """Wraps a FockEngine and accumulates the time of its builds."""

    def __init__(self, eng):
        self.eng, self.seconds, self.calls = eng, 0.0, 0

    def fock_rhf(self, P):
        t = time.perf_counter()
        G = self.eng.fock_rhf(P)
        self.seconds += time.perf_counter() - t
        self.calls += 1
        return G


def run(name, device=0, guess_model=None, runs=None, linalg="host"):
    P = _pkg()
    atoms, basis = molecule(name)
    lib = P.basis.load_library()
    out = {"molecule": name, "basis": basis}
    model = P.guess.GuessModel.load(guess_model, device=device) if guess_model else None
    if model is not None and model.basis_name != basis:
        raise ValueError(f"the guess model is for {model.basis_name}, the molecule is in {basis}")
    plan = [("fp64", "fp64", False, False), ("mixed", "mixed", False, False), ("mixed+dP", "mixed", True, False)]
    if model is not None:
        plan += [("fp64+guess", "fp64", False, True), ("mixed+guess", "mixed", False, True)]
    if runs:
        plan = [p for p in plan if p[0] in runs]
    if linalg == "device":   # the device loop has no difference-density builds
        plan = [p for p in plan if not p[2]]
    out["linalg"] = linalg
    ref = None
    for label, prec, incr, learned in plan:
        t0 = time.perf_counter()
        sysm = P.scf.System(atoms, basis, lib, device=device, precision=prec, fp32_bound=1e-8)
        t_setup = time.perf_counter() - t0
        full = _Timed(sysm.engine)
        incr_eng = _Timed(sysm.incremental_engine()) if incr else None
        t0 = time.perf_counter()
        P0 = G0 = None
        hook = None
        if learned:
            P0, G0, hook = P.guess.choose(model, sysm)
        if linalg == "device":
            r = P.scf.rhf_device(sysm.engine, sysm.H, sysm.S, sysm.enuc, sysm.nocc, P0=P0)
            full.seconds += r["build_seconds"]
        else:
            r = P.scf.rhf(full, sysm.H, sysm.S, sysm.enuc, sysm.nocc, P0=P0, G0=G0, incremental=incr_eng)
        t_scf = time.perf_counter() - t0
        out["nbasis"] = int(sysm.H.shape[0])
        sysm.close()
        if ref is None:
            ref = r["energy"]
        out[label] = {"energy": r["energy"], "dE_vs_fp64": r["energy"] - ref, "iterations": r["iterations"],
                      "converged": r["converged"], "seconds_to_convergence": t_scf, "setup_seconds": t_setup,
                      "fock_build_seconds": full.seconds + (incr_eng.seconds if incr_eng else 0.0),
                      "full_builds": full.calls, "difference_builds": incr_eng.calls if incr_eng else 0}
        if hook is not None:
            out[label]["guess"] = {"accepted": hook["accepted"], "predict_seconds": hook["predict_s"],
                                   "first_energy_learned": hook["E_first_learned"],
                                   "first_energy_default": hook["E_first_default"]}
    if model is not None:
        model.close()
    base = out.get("fp64", {}).get("seconds_to_convergence")
    if base:
        out["time_to_energy_vs_fp64"] = {k: base / v["seconds_to_convergence"] for k, v in out.items()
                                         if isinstance(v, dict) and "seconds_to_convergence" in v}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--molecule", default="c40h82", choices=["c40h82", "water32"])
    ap.add_argument("--out", default=None)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--guess-model", default=None, help="learned-guess model in the molecule's basis")
    ap.add_argument("--runs", default=None, help="comma-separated subset of fp64,mixed,mixed+dP,fp64+guess,mixed+guess")
    ap.add_argument("--linalg", default="host", choices=["host", "device"],
                    help="device: the SCF loop's diagonalisation and DIIS on the GPU (scf.rhf_device)")
    a = ap.parse_args()
    res = run(a.molecule, a.device, a.guess_model, a.runs.split(",") if a.runs else None, a.linalg)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
