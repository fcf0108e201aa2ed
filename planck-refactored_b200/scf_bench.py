"""Time to converged energy of whole RHF runs on the GPU builds.

    python planck-refactored_b200/scf_bench.py --molecule c40h82 [--out result.json]
    python planck-refactored_b200/scf_bench.py --molecule water32

Runs the same molecule three ways and reports, for each, the wall time to
convergence, the SCF iterations, the Fock-build share of that time, and the
converged energy:
  * fp64:        all-FP64 builds (the plain GPU path);
  * mixed:       FP32 for quartets whose Schwarz bound is below 1e-8;
  * mixed+dP:    mixed, with FP32 builds on the difference density between
                 full builds every 8 iterations.
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


def run(name, device=0):
    P = _pkg()
    atoms, basis = molecule(name)
    lib = P.basis.load_library()
    out = {"molecule": name, "basis": basis}
    ref = None
    for label, prec, incr in (("fp64", "fp64", False), ("mixed", "mixed", False), ("mixed+dP", "mixed", True)):
        t0 = time.perf_counter()
        sysm = P.scf.System(atoms, basis, lib, device=device, precision=prec, fp32_bound=1e-8)
        t_setup = time.perf_counter() - t0
        full = _Timed(sysm.engine)
        incr_eng = _Timed(sysm.incremental_engine()) if incr else None
        t0 = time.perf_counter()
        r = P.scf.rhf(full, sysm.H, sysm.S, sysm.enuc, sysm.nocc, incremental=incr_eng)
        t_scf = time.perf_counter() - t0
        out["nbasis"] = int(sysm.H.shape[0])
        sysm.close()
        if ref is None:
            ref = r["energy"]
        out[label] = {"energy": r["energy"], "dE_vs_fp64": r["energy"] - ref, "iterations": r["iterations"],
                      "converged": r["converged"], "seconds_to_convergence": t_scf, "setup_seconds": t_setup,
                      "fock_build_seconds": full.seconds + (incr_eng.seconds if incr_eng else 0.0),
                      "full_builds": full.calls, "difference_builds": incr_eng.calls if incr_eng else 0}
    out["speedup_mixed+dP_vs_fp64"] = out["fp64"]["seconds_to_convergence"] / out["mixed+dP"]["seconds_to_convergence"]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--molecule", default="c40h82", choices=["c40h82", "water32"])
    ap.add_argument("--out", default=None)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args()
    res = run(a.molecule, a.device)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
