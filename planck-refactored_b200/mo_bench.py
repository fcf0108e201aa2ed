"""Measure the device AO -> MO transform behind MP2 (pfk_mo_transform).

    python planck-refactored_b200/mo_bench.py [--waters 7] [--reps 3]

Workload: a seeded water cluster in 6-31G** (7 waters: 175 Cartesian
functions, the largest cluster under the 180-function limit of the dense
tensor), the MP2 block (C_occ C_vir | C_occ C_vir) of its converged RHF.
Reports, per phase, the device time from CUDA events inside the call: the
AO tensor (class kernels in tensor mode; 8-fold scatter of every screened
integral), the four quarter-transform GEMMs (FP64, cuBLAS) with their
FLOP rate against the FP64 FMA peak measured in the same run, and the copy
of the MO block to the host; and the RMP2 energy, summed on the host from
that block and on the device (pfk_rmp2_energy, the block never leaving HBM).
"""
import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def main():
    import importlib
    P = importlib.import_module("planck-refactored_b200")
    ap = argparse.ArgumentParser()
    ap.add_argument("--waters", type=int, default=7)
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()
    sysm = P.scf.System(P.workloads.water_cluster(a.waters, seed=2026), "6-31g**", P.basis.load_library())
    r = sysm.run()
    nb, no = sysm.H.shape[0], sysm.nocc
    nv = nb - no
    C = r["C"]
    eng = sysm.engine
    eng.mo_transform(C[:, :no], C[:, no:], C[:, :no], C[:, no:])   # warm-up (BLAS handle, kernels)
    times = []
    for _ in range(a.reps):
        eng.mo_transform(C[:, :no], C[:, no:], C[:, :no], C[:, no:])
        times.append(eng.mo_transform_times())
    t = min(times, key=lambda x: x[1])
    flops = 2.0 * (no * nb ** 4 + no * nv * nb ** 3 + no * nv * no * nb ** 2 + no * nv * no * nv * nb)
    fp64_peak, _ = P.measure_fma_peak(0)
    e2 = P.mp2.rmp2(eng, C, r["eps"], no)
    dev = []
    for _ in range(a.reps):
        e_dev = eng.rmp2_energy(C, r["eps"], no)
        dev.append(eng.mo_transform_times())
    td = min(dev, key=lambda x: x[1])
    sysm.close()
    out = {"workload": f"(H2O){a.waters} 6-31G** ({nb} bf), MP2 block (occ vir|occ vir), nocc {no}, nvir {nv}",
           "ao_tensor_ms": t[0], "ao_tensor_GBps_written": nb ** 4 * 8 / t[0] / 1e6,
           "gemm_ms": t[1], "gemm_flops": flops, "gemm_tflops": flops / t[1] / 1e9,
           "fp64_fma_peak_tflops": fp64_peak, "gemm_frac_of_fp64_peak": flops / t[1] / 1e9 / fp64_peak,
           "copy_out_ms": t[2], "mo_block_MB": no * nv * no * nv * 8 / 1e6,
           "rhf_energy": r["energy"], "rmp2_corr": e2,
           "rmp2_on_device": {"corr": e_dev, "ao_tensor_ms": td[0], "gemm_ms": td[1], "sum_ms": td[2],
                              "total_ms": sum(td), "block_read_GBps": 2 * no * nv * no * nv * 8 / td[2] / 1e6}}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
