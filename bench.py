"""Benchmark: direct-SCF Fock builds of a 32-water cluster (6-31G**, 800 basis
functions) on B200, one process per GPU.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision fp64|mixed] [--engine auto|os|rys]

A step is one Fock build G = J(P) - K(P)/2 of (H2O)32 / 6-31G** (Cartesian,
800 functions), tol_eri 1e-10, on a seeded symmetric density (the build's work
does not depend on the density values).  By default the build is the mixed-
precision one of the benchmark configuration (FP32 arithmetic for quartets
whose Schwarz bound is below 1e-8, FP64 roots, weights and accumulation); the
all-FP64 build is timed beside it and its speed-up and G / energy error are
reported.  The engine is `auto`: the per-class kernel choice (Rys, Obara-
Saika, or Obara-Saika at higher occupancy) is measured by the library's
autotuner on this molecule's lists during setup.  With N > 1 (torchrun, NCCL)
every rank evaluates every N-th
quartet of each class's screened quartet list and the partial G are summed
with one all-reduce per build:
strong scaling of one build.

Printed (rank 0, one JSON line): Fock builds/s of the whole job (device-timed
with CUDA events on the launch stream, max over ranks, inputs resident), the
screened shell quartets/s, an end-to-end figure through the C ABI with host
buffers, the roofline of the dominant class kernel and of the whole build
against the FP64 FMA peak measured in the same run, and a CPU baseline: the
oracle's streaming restatement of the reference's integral path on the host
cores, timed on a bounded sample of pair rows and extrapolated.

--impl reference times that CPU path alone (the reference's own direct path
needs an nb^4 = 3.3 TB tensor at 800 functions and cannot run; the streaming
restatement computes the same integrals without it).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

WORKLOAD = "(H2O)32 6-31G** Cartesian, 800 bf, RHF G=J-K/2, tol_eri 1e-10"
SEED = 2026


def _pfk():
    import importlib
    return importlib.import_module("planck-refactored_b200")


def build_shells(waters=32):
    P = _pfk()
    atoms = P.workloads.water_cluster(waters, seed=SEED)
    mol, shells = P.shells_for(atoms, "6-31g**", P.basis.load_library())
    return atoms, mol, shells


def density(nb, seed=SEED):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(nb, nb)) * 0.05
    return A + A.T


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
# CPU path: the oracle's streaming restatement of the reference's direct build
# ---------------------------------------------------------------------------
def cpu_fock_rate(shells, budget_s=12.0, seed=SEED):
    """Fock builds/s of the reference's direct path on the host cores,
    extrapolated from a stratified sample of bra AO-pair rows.  Per build the
    reference recomputes the Schwarz table serially (os.cpp:1447, timed in
    full here) and evaluates every screened canonical AO quartet with its
    per-component OS code (os.cpp:1458-1507, restated); its nb^4 tensor
    scatter and O(nb^4) digestion (os.cpp:1450, 1514-1520) cannot run at 800
    functions (3.3 TB) and are replaced by the streaming digestion, which only
    makes the baseline faster."""
    import oracle
    ob = oracle.Basis(shells)
    nb, npairs = ob.nbasis, ob.npairs
    t0 = time.perf_counter()
    Q = ob.schwarz(oracle.OS)
    t_schwarz = time.perf_counter() - t0
    Pm = density(nb)
    rng = np.random.default_rng(seed)

    def sample(strata):
        edges = np.linspace(0, npairs, strata + 1).astype(np.int64)
        rows = np.array([rng.integers(edges[i], max(edges[i] + 1, edges[i + 1])) for i in range(strata)],
                        dtype=np.int32)
        t = time.perf_counter()
        _, _, n = ob.jk_direct_rows(Pm, [Pm], rows, 1e-10, oracle.OS, Q=Q)
        dt = time.perf_counter() - t
        return dt * npairs / strata, n * npairs / strata, dt, n, strata

    est, nq, dt, n, s = sample(32)
    strata = int(min(npairs, max(32, 32 * (budget_s - dt) / max(dt, 1e-3))))
    if strata > 32 and dt < budget_s:
        est, nq, dt, n, s = sample(strata)
    t_build = t_schwarz + est
    return {"value": 1.0 / t_build, "unit": "Fock builds/s", "cores": oracle.lib().orc_num_threads(),
            "kind": "port",
            "sample": f"{s} stratified bra rows of {npairs} ({n} of ~{nq:.3g} screened AO quartets) in "
                      f"{dt:.1f}s + full serial Schwarz table {t_schwarz:.1f}s; build time extrapolated to "
                      f"{t_build:.0f}s",
            "est_seconds_per_build": t_build}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    atoms, mol, shells = build_shells()
    vals = []
    for _ in range(args.warmup):
        cpu_fock_rate(shells, budget_s=2.0)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        vals.append(cpu_fock_rate(shells, budget_s=args.ref_budget))
    wall = time.perf_counter() - t0
    v = float(np.mean([x["value"] for x in vals]))
    line = {"metric": "Fock builds/s", "value": v, "unit": "Fock builds/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded water cluster, Basis Set Exchange 6-31G**)",
            "config": {"workload": WORKLOAD, "nbasis": 800, "tol_eri": 1e-10},
            "cpu_baseline": {"value": v, "unit": "Fock builds/s", "cores": vals[-1]["cores"], "kind": "port",
                             "sample": vals[-1]["sample"]},
            "e2e": {"value": v, "unit": "Fock builds/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall,
            "note": "the reference's own direct build materialises an nb^4 tensor (3.3 TB at 800 functions) "
                    "and cannot run; timed is the oracle's restatement of its integral path with streaming "
                    "digestion on all host threads"}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# Our arm
# ---------------------------------------------------------------------------
def _traffic_from_profiles(kernel_class):
    """DRAM bytes per launch of the dominant class kernel from the committed
    ncu summary (profiles/ncu_traffic.json), when it covers this class."""
    path = os.path.join(REPO, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        e = d.get("classes", {}).get(kernel_class)
        return None if e is None else e.get("dram_bytes_per_full_launch")
    except (OSError, ValueError):
        return None


def ours_arm(args):
    import torch
    import torch.distributed as dist
    P = _pfk()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    atoms, mol, shells = build_shells(args.waters)
    t0 = time.perf_counter()
    eng = P.FockEngine(shells, device=local, engine=args.engine, precision=args.precision, fp32_bound=1e-8)
    t_setup = time.perf_counter() - t0
    tuned, t_tune = None, 0.0
    if args.engine == "auto":   # per-class kernel choice measured on this molecule's lists
        t0 = time.perf_counter()
        tuned = eng.autotune()
        t_tune = time.perf_counter() - t0
    eng.set_lanes(args.lanes)
    if world > 1:
        eng.set_shard(rank, world)
    nb = eng.nbasis
    stats = eng.class_stats(timed=False)
    n_shell = sum(v[0] for v in stats.values())          # this rank's lists are slices of these
    flops = sum(P.class_flops(k, v[1]) for k, v in stats.items()) / world
    launches = sum(1 for v in stats.values() if v[0] > 0) + 1

    Pm = density(nb)
    dP = torch.tensor(Pm, device=f"cuda:{local}", dtype=torch.float64)
    dG = torch.zeros_like(dP)
    # a real (non-default) stream: the graph is captured and replayed on it,
    # and the timing events are recorded on it
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)

    def step(e=None):
        (e or eng).fock_rhf_device(dP.data_ptr(), dG.data_ptr(), stream.cuda_stream)
        if world > 1:
            dist.all_reduce(dG)

    def device_ms(e, steps):
        for _ in range(3):
            step(e)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(steps):
            step(e)
        b.record(stream)
        torch.cuda.synchronize()
        t = a.elapsed_time(b) / steps
        if world > 1:
            tt = torch.tensor([t], device=f"cuda:{local}", dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt.item())
        return t

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    clk = clocks.stop()
    ms_step = ms / args.steps

    # end to end through the C ABI with host buffers (pinned), per step:
    # H2D of P, build, D2H of G (+ the all-reduce of the partial G when N > 1)
    Ph = torch.from_numpy(Pm).pin_memory().numpy()
    Gacc = torch.zeros_like(dP)
    for _ in range(2):
        eng.fock_rhf(Ph)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        Gh = eng.fock_rhf(Ph)
        if world > 1:
            Gacc.copy_(torch.from_numpy(Gh))
            dist.all_reduce(Gacc)
            Gh = Gacc.cpu().numpy()
    e2e_s = (time.perf_counter() - t0) / args.steps
    if world > 1:
        t = torch.tensor([e2e_s], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    h2d = nb * nb * 8 * (2 if world > 1 else 1)
    d2h = nb * nb * 8 * (2 if world > 1 else 1)

    # the plain all-FP64 GPU build on the same molecule, for the mixed-precision
    # speed-up and its error (G and the two-electron energy 1/2 tr(P G))
    mixed = None
    if args.precision == "mixed":
        step()
        torch.cuda.synchronize()
        G_mixed = dG.cpu().numpy().copy()
        e64 = P.FockEngine(shells, device=local, engine=args.engine, precision="fp64")
        if args.engine == "auto":
            e64.autotune()
        e64.set_lanes(args.lanes)
        if world > 1:
            e64.set_shard(rank, world)
        ms64 = device_ms(e64, max(3, args.steps // 2))
        G64 = dG.cpu().numpy().copy()
        e64.close()
        dG_ = G_mixed - G64
        mixed = {"fp64_gpu_builds_per_s": 1e3 / ms64, "fp64_gpu_ms_per_step": ms64,
                 "speedup_vs_fp64_gpu": ms64 / ms_step, "max_abs_dG_vs_fp64": float(np.abs(dG_).max()),
                 "dE_2e_vs_fp64_Eh": float(0.5 * (Pm * dG_).sum()), "fp32_bound": 1e-8}

    # per-class timing pass (events around each class kernel, untimed region)
    dP_host = Pm  # class_stats times a build on the context's current density
    eng.fock_rhf(dP_host)
    cls = eng.class_stats(timed=True)
    cls_rys = None
    if args.engine != "rys":   # the same classes on the Rys kernels, for the engine choice
        er = P.FockEngine(shells, device=local, engine="rys", precision=args.precision, fp32_bound=1e-8)
        if world > 1:
            er.set_shard(rank, world)
        er.fock_rhf(dP_host)
        cls_rys = er.class_stats(timed=True)
        er.close()
    fp64_peak, fp32_peak = P.measure_fma_peak(local)
    top = max(cls.items(), key=lambda kv: kv[1][2])
    top_flops = P.class_flops(top[0], top[1][1]) / world
    top_ach = top_flops / (top[1][2] * 1e-3) / 1e12 if top[1][2] > 0 else 0.0
    build_ach = flops / (ms_step * 1e-3) / 1e12

    result = None
    if rank == 0:
        value = 1e3 / ms_step
        line = {"metric": "Fock builds/s", "value": value, "unit": "Fock builds/s", "n_gpus": world,
                "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms_step,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "f64+f32",
                "data": "synthetic (seeded water cluster, Basis Set Exchange 6-31G**)",
                "config": {"workload": WORKLOAD if args.waters == 32 else f"(H2O){args.waters} 6-31G** ({nb} bf)",
                           "nbasis": nb, "tol_eri": 1e-10, "precision": args.precision, "engine": args.engine,
                           "lanes": args.lanes, "prim_tol": 1e-16,
                           "parallelism": f"quartet-list shards x{world} + NCCL all-reduce of G" if world > 1
                           else "single GPU", "l2": "inputs larger than L2: the screened quartet lists "
                           f"({n_shell * 8 / 1e9:.2f} GB) and primitive-pair data stream from HBM every build",
                           "seed": SEED},
                "eri_shell_quartets_per_s": n_shell / (ms_step * 1e-3),
                "eri_primitive_quartets_per_s": sum(v[1] for v in stats.values()) / (ms_step * 1e-3),
                "gpu_launches": launches * args.steps,
                "setup_s": t_setup,
                "e2e": {"value": 1.0 / e2e_s, "unit": "Fock builds/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "timing": "wall clock around the blocking C-ABI call"},
                "roofline": {"bound": "fp64", "kernel": f"eri class {top[0]}", "achieved": top_ach,
                             "peak": fp64_peak, "unit": "TFLOP/s", "frac": top_ach / fp64_peak,
                             "traffic": _traffic_from_profiles(top[0]),
                             "peak_source": "FP64 FMA loop measured in this run (pfk_measure_fma_peak); "
                                            "the driver's peaks file lists HBM and BF16 only",
                             "flops_per_launch": top_flops, "launch_ms": top[1][2]},
                "roofline_build": {"achieved": build_ach, "peak": fp64_peak, "unit": "TFLOP/s",
                                   "frac": build_ach / fp64_peak, "flops_per_build": flops},
                "fp32_fma_peak_tflops": fp32_peak,
                "classes_ms": {k: round(v[2], 3) for k, v in sorted(cls.items(), key=lambda kv: -kv[1][2])[:12]},
                "classes_primitive_quartets": {k: v[1] for k, v in sorted(cls.items(), key=lambda kv: -kv[1][2])[:12]},
                "classes_shell_quartets": {k: v[0] for k, v in sorted(cls.items(), key=lambda kv: -kv[1][2])[:12]},
                "autotune": None if tuned is None else
                {"seconds": t_tune, "choice": {k: v[0] for k, v in tuned.items()
                                               if k in dict(sorted(cls.items(), key=lambda kv: -kv[1][2])[:12])}},
                "classes_ms_rys_kernels": None if cls_rys is None else
                {k: round(cls_rys[k][2], 3) for k, v in sorted(cls.items(), key=lambda kv: -kv[1][2])[:12]},
                "clocks": clk}
        if mixed:
            line["mixed_precision"] = mixed
        if world == 1 and not args.no_cpu:
            line["cpu_baseline"] = {k: v for k, v in cpu_fock_rate(shells, budget_s=args.cpu_budget).items()
                                    if k != "est_seconds_per_build"}
        result = line
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0 if result is not None or rank != 0 else 1


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--engine", choices=["os", "rys", "auto"], default="auto",
                    help="integral engine (the reference's option); auto runs the autotuner at setup")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed",
                    help="mixed: FP32 below a Schwarz bound of 1e-8 (the benchmark configuration); "
                         "the all-FP64 build is timed beside it")
    ap.add_argument("--cpu-budget", type=float, default=15.0, help="seconds of CPU sampling for cpu_baseline")
    ap.add_argument("--ref-budget", type=float, default=8.0, help="seconds of CPU sampling per reference step")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--lanes", type=int, default=4, choices=[1, 2, 3, 4],
                    help="streams the class kernels of a build are spread over")
    ap.add_argument("--waters", type=int, default=32,
                    help="cluster size; 32 is the benchmark workload, smaller sizes are for profiling")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    return ours_arm(args)


if __name__ == "__main__":
    sys.exit(main())
