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

The default line also carries time_to_energy: whole RHF runs of C40H82 /
cc-pVDZ through pfk_scf_rhf, the plain all-FP64 path from the
core-Hamiltonian guess against mixed precision with the learned guess.

Other modes (--mode): eri-classes (the ERI class microbenchmark: every class
(ss|ss)..(ff|ff) on 2^20 seed-random shell quartets, OS and Rys, FP64 and
FP32, written as a JSON table with --out), mo (the AO -> MO transform and the
MP2 energy of (H2O)7), scf (whole SCF runs of one molecule several ways).
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
def cpu_fock_rate(shells, rows=4096, seed=SEED):
    """Fock builds/s of the reference's direct path on the host cores,
    extrapolated from a stratified sample of `rows` bra AO-pair rows (one row
    drawn per stratum with a fixed seed, so every call times the same rows).
    Per build the reference recomputes the Schwarz table serially
    (os.cpp:1447, timed in full here) and evaluates every screened canonical
    AO quartet with its per-component OS code (os.cpp:1458-1507, restated);
    its nb^4 tensor scatter and O(nb^4) digestion (os.cpp:1450, 1514-1520)
    cannot run at 800 functions (3.3 TB) and are replaced by the streaming
    digestion, which only makes the baseline faster."""
    import oracle
    ob = oracle.Basis(shells)
    nb, npairs = ob.nbasis, ob.npairs
    t0 = time.perf_counter()
    Q = ob.schwarz(oracle.OS)
    t_schwarz = time.perf_counter() - t0
    Pm = density(nb)
    rng = np.random.default_rng(seed)
    strata = int(min(npairs, rows))
    edges = np.linspace(0, npairs, strata + 1).astype(np.int64)
    picks = np.array([rng.integers(edges[i], max(edges[i] + 1, edges[i + 1])) for i in range(strata)],
                     dtype=np.int32)
    t = time.perf_counter()
    _, _, n = ob.jk_direct_rows(Pm, [Pm], picks, 1e-10, oracle.OS, Q=Q)
    dt = time.perf_counter() - t
    t_build = t_schwarz + dt * npairs / strata
    nq = n * npairs / strata
    return {"value": 1.0 / t_build, "unit": "Fock builds/s", "cores": oracle.lib().orc_num_threads(),
            "kind": "port",
            "sample": f"{strata} stratified bra rows of {npairs} (fixed seed {seed}; {n} of ~{nq:.3g} screened AO "
                      f"quartets) in {dt:.1f}s + full serial Schwarz table {t_schwarz:.1f}s; build time "
                      f"extrapolated to {t_build:.0f}s",
            "sample_seconds": dt + t_schwarz, "est_seconds_per_build": t_build}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    atoms, mol, shells = build_shells()
    vals = []
    for _ in range(args.warmup):
        cpu_fock_rate(shells, rows=256)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        vals.append(cpu_fock_rate(shells, rows=args.cpu_rows))
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
            "wall_s": wall, "extrapolated": True,
            "sample_seconds_per_step": wall / max(1, args.steps),
            "note": "the reference's own direct build materialises an nb^4 tensor (3.3 TB at 800 functions) "
                    "and cannot run; timed is the oracle's restatement of its integral path with streaming "
                    "digestion on all host threads, on the same fixed sample of bra rows every step, and "
                    "value / ms_per_step are that sample's time extrapolated to the whole build (each step "
                    "takes sample_seconds_per_step of wall time)"}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# Our arm
# ---------------------------------------------------------------------------
def reference_auto_rys_share(cls):
    """Share of the Cartesian component quartets of class cls, e.g. "(dp|ps)",
    that the reference's per-component `engine auto` cost model sends to Rys
    (rys.cpp:195-220: Rys when its work estimate, 2D-table size times roots
    plus the transfer and a per-root cost, is below OS's, table size times
    L + 1 plus the transfer), with the pairs oriented L(A) >= L(B) as this
    library orients them.  Reported beside the autotuner's per-class choice."""
    ls = ["spdf".index(ch) for ch in cls if ch in "spdf"]

    def carts(L):
        return [(L - yz, yz - z, z) for yz in range(L + 1) for z in range(yz + 1)]
    n = rys = 0
    for a in carts(ls[0]):
        for b in carts(ls[1]):
            for c in carts(ls[2]):
                for d in carts(ls[3]):
                    ab = [a[k] + b[k] for k in range(3)]
                    cd = [c[k] + d[k] for k in range(3)]
                    L = sum(ab) + sum(cd)
                    nroots = L // 2 + 1
                    six = float(np.prod([x + 1 for x in ab + cd]))
                    hrr = sum(b) + sum(d) + 1
                    os_work = six * (L + 1) + hrr * six * 0.25
                    rys_work = six * nroots + hrr * six * 0.20 + 24.0 * nroots
                    n += 1
                    rys += rys_work < os_work
    return rys / n


def _traffic_from_profiles(kernel_class):
    """(DRAM bytes per launch, where that number comes from) for the dominant
    class kernel, from the committed ncu summary profiles/ncu_traffic.json
    when it covers this class: a static estimate from an earlier capture, not
    a measurement of this run (ncu replays kernels and is never run inside
    the timed bench)."""
    path = os.path.join(REPO, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        e = d.get("classes", {}).get(kernel_class)
        if e is None:
            return None, None
        return e.get("dram_bytes_per_full_launch"), "static estimate, not measured in this run: " + d.get("source", "")
    except (OSError, ValueError):
        return None, None


def time_to_energy(device, runs=("fp64", "mixed+guess", "mixed+guess+dP"), model_path=None):
    """Time to the converged RHF energy of C40H82 / cc-pVDZ (1010 Cartesian
    functions; all-trans, seeded +-0.03 Angstrom noise), each arm a fresh
    context and a whole SCF through the C ABI (pfk_scf_rhf: builds, DIIS and
    diagonalisation on the device), wall-clocked from the start of the guess
    to the converged energy:
      fp64            the plain all-FP64 GPU path, core-Hamiltonian guess;
      mixed+guess     FP32 below a Schwarz bound of 1e-8, learned guess;
      mixed+guess+dP  the same with FP32 difference-density builds.
    Setup (pair data, Schwarz table, lists, one-electron integrals) is timed
    separately and is the same for every arm."""
    P = _pfk()
    atoms = P.workloads.alkane(40, seed=3, noise=0.03)
    lib = P.basis.load_library()
    model_path = model_path or os.path.join(REPO, "planck-refactored_b200", "data", "guess_model_ccpvdz.npz")
    model = P.guess.GuessModel.load(model_path, device=device)
    out = {"molecule": "C40H82 cc-pVDZ (1010 Cartesian functions), seed 3", "arms": {}}
    ref = None
    for label in runs:
        prec = "fp64" if label == "fp64" else "mixed"
        t0 = time.perf_counter()
        sysm = P.scf.System(atoms, "cc-pvdz", lib, device=device, precision=prec, fp32_bound=1e-8)
        if "dP" in label:
            sysm.incremental_engine()
        t_setup = time.perf_counter() - t0
        t0 = time.perf_counter()
        P0 = G0 = None
        hook = None
        if "guess" in label:
            P0, G0, hook = P.guess.choose(model, sysm)
        t_guess = time.perf_counter() - t0
        r = sysm.run(P0=P0, G0=G0, linalg="gpu", incremental="dP" in label)
        wall = time.perf_counter() - t0
        sysm.close()
        if ref is None:
            ref = r["energy"]
        # the first iteration from which the energy stays within 1e-6 Eh of
        # the converged one, and the time it was reached
        hist = r["history"]
        k = len(hist)
        while k > 0 and abs(hist[k - 1][1] - r["energy"]) <= 1e-6:
            k -= 1
        k = min(k, len(hist) - 1)
        out["arms"][label] = {"seconds_to_energy": wall, "iterations": r["iterations"], "converged": r["converged"],
                              "energy": r["energy"], "dE_vs_fp64_Eh": r["energy"] - ref,
                              "iterations_to_1e-6": k + 1, "seconds_to_1e-6": t_guess + hist[k][5] * 1e-3,
                              "full_builds": r["full_builds"], "difference_builds": r["difference_builds"],
                              "build_seconds": r["build_seconds"], "guess_seconds": t_guess,
                              "setup_seconds": t_setup}
        if hook is not None:
            out["arms"][label]["guess"] = {"accepted": hook["accepted"], "predict_seconds": hook["predict_s"],
                                           "first_energy_learned": hook["E_first_learned"],
                                           "first_energy_default": hook["E_first_default"]}
    model.close()
    base = out["arms"].get("fp64", {}).get("seconds_to_energy")
    if base:
        out["speedup_vs_fp64"] = {k: base / v["seconds_to_energy"] for k, v in out["arms"].items()}
        b6 = out["arms"]["fp64"]["seconds_to_1e-6"]
        out["speedup_vs_fp64_to_1e-6"] = {k: b6 / v["seconds_to_1e-6"] for k, v in out["arms"].items()}
    out["note"] = ("seconds_to_energy: to the reference's convergence tests (|dE| < 1e-10, rms and max dP < 1e-10); "
                   "below max dP ~1e-8 the loop wanders at the rounding level until one step meets them, so the "
                   "iteration count of that tail is deterministic for this code but sensitive to any change in "
                   "rounding; seconds_to_1e-6: until the energy is and stays within 1e-6 Eh of the converged one")
    return out


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
    Gpin = torch.empty(Pm.shape, dtype=torch.float64).pin_memory().numpy()
    Gacc = torch.zeros_like(dP)
    for _ in range(2):
        eng.fock_rhf(Ph, out=Gpin)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        Gh = eng.fock_rhf(Ph, out=Gpin)
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
        # how much of the build the FP32 list carries
        p32 = eng.precision_stats()
        f32 = sum(P.class_flops(k, v[1]) for k, v in p32.items())
        mixed["fp32_share_shell_quartets"] = sum(v[0] for v in p32.values()) / max(1, n_shell * world)
        mixed["fp32_share_flop_alg"] = f32 / max(1.0, flops * world)
        mixed["fp32_share_per_class"] = {
            k: {"shell_quartets": round(v[0] / max(1, stats[k][0]), 4),
                "flop_alg": round(P.class_flops(k, v[1]) / max(1.0, P.class_flops(k, stats[k][1])), 4)}
            for k, v in sorted(p32.items(), key=lambda kv: -P.class_flops(kv[0], kv[1][1]))[:12]}

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
                             "traffic": _traffic_from_profiles(top[0])[0],
                             "traffic_source": _traffic_from_profiles(top[0])[1],
                             "peak_source": "FP64 FMA loop measured in this run (pfk_measure_fma_peak); "
                                            "the measured-peaks file lists HBM copy and BF16 GEMM peaks only",
                             "flops_per_launch": top_flops, "launch_ms": top[1][2]},
                "roofline_build": {"achieved": build_ach, "peak": fp64_peak, "unit": "TFLOP/s",
                                   "frac": build_ach / fp64_peak, "flops_per_build": flops},
                "fp32_fma_peak_tflops": fp32_peak,
                "classes_ms": {k: round(v[2], 3) for k, v in sorted(cls.items(), key=lambda kv: -kv[1][2])[:12]},
                "classes_primitive_quartets": {k: v[1] for k, v in sorted(cls.items(), key=lambda kv: -kv[1][2])[:12]},
                "classes_shell_quartets": {k: v[0] for k, v in sorted(cls.items(), key=lambda kv: -kv[1][2])[:12]},
                "autotune": None if tuned is None else
                {"seconds": t_tune, "choice": {k: v[0] for k, v in tuned.items()
                                               if k in dict(sorted(cls.items(), key=lambda kv: -kv[1][2])[:12])},
                 "reference_model_rys_share": {k: round(reference_auto_rys_share(k), 3) for k, v in tuned.items()
                                               if k in dict(sorted(cls.items(), key=lambda kv: -kv[1][2])[:12])}},
                "classes_ms_rys_kernels": None if cls_rys is None else
                {k: round(cls_rys[k][2], 3) for k, v in sorted(cls.items(), key=lambda kv: -kv[1][2])[:12]},
                "clocks": clk}
        if mixed:
            line["mixed_precision"] = mixed
        if world == 1 and not args.no_cpu:
            line["cpu_baseline"] = {k: v for k, v in cpu_fock_rate(shells, rows=args.cpu_rows).items()
                                    if k != "est_seconds_per_build"}
        if world == 1 and not args.no_scf:
            # in a child process that never imports torch, as a C++ host would
            # run it: torch ships its own cuBLAS and cuSOLVER, and once loaded
            # they are the copies this library's calls bind to
            env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", str(local)))
            r = subprocess.run([sys.executable, os.path.abspath(__file__), "--mode", "time-to-energy"],
                               capture_output=True, text=True, env=env)
            tte = [x for x in r.stdout.splitlines() if x.startswith("{")]
            line["time_to_energy"] = json.loads(tte[-1]) if r.returncode == 0 and tte else \
                {"error": (r.stderr or r.stdout)[-500:]}
        result = line
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0 if result is not None or rank != 0 else 1


# ---------------------------------------------------------------------------
# ERI class microbenchmark: every class (ss|ss)..(ff|ff) on seed-random shell
# quartets, Obara-Saika and Rys kernels, FP64 and FP32-with-FP64-Boys
# ---------------------------------------------------------------------------
CLASS_LS = [(pc_a, pc_b, pk_a, pk_b)
            for x, (pc_a, pc_b) in enumerate([(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2), (3, 0), (3, 1), (3, 2),
                                               (3, 3)])
            for (pk_a, pk_b) in [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2), (3, 0), (3, 1), (3, 2), (3, 3)][:x + 1]]


def _oracle_block_check(shells, n_check, blocks, budget_s):
    """Max |GPU - oracle| over the first quartets of a class (oracle Rys
    engine, one small oracle basis per group of quartets), within a time
    budget.  blocks: {variant: (n, ncomp) host array of the same quartets}."""
    import oracle
    L = np.asarray(shells["L"])
    off = np.concatenate([[0], np.cumsum(shells["nprim"])])
    nbf = int(sum((int(l) + 1) * (int(l) + 2) // 2 for l in L[:4]))
    group = max(1, min(64, 200 // nbf))
    t0 = time.perf_counter()
    worst = {k: 0.0 for k in blocks}
    within = {k: 0 for k in blocks}
    ncomp = next(iter(blocks.values())).shape[1]
    done = 0
    t_blocks = 0.0
    while done < n_check and time.perf_counter() - t0 < budget_s:
        g = min(group, n_check - done)
        s0, s1 = 4 * done, 4 * (done + g)
        sub = {"L": L[s0:s1], "nprim": shells["nprim"][s0:s1], "center": shells["center"][s0:s1],
               "expo": shells["expo"][off[s0]:off[s1]], "coef": shells["coef"][off[s0]:off[s1]],
               "norm": shells["norm"][off[s0]:off[s1]]}
        ob = oracle.Basis(sub)
        for k in range(g):
            tb = time.perf_counter()
            ref = ob.shell_block(4 * k, 4 * k + 1, 4 * k + 2, 4 * k + 3, oracle.RYS)
            t_blocks += time.perf_counter() - tb
            for name, blk in blocks.items():
                d = np.abs(blk[done + k] - ref) / np.maximum(1.0, np.abs(ref))
                worst[name] = max(worst[name], float(d.max()))
                within[name] += int((d <= 1e-10).sum())
        done += g
    return done, {k: {"max_rel_err": worst[k], "frac_within_1e-10": within[k] / max(1, done * ncomp),
                      "cpu_quartets_per_s_1_thread": done / t_blocks if t_blocks > 0 else None}
                  for k in blocks}


def eri_classes(args):
    """Per-class throughput and accuracy of the integral kernels: 2^20
    seed-random shell quartets per class (centres in a 10 Angstrom cube,
    exponents log-uniform in [0.05, 1e4], contraction depth 1..6,
    coefficients in (0, 1]), through pfk_eri_batch in chunks that fit the
    device.  Variants: Rys FP64 (the reference for the errors), Rys FP32,
    and, for L <= 4, Obara-Saika FP64 and FP32.  Times are the kernels' own,
    from CUDA events on the launching stream."""
    import torch
    P = _pfk()
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    fp64_peak, fp32_peak = P.measure_fma_peak(0)
    rows = []
    classes = CLASS_LS if not args.classes else [CLASS_LS[int(c)] for c in args.classes.split(",")]
    for (la, lb, lc, ld) in classes:
        name = "(%s%s|%s%s)" % tuple("spdf"[x] for x in (la, lb, lc, ld))
        t_gen = time.perf_counter()
        shells, pairs, quartets = P.workloads.eri_class_quartets(la, lb, lc, ld, args.quartets, seed=SEED)
        t_gen = time.perf_counter() - t_gen
        kq = shells["nprim"].reshape(-1, 4).astype(np.int64).prod(axis=1)
        flops = P.class_flops(name, int(kq.sum()))
        batch = P.EriBatch(shells, pairs, quartets)
        nc, n = batch.ncomp, batch.n
        chunk = int(min(n, max(256, (1 << 30) // (8 * nc))))
        variants = [("rys", "fp64"), ("rys", "mixed")]
        if la + lb + lc + ld <= 4:
            variants += [("os", "fp64"), ("os", "mixed")]
        bufs = {v: torch.empty(chunk * nc, dtype=torch.float64, device="cuda:0") for v in variants}
        ms = {v: 0.0 for v in variants}
        err = {v: 0.0 for v in variants}
        rel = {v: 0.0 for v in variants}
        ncheck = min(n, args.oracle_quartets)
        keep = {v: [] for v in variants if v[1] == "fp64"}
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * len(variants))]
        with torch.cuda.stream(stream):
            batch.run(0, min(chunk, n), "rys", "fp64", bufs[variants[0]].data_ptr(), stream.cuda_stream)   # warm-up
            for first in range(0, n, chunk):
                cnt = min(chunk, n - first)
                for k, v in enumerate(variants):
                    ev[2 * k].record(stream)
                    batch.run(first, cnt, v[0], v[1], bufs[v].data_ptr(), stream.cuda_stream)
                    ev[2 * k + 1].record(stream)
                stream.synchronize()
                for k, v in enumerate(variants):
                    ms[v] += ev[2 * k].elapsed_time(ev[2 * k + 1])
                ref = bufs[variants[0]][:cnt * nc]
                for v in variants[1:]:
                    d = (bufs[v][:cnt * nc] - ref).abs()
                    err[v] = max(err[v], float(d.max()))
                    rel[v] = max(rel[v], float((d / ref.abs().clamp(min=1.0)).max()))
                if first < ncheck:
                    for v in keep:
                        take = min(cnt, ncheck - first)
                        keep[v].append(bufs[v][:take * nc].view(take, nc).cpu().numpy())
        batch.close()
        blocks = {f"{v[0]}_{v[1]}": np.concatenate(keep[v]) for v in keep if keep[v]}
        n_or, orc = (_oracle_block_check(shells, ncheck, blocks, args.oracle_budget) if ncheck > 0 else
                     (0, {f"{v[0]}_{v[1]}": {"max_rel_err": None, "frac_within_1e-10": None,
                                              "cpu_quartets_per_s_1_thread": None} for v in keep}))
        for v in variants:
            peak = fp64_peak if v[1] == "fp64" else fp32_peak
            rate = flops / (ms[v] * 1e-3) / 1e12
            row = {"class": name, "engine": v[0], "arith": "fp64" if v[1] == "fp64" else "fp32+fp64-boys",
                   "quartets": n, "primitive_quartets": int(kq.sum()), "ms": round(ms[v], 3),
                   "quartets_per_s": n / (ms[v] * 1e-3), "flop_alg_tflops": rate,
                   "frac_of_measured_peak": rate / peak,
                   "peak": "fp64 FMA" if v[1] == "fp64" else "fp32 FMA",
                   "max_abs_err_vs_rys_fp64": err[v], "max_rel_err_vs_rys_fp64": rel[v],
                   "reference_model_rys_share": round(reference_auto_rys_share(name), 3)}
            if v[1] == "fp64":
                row["oracle"] = dict(orc[f"{v[0]}_{v[1]}"], quartets=n_or)
            rows.append(row)
            print(json.dumps(row), flush=True)
    out = {"what": "ERI class microbenchmark: per-class quartets/s and error, 55 classes x {OS, Rys} x {FP64, "
                   "FP32 with FP64 Boys/roots}; OS kernels exist for L <= 4",
           "inputs": f"{args.quartets} seed-random shell quartets per class (seed {SEED}): centres uniform in a "
                     "10 Angstrom cube, exponents log-uniform in [0.05, 1e4], contraction depth uniform 1..6, "
                     "coefficients uniform in (0, 1], reference normalisation",
           "timing": "CUDA events around each kernel launch on its stream, summed over chunks; outputs are the "
                     "normalised Cartesian blocks written to HBM",
           "fp64_fma_peak_tflops": fp64_peak, "fp32_fma_peak_tflops": fp32_peak,
           "oracle": "first quartets of each class against the oracle's per-component Rys integrals "
                     f"(up to {args.oracle_quartets} quartets or {args.oracle_budget} s per class); "
                     "relative to max(1, |v|); cpu_quartets_per_s_1_thread is the oracle's rate on those quartets "
                     "(one host thread, the shell-block calls alone): the reference's per-component contraction "
                     "(rys.cpp:489-505) restated, the CPU baseline of this table",
           "host_threads_available": os.cpu_count(),
           "rows": rows}
    if args.out:
        with open(args.out, "w") as f:
            json.dump(out, f, indent=1)
    return 0


# ---------------------------------------------------------------------------
# AO -> MO transform and MP2 (pfk_mo_transform, pfk_rmp2_energy)
# ---------------------------------------------------------------------------
def mo_transform(args):
    """Device AO -> MO transform behind MP2: a seeded water cluster in 6-31G**
    (7 waters: 175 Cartesian functions, the largest cluster under the
    180-function limit of the dense tensor), the MP2 block (C_occ C_vir |
    C_occ C_vir) of its converged RHF.  Per phase, the device time from CUDA
    events inside the call: the AO tensor (class kernels in tensor mode), the
    four quarter-transform GEMMs (FP64, cuBLAS) against the FP64 FMA peak
    measured in the same run, and the copy of the block to the host; then the
    RMP2 energy summed on the host from that block and on the device
    (pfk_rmp2_energy, the block never leaving HBM)."""
    P = _pfk()
    sysm = P.scf.System(P.workloads.water_cluster(args.waters, seed=SEED), "6-31g**", P.basis.load_library())
    r = sysm.run()
    nb, no = sysm.H.shape[0], sysm.nocc
    nv = nb - no
    C = r["C"]
    eng = sysm.engine
    eng.mo_transform(C[:, :no], C[:, no:], C[:, :no], C[:, no:])   # warm-up (BLAS handle, kernels)
    times = []
    for _ in range(args.steps):
        eng.mo_transform(C[:, :no], C[:, no:], C[:, :no], C[:, no:])
        times.append(eng.mo_transform_times())
    t = min(times, key=lambda x: x[1])
    flops = 2.0 * (no * nb ** 4 + no * nv * nb ** 3 + no * nv * no * nb ** 2 + no * nv * no * nv * nb)
    fp64_peak, _ = P.measure_fma_peak(0)
    e2 = P.mp2.rmp2(eng, C, r["eps"], no)
    dev = []
    for _ in range(args.steps):
        e_dev = eng.rmp2_energy(C, r["eps"], no)
        dev.append(eng.mo_transform_times())
    td = min(dev, key=lambda x: x[1])
    sysm.close()
    out = {"workload": f"(H2O){args.waters} 6-31G** ({nb} bf), MP2 block (occ vir|occ vir), nocc {no}, nvir {nv}",
           "ao_tensor_ms": t[0], "ao_tensor_GBps_written": nb ** 4 * 8 / t[0] / 1e6,
           "gemm_ms": t[1], "gemm_flops": flops, "gemm_tflops": flops / t[1] / 1e9,
           "fp64_fma_peak_tflops": fp64_peak, "gemm_frac_of_fp64_peak": flops / t[1] / 1e9 / fp64_peak,
           "copy_out_ms": t[2], "mo_block_MB": no * nv * no * nv * 8 / 1e6,
           "rhf_energy": r["energy"], "rmp2_corr": e2,
           "rmp2_on_device": {"corr": e_dev, "ao_tensor_ms": td[0], "gemm_ms": td[1], "sum_ms": td[2],
                              "total_ms": sum(td), "block_read_GBps": 2 * no * nv * no * nv * 8 / td[2] / 1e6}}
    print(json.dumps(out), flush=True)
    return 0


# ---------------------------------------------------------------------------
# Whole SCF runs, several ways
# ---------------------------------------------------------------------------
def scf_runs(args):
    """Time to converged energy of whole RHF runs on the GPU builds, one
    molecule several ways (--runs): fp64 (all-FP64 builds, the plain GPU
    path), mixed (FP32 below a Schwarz bound of 1e-8), mixed+dP (with FP32
    difference-density builds), and fp64+guess / mixed+guess (the learned
    guess hook).  --linalg picks the loop: host (numpy), gpu (pfk_scf_rhf
    behind the C ABI) or device (the torch loop).  Molecules: C40H82 /
    cc-pVDZ (1010 Cartesian functions) and the 32-water cluster / 6-31G**
    (800)."""
    P = _pfk()
    atoms, basis = ((P.workloads.alkane(40, seed=3, noise=0.03), "cc-pvdz") if args.molecule == "c40h82"
                    else (P.workloads.water_cluster(32, seed=SEED), "6-31g**"))
    lib = P.basis.load_library()
    model_path = args.guess_model or os.path.join(
        REPO, "planck-refactored_b200", "data", "guess_model_ccpvdz.npz" if basis == "cc-pvdz" else
        "guess_model_631gs.npz")
    runs = args.runs.split(",") if args.runs else ["fp64", "mixed", "mixed+dP", "fp64+guess", "mixed+guess"]
    model = P.guess.GuessModel.load(model_path, device=0) if any("guess" in r for r in runs) else None
    out = {"molecule": args.molecule, "basis": basis, "linalg": args.linalg, "runs": {}}
    ref = None
    for label in runs:
        prec = "mixed" if label.startswith("mixed") else "fp64"
        t0 = time.perf_counter()
        sysm = P.scf.System(atoms, basis, lib, precision=prec, fp32_bound=1e-8)
        t_setup = time.perf_counter() - t0
        t0 = time.perf_counter()
        P0 = G0 = None
        if "guess" in label:
            P0, G0, _ = P.guess.choose(model, sysm)
        kw = {"G0": G0} if args.linalg != "device" else {}
        r = sysm.run(P0=P0, incremental="dP" in label, linalg=args.linalg, **kw)
        wall = time.perf_counter() - t0
        sysm.close()
        if ref is None:
            ref = r["energy"]
        out["runs"][label] = {"energy": r["energy"], "dE_vs_first_run": r["energy"] - ref,
                              "iterations": r["iterations"], "converged": r["converged"],
                              "seconds_to_convergence": wall, "setup_seconds": t_setup}
    if model is not None:
        model.close()
    print(json.dumps(out), flush=True)
    return 0


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
    ap.add_argument("--cpu-rows", type=int, default=4096,
                    help="bra AO-pair rows the CPU baseline and each reference step time (the same rows every time)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-scf", action="store_true", help="skip the C40H82 time-to-energy leg")
    ap.add_argument("--lanes", type=int, default=4, choices=[1, 2, 3, 4],
                    help="streams the class kernels of a build are spread over")
    ap.add_argument("--waters", type=int, default=32,
                    help="cluster size; 32 is the benchmark workload, smaller sizes are for profiling")
    ap.add_argument("--mode", choices=["fock", "eri-classes", "mo", "scf", "time-to-energy"], default="fock",
                    help="fock: the Fock-build benchmark (default); eri-classes: the ERI class microbenchmark; "
                         "mo: the AO->MO transform and MP2 on (H2O)7; scf: whole SCF runs several ways")
    ap.add_argument("--molecule", choices=["c40h82", "water32"], default="c40h82", help="scf: the molecule")
    ap.add_argument("--runs", default="", help="scf: comma-separated subset of fp64,mixed,mixed+dP,fp64+guess,"
                                               "mixed+guess")
    ap.add_argument("--linalg", choices=["host", "gpu", "device"], default="gpu", help="scf: the SCF loop")
    ap.add_argument("--guess-model", default="", help="scf: learned-guess model (default: the shipped one)")
    ap.add_argument("--quartets", type=int, default=1 << 20, help="eri-classes: shell quartets per class")
    ap.add_argument("--classes", default="", help="eri-classes: comma-separated class indices (default: all 55)")
    ap.add_argument("--oracle-quartets", type=int, default=4096, help="eri-classes: oracle subset per class")
    ap.add_argument("--oracle-budget", type=float, default=3.0, help="eri-classes: oracle seconds per class")
    ap.add_argument("--out", default="", help="eri-classes: JSON file for the table")
    args = ap.parse_args()
    if args.mode == "eri-classes":
        return eri_classes(args)
    if args.mode == "mo":
        if args.waters == 32:
            args.waters = 7
        return mo_transform(args)
    if args.mode == "scf":
        return scf_runs(args)
    if args.mode == "time-to-energy":
        print(json.dumps(time_to_energy(0)), flush=True)
        return 0
    if args.impl == "reference":
        return reference_arm(args)
    return ours_arm(args)


if __name__ == "__main__":
    sys.exit(main())
