"""Benchmark of the explicit residual-and-update loop on the full-annulus
rotor/stator workload (160 x 48 x 64 nodes, Roe + MUSCL van Albada, RK3,
local time step at CFL 1.0 -- the configuration's 1.2 diverges at iteration
53 in the reference build too -- Hall body force, FP64, with the fp32_kahan
arm beside it).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload annulus|map|serve|realgas|viscous]

One step = one pseudo-time iteration (all Runge-Kutta stages) of the whole
operating point. The metric is cell-stage updates per second (nodes x stages x
iterations / time). With N > 1 (launched by torch.distributed.run) every rank
advances its own replica of the operating point: the path has no exchange
between operating points, so there is no data-path collective ("replicas
only"); NCCL carries only the barrier and the max-over-ranks time.

Printed: one JSON line on rank 0.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "cell-stage updates/s"
UNIT = "cell-stage/s"
WORKLOAD = ("full-annulus rotor+stator 160x48x64, Roe+MUSCL(van Albada), RK3, local dt CFL 1.0, Hall BFM, FP64 "
            "(CFL 1.2 diverges at iteration 53 in the reference build and here alike)")
L2_BYTES = 126 * 1024 * 1024


def make_case():
    from cturbobfm_b200 import cases

    # Roe + MUSCL + RK3 at CFL 1.2 (the configuration as written) blows up at
    # iteration 53 from the uniform start in the reference solver itself; CFL
    # 1.0 runs stably. The work per iteration does not depend on the CFL.
    return cases.annulus3d(cfl=1.0)


def rank_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except OSError:
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.remove(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------- reference
def reference_iteration_seconds(ini_dir: str, n_iter: int, threads: int) -> float:
    """Per-iteration wall time of the reference build (oracle/_ref/turbobfm),
    from two runs of the same case (n_iter and 1 iterations) so set-up and
    output cancel."""
    from oracle import oracle

    env = dict(os.environ, OMP_NUM_THREADS=str(threads))

    def run(n):
        ini = os.path.join(ini_dir, "input.ini")
        lines = open(ini).read().splitlines()
        lines = [l for l in lines if not l.startswith("N_ITERATIONS")] + [f"N_ITERATIONS = {n}"]
        open(ini, "w").write("\n".join(lines) + "\n")
        t0 = time.perf_counter()
        r = subprocess.run([oracle.REF_CLI, "input.ini"], cwd=ini_dir, stdout=subprocess.DEVNULL,
                           stderr=subprocess.PIPE, env=env, timeout=900)
        if r.returncode != 0:
            raise RuntimeError("reference run failed: " + r.stderr.decode()[-300:])
        return time.perf_counter() - t0

    t1 = run(1)
    tn = run(n_iter + 1)
    return (tn - t1) / n_iter


def port_iteration_seconds(ini_path: str, n_iter: int) -> float:
    """Per-iteration time of the single-threaded C oracle (when the reference
    build is absent)."""
    from oracle.oracle import Oracle

    o = Oracle(ini_path)
    o.run(1)
    t0 = time.perf_counter()
    o.run(n_iter)
    return (time.perf_counter() - t0) / n_iter


def cpu_baseline(case, n_iter: int, one_core_iters: int = 0):
    from oracle import oracle

    stages = case.n_stages
    with tempfile.TemporaryDirectory() as d:
        ini = case.with_settings(SAVE_ITERATIONS_INTERVAL="100000000").write(d)
        if os.path.exists(oracle.REF_CLI):
            threads = os.cpu_count() or 1
            sec = reference_iteration_seconds(d, n_iter, threads)
            kind = "reference"
        else:
            threads = 1
            sec = port_iteration_seconds(ini, n_iter)
            kind = "port"
        one_core = None
        if kind == "reference" and one_core_iters > 0:
            one_core = case.n_nodes * stages / reference_iteration_seconds(d, one_core_iters, 1)
    value = case.n_nodes * stages / sec
    out = {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
           "sample": f"{n_iter} iterations of the same {case.shape[0]}x{case.shape[1]}x{case.shape[2]} case "
                     f"({n_iter * stages} stages), set-up subtracted", "seconds_per_iteration": sec}
    if one_core is not None:
        out["value_1_core"] = one_core
        out["sample_1_core"] = f"{one_core_iters} iterations on 1 thread, set-up subtracted"
    return out


def run_reference_arm(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return
    case = make_case()
    n = max(1, min(args.steps, 40))
    base = cpu_baseline(case, n)
    line = {
        "impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": args.gpus,
        "steps": n, "warmup": args.warmup, "ms_per_step": base["seconds_per_iteration"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "nodes": case.n_nodes, "stages_per_step": case.n_stages},
        "cpu_baseline": {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ ours
def blade_fraction(case) -> float:
    """Share of the nodes inside blade rows (bladePresent > 0)."""
    import numpy as np

    bp = case.fields.get("bladePresent")
    return 0.0 if bp is None else float(np.count_nonzero(bp > 0)) / bp.size


def stage_bytes_per_cell(case, word: int = 8) -> float:
    """Algorithmic bytes of one cell-stage update as the survey's measurement
    section defines them: w * (5 read U(k-1) + 5 read U^n + 5 written U(k) + 1
    read dt/V) + 8 * 3 * d bytes of face vectors (d face directions owned per
    node), plus 14 BFM fields of w bytes at blade-row nodes; the float path
    adds 40 bytes to read and write the Kahan compensation."""
    d = 3 if case.shape[2] > 1 else 2
    b = word * 16 + 8 * 3 * d + 14 * word * blade_fraction(case)
    if word == 4:
        b += 40
    return b


def algorithmic_bytes(case, kernel: str) -> float:
    """Compulsory DRAM bytes of one launch of a kernel kind (FP64). k_stage
    (one fused stage) takes the survey's per-cell-stage figure times the nodes;
    the split kernels count every input read once and every output written
    once."""
    ni, nj, nk = case.shape
    n = ni * nj * nk
    faces = {"I": (ni + 1) * nj * nk, "J": ni * (nj + 1) * nk, "K": ni * nj * (nk + 1)}
    if kernel == "k_stage":
        return stage_bytes_per_cell(case) * n
    if kernel.startswith("k_faces_"):
        f = faces[kernel[-1]]
        if kernel == "k_faces_K":
            f = int(round(f * (1.0 - blade_fraction(case))))  # blade rows have no K flux
        return 8.0 * (5 * n + 4 * f + 5 * f)  # primitives once, normal + area, flux * |S|
    if kernel == "k_prim":
        return 8.0 * (5 * n + 5 * n)
    if kernel == "k_nodes":
        # face contributions of I and J, of K outside the blade rows; stage
        # input, output, dt, volume, bladePresent and the blockage gradient (3)
        # at every node; rotation (cos, sin, r) and the BFM fields (9 of Hall)
        # at blade-row nodes only (the stage input is U^n: read once); the
        # timed launch (stage 0) also stores the next stage's primitives (5,
        # the pass k_prim made in every stage before; JST adds pressure and
        # spectral radius)
        bf = blade_fraction(case)
        contrib = faces["I"] + faces["J"] + (faces["K"] * (1.0 - bf) if nk > 1 else 0.0)
        prim_next = 5 + (2 if case.settings.get("CONVECTION_SCHEME", "").upper() == "JST" else 0)
        return 8.0 * (5 * contrib + 2 * 5 * n + 2 * n + 4 * n + (3 + 9) * n * bf + prim_next * n)
    if kernel == "k_dt":
        return 8.0 * (5 * n + 12 * n + n)
    return 0.0


SPLIT_STAGE = ("k_prim", "k_faces_I", "k_faces_J", "k_faces_K", "k_nodes", "k_periodic")
FUSED_STAGE = ("k_stage", "k_periodic")
STAGE_KERNEL_NAMES = {"split": "split (k_prim, k_faces, k_nodes)", "fused": "fused (k_stage)",
                      "persistent": "persistent (k_run, 32 iterations per launch)"}


def calls_per_iteration(case, kernel: str, fused: bool = False) -> int:
    """How often per iteration each kernel kind of ctbfm_profile_kernels runs
    (its timing covers all launches of one call), for the fused or the split
    stage."""
    s = case.n_stages
    if kernel == "k_prim":  # later stages read the primitives the node kernels store
        return 0 if fused else 1
    if kernel in SPLIT_STAGE + FUSED_STAGE:
        return s if kernel in (FUSED_STAGE if fused else SPLIT_STAGE) else 0
    return {"k_dt": 1, "k_pre": 1, "k_finalize": 1, "k_bint": 0}.get(kernel, 0)


def launches_per_iteration(case, kernel: str, fused: bool = False) -> int:
    """Kernel launches per iteration of each kind: the end faces of K lines
    (and of J lines whose rows do not fill whole warps) run in a launch of
    their own."""
    ni, nj, nk = case.shape
    n = calls_per_iteration(case, kernel, fused)
    if kernel == "k_faces_K" and nk >= 3:
        return 2 * n
    if kernel == "k_faces_J" and nj >= 3 and nk % 32 != 0:
        return 2 * n
    return n


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def traffic_table():
    try:
        return json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
    except (OSError, ValueError):
        return {}


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    from cturbobfm_b200 import Solver
    from cturbobfm_b200.replicas import max_over_ranks, whole_job_rate

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    case = make_case()
    if args.stage != "auto":  # a fixed stage (profiler runs: ncu's serialised timing would steer the autotuner)
        case = case.with_settings(GPU_STAGE_FUSION=args.stage)
    tmp = tempfile.TemporaryDirectory()
    ini = case.write(tmp.name)
    solver = Solver(ini)
    stream = torch.cuda.Stream(device=dev)
    solver.set_stream(stream.cuda_stream)
    solver.autotune()  # face tiles and stage fusion, before any timed work
    n = case.n_nodes
    stages = case.n_stages

    def barrier():
        if world > 1:
            dist.barrier()

    # warm-up (also captures the CUDA graph)
    solver.enqueue(args.warmup)
    stream.synchronize()
    if solver.status != 0:
        raise RuntimeError(f"workload stopped during warm-up (status {solver.status})")
    it0 = solver.iteration

    # device-timed steps, state resident in HBM
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        solver.enqueue(args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
    ms = ev0.elapsed_time(ev1)
    done = solver.iteration - it0
    if done != args.steps or solver.status != 0:
        raise RuntimeError(f"timed region ran {done} of {args.steps} iterations (status {solver.status})")
    ms_max = max_over_ranks(ms, dev)
    value = whole_job_rate(n * stages * args.steps, world, ms_max)

    u64 = solver.state() if world == 1 else None

    # the same workload in fp32_kahan (float fluxes and state + Kahan term,
    # double norms and integrals), device-timed the same way
    fp32 = None
    if world == 1:
        ini32 = case.with_settings(GPU_PRECISION="fp32_kahan").write(os.path.join(tmp.name, "fp32"))
        with Solver(ini32) as s32:
            s32.set_stream(stream.cuda_stream)
            s32.autotune()
            s32.enqueue(args.warmup)
            stream.synchronize()
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            f0.record(stream)
            s32.enqueue(args.steps)
            f1.record(stream)
            torch.cuda.synchronize()
            ms32 = f0.elapsed_time(f1)
            u32 = s32.state()
            rel = [float(np.abs(u32[v] - u64[v]).max() / np.abs(u64[v]).max()) for v in range(5)]
            v32 = n * stages * args.steps / (ms32 / 1e3)
            b32 = stage_bytes_per_cell(case, 4)
            pk = measured_peaks().get("hbm_gbs", 6650.0)
            mode32, ms32_tuned = s32.stage_kernels()
            fp32 = {"value": v32, "unit": UNIT, "ms_per_step": ms32 / args.steps, "status": s32.status,
                    "stage_kernels": STAGE_KERNEL_NAMES[mode32], "stage_autotuned_ms": ms32_tuned,
                    "stage_roofline": {"bytes_per_cell_stage": b32, "achieved": v32 * b32 / 1e9, "peak": pk,
                                       "unit": "GB/s", "frac": v32 * b32 / 1e9 / pk},
                    "speedup_vs_fp64": ms_max / ms32,
                    "state_rel_err_vs_fp64": {"after_iterations": args.warmup + args.steps, "per_field_max": rel}}

    # end to end through the C ABI with pinned host buffers: every step uploads
    # the state, runs one iteration and reads the state and residual norms back
    host = torch.empty((5, n), dtype=torch.float64, pin_memory=True)
    hnp = host.numpy()
    solver.state(out=hnp)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        solver.set_state(hnp)
        solver.enqueue(1)
        solver.state(out=hnp)
        solver.lognorm()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_value = whole_job_rate(n * stages * args.steps, world, max_over_ranks(e0.elapsed_time(e1), dev))

    # per-kernel device times (CUDA events on the launching stream)
    prof = solver.profile_kernels(reps=10)
    mode, _ = solver.stage_kernels()
    fused = mode == "fused"
    shares = {k: prof[k] * calls_per_iteration(case, k, fused) for k in prof}
    total = sum(shares.values()) or 1.0
    dominant = max(shares, key=shares.get)
    peaks = measured_peaks()
    peak = peaks.get("hbm_gbs", 6650.0)
    alg = algorithmic_bytes(case, dominant)
    achieved = alg / (prof[dominant] / 1e3) / 1e9 if prof[dominant] > 0 else 0.0
    traffic = traffic_table().get(dominant)
    if mode == "persistent":  # k_set_limits and one k_run per 32 iterations
        launches = 1 + -(-args.steps // 32)
    else:
        launches = args.steps * (1 + sum(launches_per_iteration(case, k, fused) for k in prof if prof[k] > 0))
    clk = clocks.summary()

    if world > 1:
        if dist.is_initialized():
            dist.barrier()
            dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {
            "workload": WORKLOAD, "nodes": n, "stages_per_step": stages,
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "l2": f"inputs larger than L2: device working set {solver_bytes(solver, case) / 2**20:.0f} MiB > 126 MiB",
            "face_tiles_autotuned": list(solver.info().face_tile),
            "stage_autotuned_ms": solver.stage_kernels()[1],
        },
        "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 5 * 8 * n,
                "d2h_bytes_per_step": 5 * 8 * n + 5 * 8},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "algorithmic_bytes_per_launch": alg, "launch_ms": prof[dominant],
                     "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
        "kernel_ms": prof, "kernel_share": {k: v / total for k, v in shares.items() if v > 0},
        "stage_kernels": "fused (k_stage)" if fused else "split (k_prim, k_faces, k_nodes)",
    }
    # stage-level view: the compulsory bytes of a fused stage per cell-stage
    # (5 words read U(k-1), 5 read U^n, 5 written, dt/V, 3 face vectors of
    # 3 FP64 words, 14 BFM words at blade-row nodes) at the measured
    # cell-stage rate
    b_stage = stage_bytes_per_cell(case)
    line["stage_roofline"] = {"bytes_per_cell_stage": b_stage, "achieved": value * b_stage / 1e9,
                              "peak": peak, "unit": "GB/s", "frac": value * b_stage / 1e9 / peak}
    if fp32:
        line["fp32_kahan"] = fp32
    if world == 1 and not args.no_map:
        # the north-star workload beside the annulus line: converged
        # op-points/hour of the batched compressor map (fp32_kahan and FP64),
        # the plain FP64 path and the reference build on the host cores
        m = map_line(args)
        nc = m.pop("not_converged")
        m["not_converged_count"] = len(nc)
        m["not_converged_first"] = nc[:5]
        line["map"] = m
    if world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(case, args.cpu_iters, one_core_iters=3)
        line["cpu_baseline"] = {k: base[k] for k in ("value", "unit", "cores", "kind", "sample", "value_1_core",
                                                     "sample_1_core") if k in base}
    print(json.dumps(line), flush=True)
    solver.close()


# ------------------------------------------------------------ compressor map
MAP_METRIC = "converged op-points/hour"
MAP_WORKLOAD = ("compressor map: {n} axisymmetric BFM instances (Hall, MAP_ROWS stage), NI x NJ ~ U{64..256} x "
                "U{24..96}, p_out/pt_in ~ U[{p0},{p1}], speed ~ U[{s0},{s1}], PCG64 seed 20261203, JST, RK4, local dt "
                "CFL 2.2, outlet ramp 2000 its, residual drop {drop} orders")


def map_workload(args) -> str:
    return (MAP_WORKLOAD.replace("{drop}", str(args.map_drop)).replace("{n}", str(args.map_n))
            .replace("{p0}", f"{args.map_pratio[0]:.2f}").replace("{p1}", f"{args.map_pratio[1]:.2f}")
            .replace("{s0}", f"{args.map_speed[0]:.2f}").replace("{s1}", f"{args.map_speed[1]:.2f}"))


def _map_launches_per_iteration(case, mode: str) -> float:
    # k_bint, k_dt, k_pre, per stage k_stage (fused) or k_faces I + k_faces J +
    # k_nodes (split; k_prim in stage 0 only), k_finalize; one k_run per 32
    # iterations (persistent)
    if mode == "persistent":
        return 1.0 / 32
    return 3 + (case.n_stages if mode == "fused" else 3 * case.n_stages + 1) + 1


def _solve_batched(solvers, stream, chunk: int, n_iter: int, case):
    """Runs the batch to convergence (or N_ITERATIONS) in chunks, dropping
    finished members from the batch whenever a quarter of it has finished;
    each batch is autotuned (face tiles, stage fusion) before it runs.
    Returns (per-member status, iterations, launches, the first batch's
    stage kernels and tuned stage times)."""
    import numpy as np

    from cturbobfm_b200 import Batch

    m = len(solvers)
    status = np.zeros(m, np.int32)
    iters = np.zeros(m, np.int64)
    active = list(range(m))
    launches = 0
    first = None
    batches = []
    while active:
        t_set = time.perf_counter()
        with Batch([solvers[i] for i in active]) as b:
            b.set_stream(stream.cuda_stream)
            b.autotune()
            mode, stage_ms = b.stage_kernels()
            batches.append({"members": len(active), "stage_kernels": mode,
                            "setup_s": round(time.perf_counter() - t_set, 4)})
            if first is None:
                first = {"stage_kernels": STAGE_KERNEL_NAMES[mode], "stage_autotuned_ms": stage_ms}
            per_iteration = _map_launches_per_iteration(case, mode)
            start = len(active)
            while True:
                b.step(chunk)
                st = b.status()
                launches += int(np.ceil(chunk * per_iteration)) + 4  # + k_set_limits and three control gathers
                for j, i in enumerate(active):
                    status[i] = st["status"][j]
                    iters[i] = st["iterations"][j]
                done = [i for i in active if status[i] != 0 or iters[i] >= n_iter]
                if len(done) * 4 >= start or len(done) == len(active):
                    break
        active = [i for i in active if not (status[i] != 0 or iters[i] >= n_iter)]
    first["batches"] = batches
    return status, iters, launches, first


def _solve_fp32_then_fp64(solvers, stream, chunk: int, n_iter: int, case, drop: int, stall: int,
                          promote: float = 1.0):
    """The precision pattern on the map: every member runs batched in
    fp32_kahan until it is within one order of its residual drop (best_drop
    >= drop - 1), stops progressing (best_drop grew by less than 0.05 orders
    in `stall` iterations) or finishes; the members that stopped without
    finishing then continue from their current state in FP64
    (ctbfm_promote_fp64), batched, to convergence. Float carries the bulk of
    the iterations; FP64 takes the last order, where the float residual
    reaches its rounding floor, so the convergence test and the converged
    state are FP64's. Returns (status, iterations, launches, stage kernels,
    promoted count, FP64 iterations)."""
    import numpy as np

    from cturbobfm_b200 import Batch

    m = len(solvers)
    status = np.zeros(m, np.int32)
    iters = np.zeros(m, np.int64)
    mark = np.zeros(m)       # best_drop at the last 0.05-order progress
    mark_it = np.zeros(m, np.int64)
    ready = np.zeros(m, bool)
    launches = 0
    first = None
    batches = []
    active = list(range(m))
    # phase A: float
    while active:
        t_set = time.perf_counter()
        with Batch([solvers[i] for i in active]) as b:
            b.set_stream(stream.cuda_stream)
            b.autotune()
            mode, stage_ms = b.stage_kernels()
            batches.append({"members": len(active), "stage_kernels": mode,
                            "setup_s": round(time.perf_counter() - t_set, 4)})
            if first is None:
                first = {"stage_kernels": STAGE_KERNEL_NAMES[mode], "stage_autotuned_ms": stage_ms}
            per_iteration = _map_launches_per_iteration(case, mode)
            start = len(active)
            while True:
                b.step(chunk)
                st = b.status()
                launches += int(np.ceil(chunk * per_iteration)) + 4
                for j, i in enumerate(active):
                    status[i] = st["status"][j]
                    iters[i] = st["iterations"][j]
                    bd = st["best_drop"][j]
                    if bd >= mark[i] + 0.05:
                        mark[i], mark_it[i] = bd, iters[i]
                    if bd >= drop - promote or iters[i] - mark_it[i] >= stall:
                        ready[i] = True
                out = [i for i in active if status[i] != 0 or iters[i] >= n_iter or ready[i]]
                if len(out) * 4 >= start or len(out) == len(active):
                    break
        active = [i for i in active if not (status[i] != 0 or iters[i] >= n_iter or ready[i])]
    # phase B: FP64 to convergence
    promote = [i for i in range(m) if status[i] == 0 and iters[i] < n_iter]
    it_a = iters.copy()
    t_pro = time.perf_counter()
    for i in promote:
        solvers[i].promote_fp64()
    first["promote_s"] = round(time.perf_counter() - t_pro, 3)
    first["batches"] = batches
    if promote:
        s_b, i_b, l_b, kb = _solve_batched([solvers[i] for i in promote], stream, chunk, n_iter, case)
        for j, i in enumerate(promote):
            status[i], iters[i] = s_b[j], i_b[j]
        launches += l_b
        first["batches_fp64"] = kb["batches"]
    fp64_iters = int(sum(iters[i] - it_a[i] for i in promote))
    return status, iters, launches, first, len(promote), fp64_iters


def _serve_map(cases32, chunk: int, stall: int, promote: float = 1.0, host_threads: int = 8):
    """The precision pattern through the serving API: every instance
    submitted from memory (ctbfm_server_submit_case) at once to a Server
    that prepares them on host threads, admits them as they are ready, runs
    the fp32_kahan solves and the solves it moved to FP64 (within one order
    of the residual drop, or stalled for `stall` iterations) as two batches
    on two streams that overlap on the device, and retires each at
    convergence. Wall time from the first submission to the last result,
    host preparation and device set-up included."""
    import numpy as np

    from cturbobfm_b200 import Server

    w0 = time.perf_counter()
    res = {}
    with Server(chunk=chunk, stall_window=stall, host_threads=host_threads, promote_orders=promote) as srv:
        ids = [srv.submit_case(c) for c in cases32]
        while len(res) < len(ids) and time.perf_counter() - w0 < 1200:
            active, _ = srv.pump()
            for r in srv.results():
                res[r["id"]] = r
            if not active:
                time.sleep(0.001)
        stats = srv.stats()
    sec = time.perf_counter() - w0
    rs = [res.get(i) for i in ids]
    status = np.array([r["status"] if r else -1 for r in rs])
    turbo = np.array([r["turbo"] if r else [np.nan] * 4 for r in rs])
    iters = np.array([r["iterations"] if r else 0 for r in rs])
    conv = int((status == 1).sum())
    return {"seconds": sec, "converged": conv, "diverged": int((status == 2).sum()),
            "points_per_hour": conv / sec * 3600.0, "status": status, "turbo": turbo, "iterations": iters,
            "errors": int(sum(1 for r in rs if r is None or r["error"])),
            "server_stats": {k: (round(v, 3) if isinstance(v, float) else v) for k, v in stats.items()}}


MAPSTEP_METRIC = "batched map iteration time"


def run_mapstep(args):
    """One batched chunk of the compressor map: the first --map-n instances of
    the map workload in one batch (--map-precision, stage kernels forced with
    --stage or autotuned), --warmup untimed iterations, then --steps timed
    iterations between cudaProfilerStart / Stop (a profiler run with
    --profile-from-start off records exactly those launches). Prints the
    device time per batched iteration."""
    import torch

    from cturbobfm_b200 import Batch, Solver, cases

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    cs = cases.compressor_map(n=args.map_n, precision=args.map_precision, drop=args.map_drop)
    tmp = tempfile.TemporaryDirectory()
    solvers = []
    for i, c in enumerate(cs):
        c = c.with_settings(GPU_STAGE_FUSION=args.stage)
        d = os.path.join(tmp.name, str(i))
        os.makedirs(d)
        solvers.append(Solver(c.write(d)))
    stream = torch.cuda.Stream()
    nodes = sum(c.n_nodes for c in cs)
    try:
        with Batch(solvers) as b:
            b.set_stream(stream.cuda_stream)
            b.autotune()
            b.step(args.warmup)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.profiler.start()
            e0.record(stream)
            b.enqueue(args.steps)
            e1.record(stream)
            torch.cuda.synchronize()
            torch.cuda.profiler.stop()
            ms = e0.elapsed_time(e1) / args.steps
            mode, stage_ms = b.stage_kernels()
    finally:
        for s in solvers:
            s.close()
    if rank != 0:
        return
    print(json.dumps({
        "metric": MAPSTEP_METRIC, "value": ms, "unit": "ms", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.map_precision == "fp64" else "f32+kahan (f64 integrals)", "data": "synthetic",
        "config": {"workload": f"the first {args.map_n} instances of the compressor map, one batch, "
                               f"{args.map_precision}", "nodes": nodes,
                   "node_stage_per_s": nodes * 4 / (ms / 1e3), "stage_kernels": mode, "stage_autotuned_ms": stage_ms},
    }))


def map_cpu_baseline(inis, iterations, n_iter: int):
    """Converged op-points/hour of the reference build on the host cores: one
    single-threaded process per instance, all at once (the way the
    reference's python/Run_All_Cases.py fans out), each timed over n_iter
    iterations with set-up subtracted; points/hour then follows from the
    iteration counts each instance needs to converge (the same algorithm,
    measured on the GPU FP64 path)."""
    from oracle import oracle

    if not os.path.exists(oracle.REF_CLI):
        return None
    env = dict(os.environ, OMP_NUM_THREADS="1")

    def launch(ini, n):
        d = os.path.dirname(ini)
        lines = [l for l in open(ini).read().splitlines() if not l.startswith("N_ITERATIONS")]
        open(ini, "w").write("\n".join(lines + [f"N_ITERATIONS = {n}"]) + "\n")
        return subprocess.Popen([oracle.REF_CLI, "input.ini"], cwd=d, stdout=subprocess.DEVNULL,
                                stderr=subprocess.DEVNULL, env=env)

    def wall(n):
        t0 = time.perf_counter()
        ps = [launch(ini, n) for ini in inis]
        for p in ps:
            p.wait(timeout=900)
        return time.perf_counter() - t0

    t1 = wall(1)
    tn = wall(n_iter + 1)
    per_round = (tn - t1) / n_iter  # seconds per iteration of all sampled instances at once
    # all sampled instances run concurrently, one per core: the batch of them
    # takes as long as the slowest, which needs max(iterations) iterations
    cores = len(inis)
    seconds = per_round * max(iterations)
    return {"value": len(inis) / seconds * 3600.0, "unit": "points/hour", "cores": cores, "kind": "reference",
            "sample": f"{len(inis)} map instances as concurrent single-threaded reference processes, "
                      f"{n_iter} iterations timed (set-up subtracted), scaled to the iterations each needs to "
                      f"converge"}


def run_map(args):
    print(json.dumps(map_line(args)), flush=True)


def map_line(args):
    """The compressor-map measurement (batched fp32_kahan, batched FP64, the
    plain FP64 path one instance at a time, the reference build on the host
    cores) as one JSON-ready dict."""
    import numpy as np
    import torch

    from cturbobfm_b200 import Solver, cases

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    cs32 = cases.compressor_map(n=args.map_n, precision="fp32_kahan", drop=args.map_drop,
                                p_ratio_range=tuple(args.map_pratio), speed_range=tuple(args.map_speed))
    n_iter = int(cs32[0].settings["N_ITERATIONS"])
    tmp = tempfile.TemporaryDirectory()

    def write(cs, tag):
        out = []
        for c in cs:
            d = os.path.join(tmp.name, tag, c.name)
            os.makedirs(d)
            out.append(c.write(d))
        return out

    inis32 = write(cs32, "fp32")
    cs64 = [c.with_settings(GPU_PRECISION="fp64") for c in cs32]
    inis64 = write(cs64, "fp64")
    nodes = np.array([c.n_nodes for c in cs32])
    stream = torch.cuda.Stream()
    results = {}
    with ClockSampler(local) as clocks:
        arms = [("batched_fp32_kahan", inis32), ("batched_fp64", inis64)]
        if args.map_pure_fp32:
            arms.append(("batched_fp32_only", inis32))
        for arm, inis in arms:
            if arm == "batched_fp64" and args.map_skip_fp64_batch:
                continue
            w0 = time.perf_counter()
            solvers = [Solver(p) for p in inis]
            setup = time.perf_counter() - w0
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            promoted, fp64_iters = 0, 0
            if arm == "batched_fp32_kahan":
                status, iters, launches, kern, promoted, fp64_iters = _solve_fp32_then_fp64(
                    solvers, stream, args.map_chunk, n_iter, cs32[0], args.map_drop, args.map_stall,
                    args.map_promote)
            else:
                status, iters, launches, kern = _solve_batched(solvers, stream, args.map_chunk, n_iter, cs32[0])
            e1.record(stream)
            torch.cuda.synchronize()
            sec = e0.elapsed_time(e1) / 1e3
            w1 = time.perf_counter()
            turbo = np.array([s.turbo()[1] for s in solvers])
            readback = time.perf_counter() - w1
            bytes_up = sum(int(s.info().device_bytes) for s in solvers)
            for s in solvers:
                s.close()
            conv = int((status == 1).sum())
            results[arm] = {"seconds": sec, "setup_seconds": setup, "readback_seconds": readback,
                            "converged": conv, "diverged": int((status == 2).sum()),
                            "points_per_hour": conv / sec * 3600.0,
                            "e2e_points_per_hour": conv / (setup + sec + readback) * 3600.0,
                            "iterations": iters.tolist(), "turbo": turbo, "status": status,
                            "node_stage_per_s": float((nodes * iters).sum() * 4 / sec), "launches": launches,
                            "device_bytes": bytes_up, "promoted_to_fp64": promoted,
                            "fp64_iteration_share": fp64_iters / max(1, int(iters.sum())), **kern}
        if not args.map_skip_served:
            results["served_fp32_kahan"] = _serve_map(cs32, args.map_chunk, args.map_stall, args.map_promote)
        # the plain FP64 path: one drop-in solver at a time, to convergence
        sample = list(range(min(args.map_plain, len(inis64))))
        plain_sec, plain_conv, plain = 0.0, 0, []
        for i in sample:
            with Solver(inis64[i]) as s:
                s.set_stream(stream.cuda_stream)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                try:
                    s.solve()
                except Exception:
                    pass
                e1.record(stream)
                torch.cuda.synchronize()
                plain_sec += e0.elapsed_time(e1) / 1e3
                plain_conv += int(s.status == 1)
                plain.append((s.status, s.iteration, s.turbo()[1]))
    clk = clocks.summary()
    r32 = results["batched_fp32_kahan"]
    plain_pph = plain_conv / plain_sec * 3600.0 if plain_sec > 0 else None
    # accuracy of the batched FP32 results against the plain FP64 solves of the same instances
    err_mf, err_pr = [], []
    for j, i in enumerate(sample):
        st, it, tb = plain[j]
        if st == 1 and r32["status"][i] == 1:
            err_mf.append(abs(r32["turbo"][i][0] - tb[0]) / abs(tb[0]))
            err_pr.append(abs(r32["turbo"][i][1] - tb[1]) / abs(tb[1]))
    line = {
        "metric": MAP_METRIC, "value": r32["points_per_hour"], "unit": "points/hour", "n_gpus": 1,
        "steps": len(cs32), "warmup": 0, "ms_per_step": r32["seconds"] * 1e3 / max(1, len(cs32)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+kahan (f64 integrals)",
        "data": "synthetic",
        "config": {"workload": map_workload(args), "instances": len(cs32),
                   "nodes_total": int(nodes.sum()),
                   "chunk_iterations": args.map_chunk, "l2": "inputs larger than L2 (working set > 126 MiB)"},
        "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
        # end to end: the serving API from memory (host preparation, uploads,
        # scheduling and results included, wall clock) when it ran, else the
        # batched arm with its set-up and read-back
        "e2e": {"value": (results["served_fp32_kahan"]["points_per_hour"] if "served_fp32_kahan" in results
                          else r32["e2e_points_per_hour"]), "unit": "points/hour",
                "via": ("ctbfm_server_submit_case, wall clock" if "served_fp32_kahan" in results
                        else "ctbfm_create_from_ini + ctbfm_batch_*, set-up and read-back included"),
                "h2d_bytes_per_step": r32["device_bytes"] / len(cs32), "d2h_bytes_per_step": 6 * 8 + 4 * 8},
        "gpu_launches": r32["launches"],
        "batched_fp32_kahan": {k: r32[k] for k in ("seconds", "setup_seconds", "converged", "diverged",
                                                   "points_per_hour", "node_stage_per_s", "stage_kernels",
                                                   "stage_autotuned_ms", "promoted_to_fp64",
                                                   "fp64_iteration_share", "promote_s", "batches",
                                                   "batches_fp64") if k in r32},
        "precision_pattern": (f"fp32_kahan for every instance until it is within {args.map_promote:g} orders of the "
                              f"residual drop or stalls for {args.map_stall} iterations, then the same solve continued "
                              "in FP64 from "
                              "its current state to convergence (FP64 convergence test and converged state)"),
        "plain_fp64": {"points_per_hour": plain_pph, "instances": len(sample), "converged": plain_conv,
                       "seconds": plain_sec, "iterations": [p[1] for p in plain]},
        "speedup_vs_plain_fp64": (r32["points_per_hour"] / plain_pph) if plain_pph else None,
        "speedup_batched_fp64_vs_plain_fp64": ((results["batched_fp64"]["points_per_hour"] / plain_pph)
                                               if plain_pph and "batched_fp64" in results else None),
        "fp32_vs_plain_fp64_rel_err": {"massflow_max": max(err_mf) if err_mf else None,
                                       "pr_tt_max": max(err_pr) if err_pr else None, "instances": len(err_mf)},
        "iterations_fp32": {"min": int(min(r32["iterations"])), "median": float(np.median(r32["iterations"])),
                            "max": int(max(r32["iterations"]))},
    }
    if "served_fp32_kahan" in results:
        rs = results["served_fp32_kahan"]
        line["served_fp32_kahan"] = {k: rs[k] for k in ("seconds", "converged", "diverged", "points_per_hour",
                                                         "errors", "server_stats")}
        line["served_fp32_kahan"]["how"] = ("ctbfm_server_submit_case of all instances at t = 0, chunk "
                                            f"{args.map_chunk}, float and FP64 batches on two streams; wall "
                                            "time from the first submission to the last result")
        line["served_fp32_kahan"]["speedup_vs_plain_fp64"] = rs["points_per_hour"] / plain_pph if plain_pph else None
        if "batched_fp64" in results:
            r64 = results["batched_fp64"]
            both = (rs["status"] == 1) & (r64["status"] == 1)
            if both.any():
                emf = np.abs(rs["turbo"][both, 0] - r64["turbo"][both, 0]) / np.abs(r64["turbo"][both, 0])
                epr = np.abs(rs["turbo"][both, 1] - r64["turbo"][both, 1]) / np.abs(r64["turbo"][both, 1])
                line["served_fp32_kahan"]["vs_batched_fp64_rel_err"] = {
                    "massflow_max": float(emf.max()), "pr_tt_max": float(epr.max()),
                    "above_1e-4": int(((emf > 1e-4) | (epr > 1e-4)).sum()), "instances": int(both.sum())}
    if "batched_fp32_only" in results:
        r = results["batched_fp32_only"]
        line["batched_fp32_only"] = {k: r[k] for k in ("seconds", "converged", "diverged", "points_per_hour",
                                                        "node_stage_per_s")}
    if "batched_fp64" in results:
        r64 = results["batched_fp64"]
        line["batched_fp64"] = {k: r64[k] for k in ("seconds", "converged", "diverged", "points_per_hour",
                                                    "node_stage_per_s", "stage_kernels", "stage_autotuned_ms")}
        both = (r32["status"] == 1) & (r64["status"] == 1)
        if both.any():
            emf = np.abs(r32["turbo"][both, 0] - r64["turbo"][both, 0]) / np.abs(r64["turbo"][both, 0])
            epr = np.abs(r32["turbo"][both, 1] - r64["turbo"][both, 1]) / np.abs(r64["turbo"][both, 1])
            dit = np.abs(np.array(r32["iterations"])[both] - np.array(r64["iterations"])[both])
            line["batched_fp32_vs_fp64_rel_err"] = {
                "massflow": {"p50": float(np.median(emf)), "p90": float(np.percentile(emf, 90)),
                             "max": float(emf.max()), "above_1e-4": int((emf > 1e-4).sum())},
                "pr_tt": {"p50": float(np.median(epr)), "p90": float(np.percentile(epr, 90)),
                          "max": float(epr.max()), "above_1e-4": int((epr > 1e-4).sum())},
                "convergence_iteration_difference": {"median": float(np.median(dit)), "max": int(dit.max())},
                "instances": int(both.sum())}
    line["not_converged"] = [
        {"name": cs32[i].name, "shape": list(cs32[i].shape[:2]),
         "p_ratio": round(float(cs32[i].patches[1].values[0]) / 101325.0, 4),
         "speed": float(cs32[i].settings["ROTATIONAL_SPEED_SCALING_FACTOR"]),
         "status": int(r32["status"][i]), "iterations": int(r32["iterations"][i])}
        for i in range(len(cs32)) if r32["status"][i] != 1]
    if not args.no_cpu_baseline:
        conv_plain = [j for j, p in enumerate(plain) if p[0] == 1]
        if conv_plain:
            base = map_cpu_baseline([inis64[sample[j]] for j in conv_plain], [plain[j][1] for j in conv_plain],
                                    args.cpu_iters * 10)
            if base:
                line["cpu_baseline"] = base
    return line


# --------------------------------------------------------------- real gas
REALGAS_WORKLOAD = ("real-gas CO2 annulus 256x96x128 (3.1M nodes), synthetic van der Waals table 60x60 per section "
                    "(1e5-1e7 Pa, 200-600 K), inlet 8.0 MPa / 310 K, Hall 15000 rpm, Roe+MUSCL(min mod), RK3, "
                    "CFL 1.0; fp32_kahan bulk with FP64 table inversions")


VISCOUS_WORKLOAD = ("laminar viscous annulus duct 160x48x64 (491520 nodes, no blade rows), outlet 0.95 pt, hub and "
                    "shroud no-slip walls, Sutherland air, JST, RK4, CFL 1.2; the same duct with inviscid walls "
                    "timed beside it")


def run_viscous(args):
    """The viscous path: the duct with no-slip walls against the same duct
    with inviscid walls (FP64 and fp32_kahan), device-timed with CUDA events
    on the solver's stream. The per-stage time difference is the cost of the
    viscous kernels (k_grad, three k_vfaces) plus the viscous terms of
    k_nodes / k_dt; its roofline fraction counts only the two new kernels'
    algorithmic bytes, so it is a lower bound for them."""
    import torch

    from cturbobfm_b200 import Solver, cases

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    tmp = tempfile.TemporaryDirectory()
    stream = torch.cuda.Stream()
    arms = {}
    with ClockSampler(local) as clocks:
        for prec in ("fp64", "fp32_kahan"):
            for visc in (True, False):
                c = cases.viscous_annulus(precision=prec, viscous=visc)
                ini = c.write(os.path.join(tmp.name, f"{prec}_{visc}"))
                with Solver(ini) as s:
                    s.set_stream(stream.cuda_stream)
                    s.enqueue(args.warmup)
                    stream.synchronize()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    torch.cuda.synchronize()
                    e0.record(stream)
                    s.enqueue(args.steps)
                    e1.record(stream)
                    torch.cuda.synchronize()
                    ms = e0.elapsed_time(e1)
                    if s.status != 0:
                        raise RuntimeError(f"viscous workload stopped (status {s.status})")
                    arms[(prec, visc)] = {"ms": ms / args.steps, "n": c.n_nodes, "stages": c.n_stages,
                                          "bytes": int(s.info().device_bytes)}
    clk = clocks.summary()
    a = arms[("fp64", True)]
    n, st, K = a["n"], a["stages"], args.steps
    ni, nj, nk = 160, 48, 64
    nf = (ni + 1) * nj * nk + ni * (nj + 1) * nk + ni * nj * (nk + 1)
    # k_grad 8*(5N + 9N + 6N + N + 12N) + k_vfaces 8*(3*(5N + 12N) + 8F) bytes per stage (FP64)
    alg = 8 * (33 * n) + 8 * (3 * 17 * n + 8 * nf)
    extra_s = (a["ms"] - arms[("fp64", False)]["ms"]) / st / 1e3
    peaks = measured_peaks()
    peak = peaks.get("hbm_gbs", 6650.0)
    peak_kind = "measured" if "hbm_gbs" in peaks else "fallback"
    achieved = alg / extra_s / 1e9 if extra_s > 0 else None
    line = {
        "metric": METRIC, "value": n * st / (a["ms"] / 1e3), "unit": UNIT, "n_gpus": 1, "steps": K,
        "warmup": args.warmup, "ms_per_step": a["ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": VISCOUS_WORKLOAD, "nodes": n, "stages_per_step": st,
                   "l2": f"inputs larger than L2: device working set {a['bytes'] / 2**20:.0f} MiB > 126 MiB"},
        "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
        "inviscid_duct_fp64": {"ms_per_step": arms[("fp64", False)]["ms"]},
        "fp32_kahan": {"viscous_ms_per_step": arms[("fp32_kahan", True)]["ms"],
                       "inviscid_ms_per_step": arms[("fp32_kahan", False)]["ms"]},
        "viscous_terms_roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                   "frac": achieved / peak if achieved else None, "peak_source": peak_kind,
                                   "algorithmic_bytes_per_stage": alg,
                                   "note": "k_grad + k_vfaces bytes over the viscous-minus-inviscid stage time"},
    }
    print(json.dumps(line), flush=True)


def run_realgas(args):
    import numpy as np
    import torch

    from cturbobfm_b200 import Solver, cases

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    tmp = tempfile.TemporaryDirectory()
    stream = torch.cuda.Stream()
    arms = {}
    with ClockSampler(local) as clocks:
        for prec in ("fp32_kahan", "fp64"):
            c = cases.realgas_annulus(precision=prec)
            ini = c.write(os.path.join(tmp.name, prec))
            with Solver(ini) as s:
                s.set_stream(stream.cuda_stream)
                s.enqueue(args.warmup)
                stream.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record(stream)
                s.enqueue(args.steps)
                e1.record(stream)
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1)
                if s.status != 0:
                    raise RuntimeError(f"real-gas workload stopped (status {s.status})")
                arms[prec] = {"ms": ms, "state": s.state(), "turbo": s.turbo()[1], "n": c.n_nodes,
                              "stages": c.n_stages, "bytes": int(s.info().device_bytes)}
    clk = clocks.summary()
    a, b = arms["fp32_kahan"], arms["fp64"]
    n, st, K = a["n"], a["stages"], args.steps
    rel = [float(np.abs(a["state"][v] - b["state"][v]).max() / np.abs(b["state"][v]).max()) for v in range(5)]
    line = {
        "metric": METRIC, "value": n * st * K / (a["ms"] / 1e3), "unit": UNIT, "n_gpus": 1, "steps": K,
        "warmup": args.warmup, "ms_per_step": a["ms"] / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+kahan (f64 table inversions, integrals)", "data": "synthetic",
        "config": {"workload": REALGAS_WORKLOAD, "nodes": n, "stages_per_step": st,
                   "l2": f"inputs larger than L2: device working set {a['bytes'] / 2**20:.0f} MiB > 126 MiB"},
        "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
        "fp64": {"value": n * st * K / (b["ms"] / 1e3), "ms_per_step": b["ms"] / K},
        "fp32_vs_fp64": {"after_iterations": args.warmup + K, "state_rel_err_per_field": rel,
                         "massflow_rel_err": float(abs(a["turbo"][0] - b["turbo"][0]) / abs(b["turbo"][0])),
                         "pr_tt_rel_err": float(abs(a["turbo"][1] - b["turbo"][1]) / abs(b["turbo"][1]))},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- serving
SERVE_WORKLOAD = ("serving: Poisson arrivals, 70% axisymmetric compressor-map requests (NI x NJ ~ U{64..256} x "
                  "U{24..96}; a fifth of them throttle + Greitzer plenum requests on U{64..128} x U{24..48}, "
                  "kt ~ U[0.8,1.0], B ~ U[0.1,0.5] mapped to GREITZER_PLENUM_VOLUME, speed ~ U[0.85,0.90], fixed dt) "
                  "and 30% 3-D annuli (U{96..160} x U{32..48} x U{32..64}), MAP_ROWS stage, static outlets "
                  "p_out/pt_in ~ U[1.00,1.20], speed ~ U[0.85,1.00], JST RK4 CFL 2.2, drop 3 orders, fp32_kahan "
                  "(float solves move to FP64 only with --serve-stall-window > 0)")


def warm_start_solution(root):
    """The converged nominal operating point of the serving mix (the map stage
    on a 128 x 48 meridional grid, p_out/pt_in 1.10, speed 0.925, FP64), as a
    volume CSV for the requests' restarts. Solved before the timed region."""
    from cturbobfm_b200 import Solver, cases

    c = cases.meridional(ni=128, nj=48, p_ratio=1.10, speed=0.925, cfl=2.2, drop=3, rows=cases.MAP_ROWS,
                         ramp=2000, n_iter=40000, name="nominal")
    d = os.path.join(root, "nominal")
    t0 = time.perf_counter()
    with Solver(c.write(d)) as s:
        s.solve()
        status, its = s.status, s.iteration
        path = s.write_solution(os.path.join(d, "nominal.csv"))
    return {"path": path, "status": status, "iterations": its, "seconds": time.perf_counter() - t0}


def run_serve(args):
    import numpy as np
    import torch

    from cturbobfm_b200 import Server, cases

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    tmp = tempfile.TemporaryDirectory()
    per_rate = {}
    warm = None
    if args.serve_warm:
        warm = warm_start_solution(tmp.name)
    with ClockSampler(local) as clocks:
        for rate in args.serve_rates:
            reqs = cases.serving_requests(args.serve_n, rate)
            inis = []
            for t, c in reqs:
                d = os.path.join(tmp.name, f"r{rate}", c.name)
                os.makedirs(d)
                if warm:
                    # start from the converged nominal operating point, mapped onto the
                    # request's grid by the reference's nearest-neighbour restart
                    c = c.with_settings(RESTART_SOLUTION="yes", RESTART_SOLUTION_FILEPATH=warm["path"],
                                        RESTART_TYPE="nearest_neighbor_axisymmetric",
                                        OUTLET_PRESSURE_RAMP_ITERATIONS="0")
                kind = "3d" if c.shape[2] > 1 else ("throttle" if "ENABLE_GREITZER_MODELING" in c.settings else "axisymmetric")
                inis.append((t, c.write(d), c.n_nodes, c.shape[2] > 1, kind))
            res = {}
            with Server(chunk=args.serve_chunk, stall_window=args.serve_stall_window, host_threads=8,
                        max_active_nodes=args.serve_max_nodes) as srv:
                t0 = time.perf_counter()
                nxt = 0
                ids = {}
                while len(res) < len(inis):
                    now = time.perf_counter() - t0
                    while nxt < len(inis) and inis[nxt][0] <= now:
                        ids[srv.submit(inis[nxt][1])] = nxt
                        nxt += 1
                    active, waiting = srv.pump()
                    for r in srv.results():
                        res[ids[r["id"]]] = r
                    if active == 0 and waiting == 0 and nxt < len(inis):
                        time.sleep(max(0.0, min(0.01, inis[nxt][0] - (time.perf_counter() - t0))))
                wall = time.perf_counter() - t0
            lat = np.array([res[i]["t_done"] - res[i]["t_submit"] for i in range(len(inis))])
            conv = np.array([res[i]["status"] == 1 for i in range(len(inis))])
            its = np.array([res[i]["iterations"] for i in range(len(inis))])
            nodes = np.array([x[2] for x in inis])
            is3d = np.array([x[3] for x in inis])
            per_rate[str(rate)] = {
                "requests": len(inis), "converged": int(conv.sum()),
                "diverged": int(sum(res[i]["status"] == 2 for i in range(len(inis)))),
                "errors": int(sum(res[i]["error"] != 0 for i in range(len(inis)))),
                "rerun_fp64": int(sum(res[i]["precision"] == 0 for i in range(len(inis)))),
                "p50_s": float(np.percentile(lat[conv], 50)) if conv.any() else None,
                "p99_s": float(np.percentile(lat[conv], 99)) if conv.any() else None,
                "p50_s_axisymmetric": float(np.percentile(lat[conv & ~is3d], 50)) if (conv & ~is3d).any() else None,
                "p50_s_3d": float(np.percentile(lat[conv & is3d], 50)) if (conv & is3d).any() else None,
                "points_per_hour": float(conv.sum() / wall * 3600.0), "wall_s": wall,
                "arrival_window_s": inis[-1][0],
                "node_stage_per_s": float((nodes * its).sum() * 4 / wall),
                "by_kind": {k: {"requests": int(sum(x[4] == k for x in inis)),
                                "converged": int(sum(conv[i] for i in range(len(inis)) if inis[i][4] == k)),
                                "diverged": int(sum(res[i]["status"] == 2 for i in range(len(inis)) if inis[i][4] == k)),
                                "rerun_fp64": int(sum(res[i]["precision"] == 0 for i in range(len(inis))
                                                      if inis[i][4] == k))}
                            for k in ("axisymmetric", "throttle", "3d")},
            }
    clk = clocks.summary()
    first = per_rate[str(args.serve_rates[0])]
    line = {
        "metric": "serving p50 time-to-converged", "value": first["p50_s"], "unit": "s", "n_gpus": 1,
        "steps": first["requests"], "warmup": 0, "ms_per_step": first["wall_s"] * 1e3 / first["requests"],
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32+kahan (f64 integrals)",
        "data": "synthetic",
        "config": {"workload": SERVE_WORKLOAD, "rates_per_s": args.serve_rates, "requests_per_rate": args.serve_n,
                   "chunk_iterations": args.serve_chunk, "max_active_nodes": args.serve_max_nodes,
                   "stall_window": args.serve_stall_window,
                   "warm_start": (None if not warm else
                                  {"from": "converged nominal point, 128x48 meridional, p_out/pt_in 1.10, speed 0.925",
                                   "restart_type": "nearest_neighbor_axisymmetric", "outlet_ramp": 0,
                                   "nominal_iterations": warm["iterations"], "nominal_status": warm["status"],
                                   "nominal_seconds_untimed": warm["seconds"]}),
                   "clock": "host wall clock from submit to retirement"},
        "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
        "per_rate": per_rate,
    }
    print(json.dumps(line), flush=True)


def solver_bytes(solver, case) -> float:
    # state 3 buffers + face metrics/contributions + node arrays (estimate from sizes)
    ni, nj, nk = case.shape
    n = ni * nj * nk
    f = (ni + 1) * nj * nk + ni * (nj + 1) * nk + ni * nj * (nk + 1)
    return 8.0 * (15 * n + 9 * f + 40 * n)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-iters", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["annulus", "map", "mapstep", "serve", "realgas", "viscous"],
                    default="annulus",
                    help="annulus: the 160x48x64 full-annulus loop (default); map: the batched compressor map; "
                         "serve: continuous batching of arriving requests")
    ap.add_argument("--map-n", type=int, default=256)
    ap.add_argument("--map-precision", choices=["fp64", "fp32_kahan"], default="fp32_kahan",
                    help="mapstep: the batch's GPU_PRECISION")
    ap.add_argument("--stage", choices=["auto", "split", "fused", "persistent"], default="auto",
                    help="GPU_STAGE_FUSION of the timed solvers (mapstep: of every member; default: autotuned)")
    ap.add_argument("--map-drop", type=int, default=4, help="RESIDUALS_DROP_CONVERGENCE of the map instances")
    ap.add_argument("--map-pratio", type=float, nargs=2, default=[1.00, 1.20],
                    help="range of the outlet static pressure over the inlet total pressure")
    ap.add_argument("--map-speed", type=float, nargs=2, default=[0.85, 1.00], help="range of the shaft-speed scaling")
    ap.add_argument("--map-stall", type=int, default=3000,
                    help="float members without 0.05 orders of progress for this many iterations move to FP64")
    ap.add_argument("--map-pure-fp32", action="store_true",
                    help="also run the map in fp32_kahan alone (no FP64 finish)")
    ap.add_argument("--no-map", action="store_true", help="leave the compressor-map object out of the default line")
    ap.add_argument("--map-chunk", type=int, default=250)
    ap.add_argument("--map-promote", type=float, default=1.0,
                    help="float members within this many orders of the residual drop move to FP64")
    ap.add_argument("--map-plain", type=int, default=8, help="instances solved one at a time on the plain FP64 path")
    ap.add_argument("--map-skip-fp64-batch", action="store_true")
    ap.add_argument("--map-skip-served", action="store_true",
                    help="leave out the map run through the serving API")
    ap.add_argument("--serve-rates", type=float, nargs="+", default=[5.0, 20.0, 80.0])
    ap.add_argument("--serve-n", type=int, default=48)
    ap.add_argument("--serve-chunk", type=int, default=100)
    ap.add_argument("--serve-warm", action="store_true",
                    help="serve: every request restarts from one converged nominal operating point")
    ap.add_argument("--serve-stall-window", type=int, default=0,
                    help="serve: > 0 lets the server move stalled float solves to FP64 and re-run diverged ones in FP64")
    ap.add_argument("--serve-max-nodes", type=int, default=1500000,
                    help="grid nodes admitted at once (about what fills the GPU; 0: no limit, every arrival "
                         "shares the device at once)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.workload == "map":
        run_map(args)
    elif args.workload == "mapstep":
        run_mapstep(args)
    elif args.workload == "serve":
        run_serve(args)
    elif args.workload == "realgas":
        run_realgas(args)
    elif args.workload == "viscous":
        run_viscous(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
