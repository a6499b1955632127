"""Benchmark of the explicit residual-and-update loop on the full-annulus
rotor/stator workload (160 x 48 x 64 nodes, Roe + MUSCL van Albada, RK3,
local time step at CFL 1.2, Hall body force, FP64).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

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


def cpu_baseline(case, n_iter: int):
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
    value = case.n_nodes * stages / sec
    return {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"{n_iter} iterations of the same {case.shape[0]}x{case.shape[1]}x{case.shape[2]} case "
                      f"({n_iter * stages} stages), set-up subtracted", "seconds_per_iteration": sec}


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
def algorithmic_bytes(case, kernel: str) -> float:
    """Compulsory DRAM bytes of one launch of a kernel kind (FP64): every input
    read once, every output written once."""
    ni, nj, nk = case.shape
    n = ni * nj * nk
    faces = {"I": (ni + 1) * nj * nk, "J": ni * (nj + 1) * nk, "K": ni * nj * (nk + 1)}
    if kernel.startswith("k_faces_"):
        f = faces[kernel[-1]]
        return 8.0 * (5 * n + 4 * f + 5 * f)  # primitives once, normal + area, flux * |S|
    if kernel == "k_prim":
        return 8.0 * (5 * n + 5 * n)
    if kernel == "k_nodes":
        # face contributions of 3 directions, stage input, U^n, output, dt, volume,
        # rotation (cos, sin, r) and the BFM fields of the node (14)
        return 8.0 * (5 * sum(faces.values()) + 3 * 5 * n + 2 * n + 3 * n + 14 * n)
    if kernel == "k_dt":
        return 8.0 * (5 * n + 12 * n + n)
    return 0.0


def launches_per_iteration(case, kernel: str) -> int:
    s = case.n_stages
    return {"k_faces_I": s, "k_faces_J": s, "k_faces_K": s, "k_nodes": s, "k_periodic": s, "k_prim": s, "k_dt": 1,
            "k_pre": 1, "k_finalize": 1, "k_bint": 0}.get(kernel, 0)


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

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    case = make_case()
    tmp = tempfile.TemporaryDirectory()
    ini = case.write(tmp.name)
    solver = Solver(ini)
    stream = torch.cuda.Stream(device=dev)
    solver.set_stream(stream.cuda_stream)
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
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * n * stages * args.steps / (ms_max / 1e3)

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
    te = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * n * stages * args.steps / (float(te.item()) / 1e3)

    # per-kernel device times (CUDA events on the launching stream)
    prof = solver.profile_kernels(reps=10)
    shares = {k: prof[k] * launches_per_iteration(case, k) for k in prof}
    total = sum(shares.values()) or 1.0
    dominant = max(shares, key=shares.get)
    peaks = measured_peaks()
    peak = peaks.get("hbm_gbs", 6650.0)
    alg = algorithmic_bytes(case, dominant)
    achieved = alg / (prof[dominant] / 1e3) / 1e9 if prof[dominant] > 0 else 0.0
    traffic = traffic_table().get(dominant)
    launches = args.steps * (1 + sum(launches_per_iteration(case, k) for k in prof if prof[k] > 0))
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
    }
    if world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(case, args.cpu_iters)
        line["cpu_baseline"] = {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")}
    print(json.dumps(line), flush=True)
    solver.close()


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
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
