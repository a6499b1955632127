"""Compressor-map front-end: the reference's python/Run_All_Cases.py and
python/Extract_Characteristics.py on the batched GPU path.

The reference runs one ``turbobfm input.ini`` process per run folder
(Run_All_Cases.py:18-98) and then reads the last row of every folder's
turbo.csv into characteristics.csv (Extract_Characteristics.py:17-52). Here
every folder's operating point becomes a solver, the solvers that share
GPU_PRECISION and N_ITERATIONS advance together as one batch on the device,
and each folder receives the files the reference's solve leaves behind
(Solver::solve, src/solver.cpp:1296-1424): residuals.csv, turbo.csv (with
TURBO_OUTPUT = yes) and the final volume CSV under Volume_CSV/ (the
intermediate volume files of every SAVE_ITERATIONS_INTERVAL are not
written). The rows of
residuals.csv and turbo.csv are the ones the reference has flushed when its
loop ends, with its time column (writeLogResidualsToCsvFile and
writeTurboPerformanceToCsvFile, src/solver.cpp:2516-2595).

    from cturbobfm_b200 import compressor_map
    data = compressor_map.run_cases("speedline_100")
    compressor_map.write_characteristics(data, "characteristics.csv")
"""

from __future__ import annotations

import os
from typing import Dict, List, Optional, Tuple

import numpy as np

RUN_PREFIXES = ("KT", "PREQ", "P", "MF")


def run_folders(input_folder: str) -> List[str]:
    """Folders named <KT|PREQ|P|MF>_<number>, sorted by the number
    (Run_All_Cases.py:27-35, Extract_Characteristics.py:22-28)."""
    folders = [f for f in os.listdir(input_folder) if f.split("_")[0] in RUN_PREFIXES]
    folders.sort(key=lambda f: float(f.split("_")[1]))
    return folders


def read_ini(path: str) -> Dict[str, str]:
    """KEY = value lines of an input.ini; ';' comments and '[' lines skipped
    (Config::Config, src/config.cpp:15-44)."""
    out = {}
    with open(path) as f:
        for line in f:
            s = line.strip()
            if not s or s[0] in ";[" or "=" not in s:
                continue
            k, v = s.split("=", 1)
            out[k.strip()] = v.strip()
    return out


def _bool(v: Optional[str], default: bool) -> bool:
    if v is None:
        return default
    return v.strip().lower() in ("yes", "true", "1", "on")


def flush_points(n_done: int, status: int, max_iter: int, interval: int, buffer: int) -> List[int]:
    """Iterations after which the reference appends its residual and turbo
    buffers to the CSV files: every multiple of SAVE_ITERATIONS_INTERVAL, the
    last iteration N_ITERATIONS, whenever HISTORY_BUFFER_SIZE rows are
    waiting, and at convergence (src/solver.cpp:1399-1421). A diverged run
    ends at the norm's exception without a flush (status 2)."""
    out = []
    waiting = 0
    for it in range(1, n_done + 1):  # completed iterations (a diverged one records no row)
        waiting += 1
        converged_here = status == 1 and it == n_done
        if converged_here or it % interval == 0 or it == max_iter or waiting >= buffer:
            out.append(it)
            waiting = 0
    return out


def turbo_rows(turbo: np.ndarray, time: np.ndarray, flushes: List[int],
               greitzer: bool = False) -> List[Tuple[float, ...]]:
    """turbo.csv rows: (time in microseconds, mass flow, PRtt, TRtt, ETAtt)
    for the flushed iterations. The reference writes its turbo list against
    Solver::_time entry by entry, a list that starts with the initial time
    and, like the turbo list, is emptied at every flush
    (src/solver.cpp:2577-2591): before the first flush a row carries the time
    at the start of its iteration, after it the time at its end. With the
    Greitzer model the turbo list also starts with the initial state's
    values (Solver::initializeSolutionArrays, src/solver.cpp:803-806), which
    are the first iteration's, so every iteration's row carries its end time
    after an extra first row at time 0."""
    rows = []
    if not flushes:
        return rows
    first = flushes[0]
    if greitzer:
        rows.append((0.0, turbo[0, 0], turbo[0, 1], turbo[0, 2], turbo[0, 3]))
    for k in range(1, flushes[-1] + 1):
        if greitzer or k > first:
            t = time[k - 1]
        else:
            t = time[k - 2] if k >= 2 else 0.0
        rows.append((t * 1e6, turbo[k - 1, 0], turbo[k - 1, 1], turbo[k - 1, 2], turbo[k - 1, 3]))
    return rows


def _g(v: float) -> str:
    """C++ ostream's default formatting of a double (6 significant digits)."""
    return "%g" % v


def _solution_name(settings: Dict[str, str], it: int) -> str:
    """Output::getOutputFilename (src/output.cpp:370-382)."""
    name = settings.get("SOLUTION_NAME", "results")
    if _bool(settings.get("SAVE_UNSTEADY"), True):
        return f"{name}_{it:06d}"
    return name


def _write_outputs(folder: str, settings: Dict[str, str], solver, max_iter: int) -> Dict[str, object]:
    h = solver.history()
    status = solver.status
    n = len(h["lognorm"])
    interval = int(float(settings.get("SAVE_ITERATIONS_INTERVAL", "1")))
    buffer = int(float(settings.get("HISTORY_BUFFER_SIZE", str(interval))))
    flushes = flush_points(n, status, max_iter, max(interval, 1), max(buffer, 1))
    end = flushes[-1] if flushes else 0
    if end:
        with open(os.path.join(folder, "residuals.csv"), "w") as f:
            f.write("Rho,RhoU,RhoV,RhoW,RhoE\n")
            for r in h["lognorm"][:end]:
                f.write(",".join(_g(v) for v in r) + "\n")
    if end and _bool(settings.get("TURBO_OUTPUT"), False):
        with open(os.path.join(folder, "turbo.csv"), "w", encoding="utf-8") as f:
            f.write("Time[μs],Massflow[kg/s],PRtt,TRtt,ETAtt\n")
            greitzer = _bool(settings.get("ENABLE_GREITZER_MODELING"), False)
            for row in turbo_rows(h["turbo"], h["time"], flushes, greitzer):
                f.write(",".join(_g(v) for v in row) + "\n")
    solution = None
    if status != 2 and n:
        os.makedirs(os.path.join(folder, "Volume_CSV"), exist_ok=True)
        solution = os.path.join(folder, "Volume_CSV", _solution_name(settings, n) + ".csv")
        solver.write_solution(solution)
    return {"status": status, "iterations": n, "solution": solution}


def run_cases(input_folder: str, verbose: bool = True) -> Dict[str, Dict[str, object]]:
    """Runs every run folder's input.ini on the GPU and writes its output
    files; returns {folder: {"status", "iterations", "solution"}} (status 1
    converged, 2 diverged, 0 reached N_ITERATIONS). Folders without an
    input.ini are skipped with the reference's warning."""
    from .solver import Batch, Solver

    groups: Dict[Tuple[int, int], List[Tuple[str, Dict[str, str], Solver]]] = {}
    results: Dict[str, Dict[str, object]] = {}
    solvers = []
    try:
        for run in run_folders(input_folder):
            path = os.path.join(input_folder, run)
            ini = os.path.join(path, "input.ini")
            if not os.path.exists(ini):
                if verbose:
                    print(f"WARNING: input.ini not found in {path}, skipping.")
                continue
            s = Solver(ini)
            solvers.append(s)
            settings = read_ini(ini)
            key = (s.info().precision, s.info().max_iterations)
            groups.setdefault(key, []).append((run, settings, s))
        for (_, max_iter), members in groups.items():
            with Batch([m[2] for m in members]) as b:
                b.step(max_iter)
            for run, settings, s in members:
                results[run] = _write_outputs(os.path.join(input_folder, run), settings, s, max_iter)
                if verbose:
                    print(f"Run {run}: status {results[run]['status']} after {results[run]['iterations']} iterations.")
    finally:
        for s in solvers:
            s.close()
    return results


def read_solutions(input_folder: str, verbose: bool = True) -> Dict[str, np.ndarray]:
    """The last row of every run folder's turbo.csv
    (Extract_Characteristics.py:17-42); a run folder without one (no
    input.ini, or TURBO_OUTPUT off) is skipped with a warning where the
    reference's script stops with an error."""
    import pandas as pd

    out = {"Massflow": [], "PRtt": [], "TRtt": [], "ETAtt": []}
    for run in run_folders(input_folder):
        path = os.path.join(input_folder, run, "turbo.csv")
        if not os.path.exists(path):
            if verbose:
                print(f"WARNING: turbo.csv not found in {os.path.join(input_folder, run)}, skipping.")
            continue
        df = pd.read_csv(path)
        out["Massflow"].append(df["Massflow[kg/s]"].to_numpy()[-1])
        out["PRtt"].append(df["PRtt"].to_numpy()[-1])
        out["TRtt"].append(df["TRtt"].to_numpy()[-1])
        out["ETAtt"].append(df["ETAtt"].to_numpy()[-1])
    return {k: np.array(v) for k, v in out.items()}


def write_characteristics(data: Dict[str, np.ndarray], path: str = "characteristics.csv") -> str:
    """characteristics.csv (Extract_Characteristics.py:46-52)."""
    with open(path, "w") as f:
        f.write("MassFlow [kg/s],PRtt [-],TRtt [-],ETAtt [-]\n")
        for i in range(len(data["Massflow"])):
            f.write(f"{data['Massflow'][i]:.6f},{data['PRtt'][i]:.6f},{data['TRtt'][i]:.6f},{data['ETAtt'][i]:.6f}\n")
    return path


def main(argv=None) -> int:
    import argparse

    ap = argparse.ArgumentParser(description="Runs the KT_/PREQ_/P_/MF_ folders of a speed line as one GPU batch "
                                             "and writes characteristics.csv.")
    ap.add_argument("input_folder")
    ap.add_argument("--output", default="characteristics.csv")
    args = ap.parse_args(argv)
    run_cases(args.input_folder)
    write_characteristics(read_solutions(args.input_folder), args.output)
    print(f"Characteristics saved to {args.output}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
