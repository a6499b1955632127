"""Generates the golden fixtures under tests/golden/ from the reference's own
regression cases (test/regression_tests/* of CTurboBFM).

For each case the script
  * reads the case's input.ini and grid file and rebuilds the boundaries.csv
    the upstream repository does not ship (INFLOW on the I start face, OUTFLOW
    on the I end face, LOWER_WALL / UPPER_WALL on the J faces, PER1 / PER2 on
    the K faces, the patch naming every case uses);
  * runs the reference solver built from its own sources
    (oracle/_ref/ref_harness, see oracle/refbuild/Makefile) for a fixed
    number of iterations and, for the cheap cases, to its convergence test;
  * stores the inputs and the outputs (full-precision states, residual-norm
    histories, turbo performance) in <case>.npz, plus the Density, Pressure
    and Temperature columns of the case's shipped reference.csv.

Run from the repository root with the reference mounted:
    python tests/golden/make_golden.py /path/to/reference
"""

from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cturbobfm_b200 import cases  # noqa: E402
from oracle.oracle import ref_harness  # noqa: E402

CASES = {
    # name: (iterations for the fixed-length run, run to convergence too)
    "CircularBump2D": (50, True),
    "AxisymmetricSwirlingChannel": (50, True),
    "CircularBump3D_PeriodicSwirl": (30, True),
    "GER4_Axisymmetric_Hall": (50, True),
    "GER4_Axisymmetric_HallThollet": (50, True),
    "GER4_FullAnnulus": (30, False),
}


def read_ini(path):
    out = []
    for line in open(path):
        s = line.strip()
        if not s or s[0] in ";[#" or "=" not in s:
            continue
        k, v = s.split("=", 1)
        out.append((k.strip(), v.strip()))
    return out


def boundaries_text(shape, names):
    ni, nj, nk = shape
    rows = [("INFLOW", 0, 0, 0, nj, 0, nk), ("OUTFLOW", ni, ni, 0, nj, 0, nk),
            ("LOWER_WALL", 0, ni, 0, 0, 0, nk), ("UPPER_WALL", 0, ni, nj, nj, 0, nk)]
    if "PER1" in names:
        rows += [("PER1", 0, ni, 0, nj, 0, 0), ("PER2", 0, ni, 0, nj, nk, nk)]
    text = f"NI={ni}\nNJ={nj}\nNK={nk}\nPATCH_NAME,I_MIN,I_MAX,J_MIN,J_MAX,K_MIN,K_MAX\n"
    return text + "".join(",".join(str(v) for v in r) + "\n" for r in rows)


def write_case(directory, settings, grid, shape, btext, n_iter):
    os.makedirs(directory, exist_ok=True)
    names = list(grid.keys())
    data = np.stack([grid[n].reshape(-1) for n in names], axis=1)
    with open(os.path.join(directory, "grid.csv"), "w") as f:
        f.write(f"NI={shape[0]}\nNJ={shape[1]}\nNK={shape[2]}\n" + ",".join(names) + "\n")
        np.savetxt(f, data, fmt="%.17g", delimiter=",")
    open(os.path.join(directory, "boundaries.csv"), "w").write(btext)
    s = dict(settings)
    s.update({"GRID_FILE": "grid.csv", "BOUNDARY_CONDITIONS_FILEPATH": "boundaries.csv",
              "SAVE_ITERATIONS_INTERVAL": "100000000", "N_ITERATIONS": str(n_iter)})
    ini = os.path.join(directory, "input.ini")
    with open(ini, "w") as f:
        f.write("[CFD]\n" + "".join(f"{k} = {v}\n" for k, v in s.items()))
    return ini


def shipped_columns(path):
    _, cols = cases.read_grid_csv(path)
    return {k: cols[k].reshape(-1) for k in ("Density", "Pressure", "Temperature") if k in cols}


def main(ref_root):
    for name, (n_iter, converge) in CASES.items():
        cdir = os.path.join(ref_root, "test", "regression_tests", name)
        settings = dict(read_ini(os.path.join(cdir, "input.ini")))
        shape, grid = cases.read_grid_csv(os.path.join(cdir, settings["GRID_FILE"]))
        btext = boundaries_text(shape, settings)
        out = {"ini": np.array("\n".join(f"{k} = {v}" for k, v in settings.items())),
               "boundaries": np.array(btext), "shape": np.array(shape),
               "grid_names": np.array(list(grid.keys()))}
        for k, v in grid.items():
            out["grid_" + k] = v
        with tempfile.TemporaryDirectory() as d:
            ini = write_case(d, settings, grid, shape, btext, n_iter)
            r = ref_harness("steps", ini, n_iter)
            out.update({"n_iter": np.array(r["iterations"]), "state": r["state"], "lognorm": r["lognorm"],
                        "massflow": r["massflow"], "turbo": r["turbo"], "hub": r["hub"], "time": np.array(r["time"])})
            if converge:
                ini = write_case(os.path.join(d, "conv"), settings, grid, shape, btext, 200000)
                rc = ref_harness("steps", ini, 200000, timeout=3600)
                out.update({"conv_iterations": np.array(rc["iterations"]), "conv_status": np.array(rc["converged"]),
                            "conv_state": rc["state"], "conv_lognorm_last": rc["lognorm"][-1]})
        ref_csv = os.path.join(cdir, "reference.csv")
        if os.path.exists(ref_csv):
            for k, v in shipped_columns(ref_csv).items():
                out["shipped_" + k] = v
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, shape, "iterations", int(out["n_iter"]),
              "converged at", int(out["conv_iterations"]) if converge else "-", flush=True)


if __name__ == "__main__":
    from oracle.oracle import reference_root

    main(sys.argv[1] if len(sys.argv) > 1 else reference_root())
