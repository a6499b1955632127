"""Materialises the golden fixtures of tests/golden/*.npz (made by
tests/golden/make_golden.py from the reference's regression cases) as case
directories in the reference's file formats."""

import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def fixture_names():
    return sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False))


def write_case(fx, directory, n_iter):
    """Writes grid.csv, boundaries.csv and input.ini of a fixture; N_ITERATIONS
    is set to n_iter. Returns the ini path."""
    os.makedirs(directory, exist_ok=True)
    shape = tuple(int(v) for v in fx["shape"])
    names = [str(n) for n in fx["grid_names"]]
    data = np.stack([fx["grid_" + n].reshape(-1) for n in names], axis=1)
    with open(os.path.join(directory, "grid.csv"), "w") as f:
        f.write(f"NI={shape[0]}\nNJ={shape[1]}\nNK={shape[2]}\n" + ",".join(names) + "\n")
        np.savetxt(f, data, fmt="%.17g", delimiter=",")
    with open(os.path.join(directory, "boundaries.csv"), "w") as f:
        f.write(str(fx["boundaries"]))
    settings = {}
    for line in str(fx["ini"]).splitlines():
        k, v = line.split("=", 1)
        settings[k.strip()] = v.strip()
    settings.update({"GRID_FILE": "grid.csv", "BOUNDARY_CONDITIONS_FILEPATH": "boundaries.csv",
                     "SAVE_ITERATIONS_INTERVAL": "100000000", "N_ITERATIONS": str(n_iter)})
    ini = os.path.join(directory, "input.ini")
    with open(ini, "w") as f:
        f.write("[CFD]\n" + "".join(f"{k} = {v}\n" for k, v in settings.items()))
    return ini


def primitive_fields(u, gamma, rgas):
    """Density, pressure and temperature from a conservative state (5, N),
    as FluidIdeal computes them (src/fluid_ideal.cpp:74-112)."""
    rho = u[0]
    vx, vy, vz, et = u[1] / rho, u[2] / rho, u[3] / rho, u[4] / rho
    vm = np.sqrt(vx * vx + vy * vy + vz * vz)
    e = et - 0.5 * (vm * vm)
    p = (gamma - 1) * rho * e
    return rho, p, p / (rho * rgas)


def l2_relative(a, b):
    """The regression tests' error measure (test/regression_tests/test_cases.py:82-88)."""
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


RESTART = os.path.join(GOLDEN, "restart")


def restart_fixture_names(prefix=""):
    """Fixtures of tests/golden/restart/ (made by make_restart_golden.py)."""
    return sorted(n for n in (os.path.splitext(os.path.basename(p))[0]
                              for p in glob.glob(os.path.join(RESTART, "*.npz"))) if n.startswith(prefix))


def load_restart(name):
    return dict(np.load(os.path.join(RESTART, name + ".npz"), allow_pickle=False))


def restart_case(fx):
    """The fixture's target case as a cases.Case."""
    import json

    from cturbobfm_b200 import cases

    names = [str(n) for n in fx["field_names"] if str(n)]
    patches = [cases.Patch(**p) for p in json.loads(str(fx["patches"]))]
    return cases.Case(name=str(fx["name"]), x=fx["x"], y=fx["y"], z=fx["z"],
                      fields={n: fx["field_" + n] for n in names}, patches=patches,
                      settings=json.loads(str(fx["settings"])))


def write_restart_case(fx, directory, **settings):
    """Writes the fixture's case (and its restart.csv, if any); returns the
    ini path. Extra settings override the fixture's."""
    case = restart_case(fx)
    if settings:
        case = case.with_settings(**settings)
    ini = case.write(directory)
    if "restart_csv" in fx:
        with open(os.path.join(directory, "restart.csv"), "w") as f:
            f.write(str(fx["restart_csv"]))
    return ini
