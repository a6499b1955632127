"""Generates the restart and solution-output fixtures under
tests/golden/restart/ with the reference build (oracle/_ref, see
oracle/refbuild/Makefile).

Restart fixtures: the reference's own solver (oracle/_ref/turbobfm) runs a
small source case and writes its volume CSV (Output::writeSolution,
src/output.cpp:384-447); a target case then starts from that file with
RESTART_SOLUTION = yes, and the reference harness (oracle/_ref/ref_harness)
records the state right after the restart initialisation
(Solver::initializeSolutionFromRestart, src/solver.cpp:890-1295) and after a
few iterations. The refined targets put nodes exactly half-way between
source nodes, so the fixtures also pin how the nearest-neighbour search
resolves equal distances.

Output fixtures: the reference's volume CSV of a small case after a few
iterations, with the state it was written from (two of them viscous, with
the viscosity, wall shear stress and y+ columns).

Each <name>.npz holds the target case (coordinates, grid fields, patches and
settings as JSON), the restart file text, and the reference's results.

Run from the repository root with the reference build present:
    python tests/golden/restart/make_restart_golden.py
"""

from __future__ import annotations

import dataclasses
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, ROOT)

from cturbobfm_b200 import cases  # noqa: E402
from oracle.oracle import REF_CLI, ref_harness  # noqa: E402


def reference_solution(case, n_iter, fields):
    """Runs the reference solver n_iter iterations; returns its volume CSV text."""
    with tempfile.TemporaryDirectory() as d:
        c = case.with_settings(N_ITERATIONS=str(n_iter), SAVE_ITERATIONS_INTERVAL=str(n_iter),
                               OUTPUT_FIELDS_TYPE=fields, SAVE_UNSTEADY="no")
        c.write(d)
        r = subprocess.run([REF_CLI, "input.ini"], cwd=d, capture_output=True, text=True,
                           env=dict(os.environ, OMP_NUM_THREADS="1"), timeout=600)
        if r.returncode != 0:
            raise RuntimeError(r.stderr[-400:])
        return open(os.path.join(d, "Volume_CSV", "results.csv")).read()


def pack_case(case):
    return {"x": case.x, "y": case.y, "z": case.z,
            "field_names": np.array(list(case.fields.keys()) or [""]),
            **{"field_" + k: v for k, v in case.fields.items()},
            "patches": np.array(json.dumps([dataclasses.asdict(p) for p in case.patches])),
            "settings": np.array(json.dumps(case.settings)), "name": np.array(case.name)}


def restart_fixture(name, source, source_iters, target, restart_type, n_iter):
    text = reference_solution(source, source_iters, "secondary")
    kw = {"RESTART_SOLUTION": "yes", "RESTART_SOLUTION_FILEPATH": "restart.csv"}
    if restart_type:
        kw["RESTART_TYPE"] = restart_type
    target = target.with_settings(**kw)
    with tempfile.TemporaryDirectory() as d:
        ini = target.write(d)
        open(os.path.join(d, "restart.csv"), "w").write(text)
        init = ref_harness("steps", ini, 0)["state"]
        after = ref_harness("steps", ini, n_iter)
    out = pack_case(target)
    out.update({"restart_csv": np.array(text), "init_state": init, "n_iter": np.array(after["iterations"]),
                "state": after["state"]})
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, target.shape, "from", source.shape, restart_type, flush=True)


def output_fixture(name, case, n_iter, fields):
    text = reference_solution(case, n_iter, fields)
    with tempfile.TemporaryDirectory() as d:
        r = ref_harness("steps", case.write(d), n_iter)
    out = pack_case(case)
    out.update({"solution_csv": np.array(text), "n_iter": np.array(r["iterations"]), "state": r["state"],
                "fields_type": np.array(fields)})
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, case.shape, fields, flush=True)


def viscous(case, mu):
    """Laminar viscous run with the J-face walls as no-slip walls at rest."""
    for m in (2, 3):
        case.patches[m] = dataclasses.replace(case.patches[m], spec="no_slip_wall, 0, 0, 0")
    return case.with_settings(VISCOSITY_ACTIVE="yes", FLUID_CP="1004.675", FLUID_PRANDTL_NUMBER="0.72",
                              FLUID_MU_CONSTANT=repr(mu))


def main():
    bump = cases.bump2d(ni=24, nj=10, name="bump_src")
    restart_fixture("bump_standard", bump, 40, cases.bump2d(ni=24, nj=10, name="bump_same"), None, 10)
    restart_fixture("bump_nearest_ties", bump, 40, cases.bump2d(ni=47, nj=19, name="bump_fine"), None, 10)
    mer = cases.meridional(ni=16, nj=7, rows=cases.MAP_ROWS, name="mer_src")

    def ann(ni, nj, nk, nm):
        return cases.annulus3d(ni=ni, nj=nj, nk=nk, rows=cases.MAP_ROWS, scheme="JST", muscl=False, limiter="None",
                               rk=4, cfl=1.0, name=nm)

    restart_fixture("annulus_axisymmetric", mer, 40, ann(16, 7, 5, "ann_same_plane"), "axisymmetric", 5)
    restart_fixture("annulus_nearest_axi", mer, 40, ann(23, 10, 5, "ann_fine"), None, 5)
    restart_fixture("meridional_nearest_ties", mer, 40,
                    cases.meridional(ni=31, nj=13, rows=cases.MAP_ROWS, name="mer_fine"), None, 10)
    output_fixture("output_bump_secondary", cases.bump2d(ni=24, nj=10, name="bump_out"), 20, "secondary")
    output_fixture("output_meridional_primary", cases.meridional(ni=16, nj=7, rows=cases.MAP_ROWS, name="mer_out"),
                   20, "primary")
    output_fixture("output_bump_viscous", viscous(cases.bump2d(ni=24, nj=10, name="bump_visc"), 0.02), 20, "secondary")
    sector = cases.annulus3d(ni=16, nj=7, nk=5, scheme="JST", muscl=False, rk=4, bfm_model="None", name="ann_visc")
    sector = sector.with_settings(BFM_ACTIVE="no", BLOCKAGE_ACTIVE="no")
    output_fixture("output_annulus_viscous_primary", viscous(sector, 0.01), 10, "primary")


if __name__ == "__main__":
    main()
