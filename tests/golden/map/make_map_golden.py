"""Generates tests/golden/map/speedline.npz with the reference build
(oracle/_ref/turbobfm, see oracle/refbuild/Makefile): a small speed line of
run folders in the layout python/Run_All_Cases.py expects (P_, PREQ_ and KT_
folders, one folder without an input.ini, one unrelated folder), each solved
by the reference's own solver in its folder, and the files it leaves there:
turbo.csv, residuals.csv and the names of its volume CSV files. The
characteristics are the last turbo.csv rows, as
python/Extract_Characteristics.py reads them.

Run from the repository root with the reference build present:
    python tests/golden/map/make_map_golden.py
"""

from __future__ import annotations

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
from oracle.oracle import REF_CLI  # noqa: E402

N_ITER = 300


def folders():
    common = dict(N_ITERATIONS=str(N_ITER), SAVE_ITERATIONS_INTERVAL="100")
    p = cases.meridional(ni=16, nj=7, rows=cases.MAP_ROWS, p_ratio=1.02, drop=8, name="P_1.02")
    p = p.with_settings(HISTORY_BUFFER_SIZE="70", SAVE_UNSTEADY="no", **common)
    preq = cases.meridional(ni=16, nj=7, rows=cases.MAP_ROWS, p_ratio=1.05, drop=2, outlet="radial_equilibrium",
                            name="PREQ_1.05").with_settings(SAVE_UNSTEADY="yes", HISTORY_BUFFER_SIZE="1000000",
                                                            **common)
    kt = cases.throttle_request(16, 7, 0.9, 0.3, 0.9, name="KT_0.9", precision=None).with_settings(
        SAVE_UNSTEADY="no", HISTORY_BUFFER_SIZE="1000000", **common)
    return [p, preq, kt]


def main():
    out = {"n_iter": np.array(N_ITER)}
    meta = []
    with tempfile.TemporaryDirectory() as root:
        for c in folders():
            d = os.path.join(root, c.name)
            c.write(d)
            r = subprocess.run([REF_CLI, "input.ini"], cwd=d, capture_output=True, text=True,
                               env=dict(os.environ, OMP_NUM_THREADS="1"), timeout=600)
            if r.returncode != 0:
                raise RuntimeError(r.stderr[-400:])
            files = {}
            for f in ("input.ini", "grid.csv", "boundaries.csv"):
                files["in_" + f] = open(os.path.join(d, f)).read()
            for f in ("turbo.csv", "residuals.csv"):
                files["out_" + f] = open(os.path.join(d, f), encoding="utf-8").read()
            vols = sorted(os.listdir(os.path.join(d, "Volume_CSV")))
            for k, v in files.items():
                out[f"{c.name}/{k}"] = np.array(v)
            meta.append({"name": c.name, "volume_files": vols})
            print(c.name, "rows", files["out_turbo.csv"].count("\n") - 1, "volume", vols, flush=True)
    meta.append({"name": "P_1.10", "volume_files": None})  # a run folder without input.ini
    out["folders"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(HERE, "speedline.npz"), **out)


if __name__ == "__main__":
    main()
