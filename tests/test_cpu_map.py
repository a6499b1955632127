"""The compressor-map front-end's host logic against the reference's
scripts and files: run-folder discovery and order (Run_All_Cases.py,
Extract_Characteristics.py), the reference's flush schedule and time column
of turbo.csv (checked on files the reference build wrote), and the
characteristics file."""

import os

import numpy as np

import map_util
from cturbobfm_b200 import compressor_map as cm


def test_run_folders_follow_the_reference_rule(tmp_path):
    for d in ("P_1.10", "KT_0.9", "PREQ_1.05", "notes", "MF_2", "P_0.95", "Volume_CSV"):
        (tmp_path / d).mkdir()
    assert cm.run_folders(str(tmp_path)) == ["KT_0.9", "P_0.95", "PREQ_1.05", "P_1.10", "MF_2"]


def test_flush_points():
    assert cm.flush_points(300, 0, 300, 100, 70) == [70, 100, 170, 200, 270, 300]
    assert cm.flush_points(171, 1, 300, 100, 10 ** 6) == [100, 171]
    assert cm.flush_points(150, 2, 300, 100, 10 ** 6) == [100]
    assert cm.flush_points(0, 2, 300, 100, 100) == []


def test_reference_files_follow_the_flush_schedule():
    fx, meta = map_util.load()
    rows = {m["name"]: map_util.table(str(fx[m["name"] + "/out_turbo.csv"]))[1] for m in meta if m["volume_files"]}
    assert len(rows["P_1.02"]) == cm.flush_points(300, 0, 300, 100, 70)[-1]
    assert len(rows["PREQ_1.05"]) == 171  # converged at 171
    assert len(rows["KT_0.9"]) == 301  # Greitzer: one more row, the initial state's
    t = rows["P_1.02"][:, 0]
    # before the first flush (70) a row carries its iteration's start time, after it the end time
    steps = np.diff(t)
    assert steps[69] > 1.5 * steps[68] and steps[69] > 1.5 * steps[70]
    kt = rows["KT_0.9"]
    assert kt[0, 0] == 0.0 and np.array_equal(kt[0, 1:], kt[1, 1:])


def test_characteristics_are_the_last_turbo_rows(tmp_path):
    fx, meta = map_util.write_reference_outputs(str(tmp_path))
    runs = [m["name"] for m in meta if m["volume_files"]]
    os.rmdir(tmp_path / "P_1.10")
    data = cm.read_solutions(str(tmp_path))
    assert cm.run_folders(str(tmp_path)) == ["KT_0.9", "P_1.02", "PREQ_1.05"]
    out = cm.write_characteristics(data, str(tmp_path / "characteristics.csv"))
    lines = open(out).read().splitlines()
    assert lines[0] == "MassFlow [kg/s],PRtt [-],TRtt [-],ETAtt [-]"
    for line, run in zip(lines[1:], ["KT_0.9", "P_1.02", "PREQ_1.05"]):
        last = map_util.table(str(fx[run + "/out_turbo.csv"]))[1][-1]
        assert line == ",".join(f"{v:.6f}" for v in last[1:])
    assert len(runs) == 3
