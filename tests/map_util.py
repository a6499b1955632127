"""The speed-line fixture of tests/golden/map/ (made by make_map_golden.py
with the reference build) as run folders."""

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "map", "speedline.npz")


def load():
    fx = dict(np.load(FIXTURE, allow_pickle=False))
    return fx, json.loads(str(fx["folders"]))


def write_inputs(root):
    """The run folders with their inputs (plus a run folder without an
    input.ini and an unrelated folder); returns the fixture."""
    fx, meta = load()
    for m in meta:
        d = os.path.join(root, m["name"])
        os.makedirs(d, exist_ok=True)
        for f in ("input.ini", "grid.csv", "boundaries.csv"):
            key = f"{m['name']}/in_{f}"
            if key in fx:
                with open(os.path.join(d, f), "w") as out:
                    out.write(str(fx[key]))
    os.makedirs(os.path.join(root, "notes"), exist_ok=True)
    return fx, meta


def write_reference_outputs(root):
    """The reference's turbo.csv / residuals.csv in the run folders."""
    fx, meta = load()
    for m in meta:
        d = os.path.join(root, m["name"])
        os.makedirs(d, exist_ok=True)
        for f in ("turbo.csv", "residuals.csv"):
            key = f"{m['name']}/out_{f}"
            if key in fx:
                with open(os.path.join(d, f), "w", encoding="utf-8") as out:
                    out.write(str(fx[key]))
    return fx, meta


def table(text):
    lines = text.splitlines()
    return lines[0], np.array([[float(v) for v in l.split(",")] for l in lines[1:] if l.strip()])
