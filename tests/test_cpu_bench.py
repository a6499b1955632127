"""Host logic of bench.py that needs no GPU: the reference arm's JSON line
(the reference build, or the oracle port when the build is absent, timed on
the host cores), its rank-0-only rule under torchrun, and the byte and launch
counts behind the roofline figures."""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _run(args, env=None, timeout=600):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, env=e,
                          capture_output=True, text=True, timeout=timeout)


def test_reference_arm_prints_one_contract_line():
    r = _run(["--impl", "reference", "--steps", "1", "--warmup", "3"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["higher_is_better"] is True and line["n_gpus"] == 1
    assert line["config"]["workload"] == bench.WORKLOAD
    assert line["value"] > 0 and line["ms_per_step"] > 0
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_runs_on_rank_0_only():
    r = _run(["--impl", "reference", "--gpus", "2", "--steps", "1"],
             env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]


@pytest.fixture(scope="module")
def annulus():
    return bench.make_case()


def test_stage_bytes_per_cell_stage(annulus):
    # w (5 + 5 + 5 + 1) + 8 * 3 * 3 + 14 w at the 33.75 % blade-row nodes
    assert bench.blade_fraction(annulus) == pytest.approx(0.3375)
    assert bench.stage_bytes_per_cell(annulus) == pytest.approx(8 * 16 + 72 + 14 * 8 * 0.3375)
    assert round(bench.stage_bytes_per_cell(annulus), 1) == 237.8
    assert round(bench.stage_bytes_per_cell(annulus, word=4), 1) == 194.9


def test_roofline_bytes_do_not_exceed_measured_traffic(annulus):
    """The kernels whose fraction is reported from algorithmic bytes (the node
    kernel of the split stage, the fused stage kernel) count no more bytes
    than ncu measured in DRAM for one launch; the rest of the gap is re-reads."""
    traffic = bench.traffic_table()
    for k in ("k_nodes", "k_stage"):
        alg = bench.algorithmic_bytes(annulus, k)
        assert 0 < alg <= traffic[k], (k, alg, traffic[k])
        assert alg >= 0.5 * traffic[k], (k, alg, traffic[k])


def test_launch_counts_per_iteration(annulus):
    s = annulus.n_stages
    assert s == 3
    split = {k: bench.calls_per_iteration(annulus, k) for k in bench.SPLIT_STAGE + bench.FUSED_STAGE}
    fused = {k: bench.calls_per_iteration(annulus, k, fused=True) for k in bench.SPLIT_STAGE + bench.FUSED_STAGE}
    assert split["k_prim"] == 1 and fused["k_prim"] == 0  # later stages read stored primitives
    for k in ("k_faces_I", "k_faces_J", "k_faces_K", "k_nodes"):
        assert split[k] == s and fused[k] == 0
    assert split["k_stage"] == 0 and fused["k_stage"] == s
    assert split["k_periodic"] == fused["k_periodic"] == s
    # K lines run plain and end faces as two launches; nk = 64 rows of J fill whole warps
    assert bench.launches_per_iteration(annulus, "k_faces_K") == 2 * s
    assert bench.launches_per_iteration(annulus, "k_faces_J") == s
    assert bench.launches_per_iteration(annulus, "k_faces_I") == s
