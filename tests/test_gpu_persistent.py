"""The persistent iteration kernel (k_run, GPU_STAGE_FUSION = persistent)
against the split stage kernels (GPU_STAGE_FUSION = split) on the same case
files. k_run runs the split kernels' bodies over the same tiles, one phase
after another behind a grid barrier, so in FP64 states, norms, time and
iteration counts agree bit for bit, also when members converge or stop at
different iterations inside one launch."""

import os

import numpy as np
import pytest

from cturbobfm_b200 import cases
from parity_cases import CASES

pytestmark = pytest.mark.gpu


def _eligible(case):
    s = case.settings
    return (s.get("VISCOSITY_ACTIVE", "no").lower() not in ("yes", "true", "1")
            and s.get("TURBULENCE_ACTIVE", "no").lower() not in ("yes", "true", "1")
            and case.table is None)


PERSISTENT_CASES = [n for n in sorted(CASES) if _eligible(CASES[n][0]())]


def rel_err(a, b):
    scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return (np.abs(a - b).max(axis=1) / scale).max()


def _run(case, n, fusion, tmp_path, tag, solve=False):
    from cturbobfm_b200 import Solver, SolverDiverged

    ini = case.with_settings(GPU_STAGE_FUSION=fusion).write(str(tmp_path / tag))
    with Solver(ini) as s:
        assert s.info().persistent_stage == (1 if fusion == "persistent" else 0)
        if solve:
            try:
                done = s.solve()
            except SolverDiverged:
                done = None
        else:
            done = s.step(n)
        return done, s.state(), s.history(), s.time, s.status, s.iteration


def test_eligible_cases_cover_both_schemes_and_periodic_sectors():
    names = set(PERSISTENT_CASES)
    assert len(names) >= 25
    assert {"annulus_roe_hall", "sector45_mass_flow", "bump_jst_rk4", "meridional_chima"} <= names


@pytest.mark.parametrize("name", PERSISTENT_CASES)
def test_persistent_equals_split(name, tmp_path):
    make, n = CASES[name]
    a = _run(make(), n, "split", tmp_path, "split")
    b = _run(make(), n, "persistent", tmp_path, "persistent")
    assert a[0] == b[0] == n
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(a[2]["lognorm"], b[2]["lognorm"])
    assert a[3] == b[3]


def test_persistent_converges_at_the_same_iteration(tmp_path):
    """solve() to a 2-order drop: the convergence test fires inside a k_run
    launch, which stops at that iteration as the split graphs do."""
    c = cases.bump2d(ni=40, nj=16).with_settings(RESIDUALS_DROP_CONVERGENCE="2", N_ITERATIONS="3000")
    a = _run(c, 0, "split", tmp_path, "split", solve=True)
    b = _run(c, 0, "persistent", tmp_path, "persistent", solve=True)
    assert a[4] == b[4] == 1
    assert a[5] == b[5]
    assert np.array_equal(a[1], b[1])


def test_persistent_batch_of_uneven_members_equals_split(tmp_path):
    """A batch of compressor-map instances of different sizes and operating
    points (JST, RK4, Hall forces) with N_ITERATIONS that end inside a
    launch, in one persistent group: each member bit for bit as in the split
    batch."""
    from cturbobfm_b200 import Batch, Solver

    cs = cases.compressor_map(n=6, seed=7, precision="fp64", drop=4)
    cs = [c.with_settings(N_ITERATIONS=str(150 + 37 * i)) for i, c in enumerate(cs)]
    out = {}
    for fusion in ("split", "persistent"):
        inis = []
        for i, c in enumerate(cs):
            d = tmp_path / fusion / str(i)
            os.makedirs(d)
            inis.append(c.with_settings(GPU_STAGE_FUSION=fusion).write(str(d)))
        solvers = [Solver(p) for p in inis]
        try:
            with Batch(solvers) as b:
                assert b.stage_kernels()[0] == fusion
                b.step(400)
            out[fusion] = [(s.iteration, s.status, s.state()) for s in solvers]
        finally:
            for s in solvers:
                s.close()
    for (ia, sa, ua), (ib, sb, ub) in zip(out["split"], out["persistent"]):
        assert ia == ib and sa == sb
        assert np.array_equal(ua, ub)


@pytest.mark.parametrize("name", ["annulus_roe_hall", "sector45_mass_flow", "meridional_hall"])
def test_persistent_matches_split_in_float(name, tmp_path):
    """fp32_kahan: the same bodies compiled in another unit with the float
    flags; the compiler may contract an expression differently there, so the
    bound is the float path's stated tolerance (1e-3 relative per field)."""
    make, n = CASES[name]
    c = make().with_settings(GPU_PRECISION="fp32_kahan")
    a = _run(c, n, "split", tmp_path, "split")
    b = _run(c, n, "persistent", tmp_path, "persistent")
    assert a[0] == b[0]
    assert rel_err(b[1], a[1]) <= 1e-3


def test_autotuner_times_the_persistent_kernel(tmp_path):
    from cturbobfm_b200 import Solver

    with Solver(cases.bump2d(ni=48, nj=20).write(str(tmp_path / "a"))) as s:
        s.autotune()
        mode, ms = s.stage_kernels()
        assert ms["split"] > 0 and ms["persistent"] > 0
        # a small 2-D grid: one launch instead of several per stage
        assert mode in ("persistent", "fused")
    viscous = CASES["bump_viscous_roe_muscl"][0]()
    with Solver(viscous.write(str(tmp_path / "v"))) as s:
        s.autotune()
        mode, ms = s.stage_kernels()
        assert ms["persistent"] == 0 and mode != "persistent"
