"""GPU behaviour beyond the small parity cases: divergence at the same
iteration as the oracle, full-size workloads against the oracle for a few
iterations, determinism, and the stop-at-convergence contract."""

import numpy as np
import pytest

from cturbobfm_b200 import cases

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return (np.abs(a - b).max(axis=1) / scale).max()


def test_divergence_is_reported_at_the_oracles_iteration(tmp_path, oracle_lib):
    from cturbobfm_b200 import Solver, SolverDiverged

    ini = cases.bump2d(ni=96, nj=32, scheme="Roe", muscl=True, limiter="van albada", rk=3, cfl=1.2).write(str(tmp_path))
    ro = oracle_lib.Oracle(ini).run(500)
    assert ro["status"] == 2
    with Solver(ini) as s:
        with pytest.raises(SolverDiverged, match="Solver diverged"):
            s.step(500)
        assert s.iteration == ro["iterations"]
        assert s.status == 2
        with pytest.raises(SolverDiverged):  # a diverged run stays stopped and keeps reporting it
            s.step(10)
        assert s.iteration == ro["iterations"]


def test_bump_192x64_matches_the_reference_after_5000_iterations(tmp_path):
    """The 192 x 64 bump channel (JST, RK4, local dt at CFL 2.0, uniform
    inlet start) after 5000 iterations against the reference solver's own
    run (fixture tests/golden/c1/bump2d_c1_5000.npz, made by
    tests/golden/c1/make_c1_golden.py): 1e-12 relative per field, 1e-10 on every
    log10 residual norm of the history."""
    import os

    from cturbobfm_b200 import Solver

    fx = np.load(os.path.join(os.path.dirname(__file__), "golden", "c1", "bump2d_c1_5000.npz"))
    n = int(fx["n_iter"])
    ini = cases.bump2d().write(str(tmp_path))
    with Solver(ini) as s:
        assert s.step(n) == n
        assert rel_err(s.state(), fx["state"]) <= 1e-12
        h = s.history()
        assert np.abs(h["lognorm"] - fx["lognorm"]).max() <= 1e-10
        assert abs(s.time - float(fx["time"])) <= 1e-12 * float(fx["time"])


@pytest.mark.parametrize("which,n", [("bump2d_192x64", 20), ("annulus3d_160x48x64", 10)])
def test_full_size_workloads_match_oracle(which, n, tmp_path, oracle_lib):
    from cturbobfm_b200 import Solver

    case = cases.bump2d() if which.startswith("bump") else cases.annulus3d()
    ini = case.write(str(tmp_path))
    o = oracle_lib.Oracle(ini)
    o.run(n)
    with Solver(ini) as s:
        assert s.step(n) == n
        assert rel_err(s.state(), o.state()) <= 1e-12
        assert np.abs(s.lognorm() - o.history()["lognorm"][-1]).max() <= 1e-10


def test_runs_are_deterministic(tmp_path):
    from cturbobfm_b200 import Solver

    ini = cases.annulus3d(ni=80, nj=24, nk=33, cfl=1.0).write(str(tmp_path))
    out = []
    for _ in range(2):
        with Solver(ini) as s:
            s.step(25)
            out.append((s.state(), s.lognorm()))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_step_chunks_equal_one_long_step(tmp_path):
    from cturbobfm_b200 import Solver

    ini = cases.meridional(ni=48, nj=16).write(str(tmp_path))
    with Solver(ini) as a, Solver(ini) as b:
        a.step(37)
        for n in (1, 8, 3, 16, 9):
            b.step(n)
        assert np.array_equal(a.state(), b.state())
        assert a.time == b.time


def test_full_size_real_gas_workload_matches_oracle(tmp_path, oracle_lib):
    from cturbobfm_b200 import Solver

    # the 256 x 96 x 128 CO2 annulus (3.1 M nodes): one iteration, FP64
    ini = cases.realgas_annulus().write(str(tmp_path))
    o = oracle_lib.Oracle(ini)
    o.run(1)
    with Solver(ini) as s:
        assert s.step(1) == 1
        assert rel_err(s.state(), o.state()) <= 1e-12
        assert np.abs(s.lognorm() - o.history()["lognorm"][-1]).max() <= 1e-10
