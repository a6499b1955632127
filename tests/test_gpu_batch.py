"""Batches: several operating points advanced by one launch per kernel family
(ctbfm_batch_*). Every member must compute bit for bit what it computes
alone, whatever the other members are (grid sizes, topologies, schemes,
stage counts), and stop on the device at its own convergence or divergence
iteration. Also the fp32_kahan -> FP64 promotion."""

import os

import numpy as np
import pytest

from cturbobfm_b200 import cases

pytestmark = pytest.mark.gpu


def _mixed_cases(prec):
    """Uneven members: 2-D JST RK4, 2-D Roe RK3, axisymmetric BFM (two
    sizes, two operating points), 3-D periodic Roe MUSCL RK3 with Hall."""
    out = [
        cases.bump2d(ni=48, nj=16, n_iter=100000),
        cases.bump2d(ni=40, nj=20, scheme="Roe", muscl=True, limiter="van leer", rk=3, cfl=1.0, n_iter=100000),
        cases.meridional(ni=40, nj=16, p_ratio=1.05, speed=0.8),
        cases.meridional(ni=64, nj=24, p_ratio=1.2, speed=1.0),
        cases.annulus3d(ni=30, nj=10, nk=13, cfl=1.0),
    ]
    return [c.with_settings(GPU_PRECISION=prec) for c in out]


def _write(cs, root):
    inis = []
    for m, c in enumerate(cs):
        d = os.path.join(root, f"m{m}")
        os.makedirs(d)
        inis.append(c.write(d))
    return inis


@pytest.mark.parametrize("prec", ["fp64", "fp32_kahan"])
def test_batch_members_match_their_solo_runs_bit_for_bit(prec, tmp_path):
    from cturbobfm_b200 import Batch, Solver

    inis = _write(_mixed_cases(prec), str(tmp_path))
    n = 37  # not a multiple of the 8-iteration graph
    solo = []
    for ini in inis:
        with Solver(ini) as s:
            assert s.step(n) == n
            solo.append((s.state(), s.lognorm(), s.turbo()[1], s.time))
    solvers = [Solver(ini) for ini in inis]
    try:
        with Batch(solvers) as b:
            assert b.step(20) == 20
            assert b.step(n - 20) == n - 20
            st = b.status()
        assert (st["iterations"] == n).all() and (st["status"] == 0).all()
        for m, s in enumerate(solvers):
            u, ln, tb, t = solo[m]
            assert np.array_equal(s.state(), u), m
            assert np.array_equal(s.lognorm(), ln), m
            assert np.array_equal(st["lognorm"][m], ln), m
            assert np.array_equal(s.turbo()[1], tb), m
            assert s.time == t
            assert s.iteration == n
    finally:
        for s in solvers:
            s.close()


def test_batch_member_stops_at_its_own_convergence(tmp_path):
    from cturbobfm_b200 import Batch, Solver

    quick = cases.bump2d(ni=48, nj=16, n_iter=100000).with_settings(RESIDUALS_DROP_CONVERGENCE="2")
    slow = cases.bump2d(ni=64, nj=24, n_iter=100000)
    inis = _write([quick, slow], str(tmp_path))
    with Solver(inis[0]) as s:
        s.step(5000)
        assert s.status == 1
        it_conv = s.iteration
        u_conv = s.state()
    solvers = [Solver(ini) for ini in inis]
    try:
        with Batch(solvers) as b:
            b.step(it_conv + 100)
            st = b.status()
        assert st["status"][0] == 1 and st["iterations"][0] == it_conv
        assert st["status"][1] == 0 and st["iterations"][1] == it_conv + 100
        assert np.array_equal(solvers[0].state(), u_conv)
        assert st["best_drop"][0] >= 2.0
    finally:
        for s in solvers:
            s.close()


def test_batch_rejects_mixed_precision_and_duplicates(tmp_path):
    from cturbobfm_b200 import Batch, CtbfmError, Solver
    from cturbobfm_b200.solver import CTBFM_E_ARGUMENT

    inis = _write([cases.bump2d(ni=32, nj=12), cases.bump2d(ni=32, nj=12).with_settings(GPU_PRECISION="fp32_kahan")],
                  str(tmp_path))
    a, b = Solver(inis[0]), Solver(inis[1])
    try:
        with pytest.raises(CtbfmError) as e:
            Batch([a, b])
        assert e.value.code == CTBFM_E_ARGUMENT
        with pytest.raises(CtbfmError) as e:
            Batch([a, a])
        assert e.value.code == CTBFM_E_ARGUMENT
    finally:
        a.close()
        b.close()


def test_promotion_carries_the_solve_over_to_fp64(tmp_path):
    from cturbobfm_b200 import Solver

    ini = cases.meridional(ni=48, nj=16, p_ratio=1.1).with_settings(GPU_PRECISION="fp32_kahan").write(str(tmp_path))
    with Solver(ini) as s:
        assert s.info().precision == 1
        s.step(60)
        u = s.state()
        t = s.time
        s.promote_fp64()
        assert s.info().precision == 0
        assert s.iteration == 60 and s.time == t
        assert np.array_equal(s.state(), u)  # U - Uc carried over exactly
        assert s.step(40) == 40
        assert s.iteration == 100
        assert len(s.history()["lognorm"]) == 40
        assert np.isfinite(s.state()).all()


def test_autotuned_face_tiles_leave_results_unchanged(tmp_path, oracle_lib):
    from cturbobfm_b200 import Solver

    # 100 iterations trigger the face-tile autotuner at the first enqueue;
    # the state must still match the oracle as closely as untuned runs do
    ini = cases.bump2d(ni=96, nj=32).write(str(tmp_path))
    o = oracle_lib.Oracle(ini)
    o.run(100)
    with Solver(ini) as s:
        assert s.step(100) == 100
        tiles = list(s.info().face_tile)
        u = s.state()
    assert all(t in (256, 512, 1024, 2048) for t in tiles)
    ref = o.state()
    err = (np.abs(u - ref).max(axis=1) / np.maximum(np.abs(ref).max(axis=1), 1e-300)).max()
    assert err <= 1e-12
