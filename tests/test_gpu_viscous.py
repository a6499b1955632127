"""Laminar viscous path (VISCOSITY_ACTIVE, no-slip walls at rest) on the GPU
beyond the short parity runs: batches that mix viscous and inviscid members
stay bit for bit equal to the solo runs, and a viscous channel converges at
the oracle's iteration to the oracle's state (1e-10 relative per field after
about 800 iterations; the FP64 kernels differ from the oracle only
through pow() in Sutherland's law and the log10 of the norms)."""

import os

import numpy as np
import pytest

from cturbobfm_b200 import cases
from parity_cases import _sector, _viscous

pytestmark = pytest.mark.gpu


def _write(cs, root):
    inis = []
    for m, c in enumerate(cs):
        d = os.path.join(root, f"m{m}")
        os.makedirs(d)
        inis.append(c.write(d))
    return inis


@pytest.mark.parametrize("prec", ["fp64", "fp32_kahan"])
def test_batch_mixing_viscous_and_inviscid_members_matches_solo_runs(prec, tmp_path):
    from cturbobfm_b200 import Batch, Solver

    cs = [
        _viscous(cases.bump2d(ni=40, nj=16, n_iter=100000)),
        cases.bump2d(ni=48, nj=16, n_iter=100000),
        _viscous(_sector(30.0, nk=7), mu=0.01),
        _viscous(cases.bump2d(ni=32, nj=20, scheme="Roe", muscl=True, limiter="van albada", rk=3, cfl=0.8,
                              n_iter=100000), mu=0.02),
    ]
    inis = _write([c.with_settings(GPU_PRECISION=prec) for c in cs], str(tmp_path))
    n = 29
    solo = []
    for ini in inis:
        with Solver(ini) as s:
            assert s.step(n) == n
            solo.append((s.state(), s.lognorm()))
    solvers = [Solver(ini) for ini in inis]
    try:
        with Batch(solvers) as b:
            assert b.step(n) == n
        for m, s in enumerate(solvers):
            assert np.array_equal(s.state(), solo[m][0]), m
            assert np.array_equal(s.lognorm(), solo[m][1]), m
    finally:
        for s in solvers:
            s.close()


def test_viscous_channel_converges_like_the_oracle(tmp_path, oracle_lib):
    from cturbobfm_b200 import Solver

    c = _viscous(cases.bump2d(ni=24, nj=12, n_iter=20000), mu=0.02, RESIDUALS_DROP_CONVERGENCE="3")
    ini = c.write(str(tmp_path))
    o = oracle_lib.Oracle(ini)
    r = o.run(20000)
    assert r["converged"] == 1
    with Solver(ini) as s:
        s.solve()
        assert s.status == 1
        assert s.iteration == r["iterations"]
        u = s.state()
    ref = o.state()
    scale = np.maximum(np.abs(ref).max(axis=1), 1e-300)
    assert (np.abs(u - ref).max(axis=1) / scale).max() <= 1e-10
    # no-slip: zero momentum on the wall nodes (j = 0 and j = nj - 1)
    m = u[1:4].reshape(3, 24, 12)
    assert np.all(m[:, :, 0] == 0.0) and np.all(m[:, :, -1] == 0.0)


def test_no_slip_wall_without_viscosity_matches_the_inviscid_wall(tmp_path):
    """Without VISCOSITY_ACTIVE a no_slip_wall patch is an inviscid wall, as
    in the reference: the same states bit for bit."""
    import dataclasses

    from cturbobfm_b200 import Solver

    base = cases.bump2d(ni=40, nj=16)
    ns = cases.bump2d(ni=40, nj=16)
    for m in (2, 3):
        ns.patches[m] = dataclasses.replace(ns.patches[m], spec="no_slip_wall")
    out = []
    for k, c in enumerate((base, ns)):
        with Solver(c.write(str(tmp_path / str(k)))) as s:
            assert s.step(50) == 50
            out.append(s.state())
    assert np.array_equal(out[0], out[1])
