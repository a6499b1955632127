"""The CPU oracle (oracle/ctbfm_oracle.c) pinned against the reference:
  * bit for bit against the golden fixtures made by the reference build from
    the reference's own regression cases (tests/golden/);
  * against the regression cases' shipped reference.csv with the reference's
    own gate (relative L2 <= 3e-2, test/regression_tests/test_cases.py:82-88);
  * bit for bit against the reference build on every parity case, when that
    build is present (oracle/_ref, built from the reference's sources when
    they are available).
"""

import numpy as np
import pytest

import golden_util as gu
from parity_cases import CASES


@pytest.mark.parametrize("name", gu.fixture_names())
def test_oracle_matches_golden_iterations(name, tmp_path, oracle_lib):
    fx = gu.load(name)
    n = int(fx["n_iter"])
    ini = gu.write_case(fx, str(tmp_path), n)
    o = oracle_lib.Oracle(ini)
    r = o.run(n)
    assert r["iterations"] == n
    assert np.array_equal(o.state(), fx["state"])
    h = o.history()
    assert np.array_equal(h["lognorm"], fx["lognorm"])
    assert np.array_equal(h["massflow"], fx["massflow"])
    assert np.array_equal(h["turbo"], fx["turbo"])
    assert o.time == float(fx["time"])


@pytest.mark.parametrize("name", [n for n in gu.fixture_names() if "conv_state" in gu.load(n)])
def test_oracle_converges_like_reference(name, tmp_path, oracle_lib):
    fx = gu.load(name)
    ini = gu.write_case(fx, str(tmp_path), 200000)
    o = oracle_lib.Oracle(ini)
    r = o.run(200000)
    assert r["converged"] == 1
    assert r["iterations"] == int(fx["conv_iterations"])
    assert np.array_equal(o.state(), fx["conv_state"])


@pytest.mark.parametrize("name", [n for n in gu.fixture_names() if "shipped_Density" in gu.load(n)
                                  and "conv_state" in gu.load(n)])
def test_converged_fields_pass_the_reference_regression_gate(name, oracle_lib):
    fx = gu.load(name)
    settings = dict(l.split("=", 1) for l in str(fx["ini"]).splitlines())
    settings = {k.strip(): v.strip() for k, v in settings.items()}
    rho, p, t = gu.primitive_fields(fx["conv_state"], float(settings["FLUID_GAMMA"]),
                                    float(settings["FLUID_R_CONSTANT"]))
    for mine, key in ((rho, "Density"), (p, "Pressure"), (t, "Temperature")):
        assert gu.l2_relative(mine, fx["shipped_" + key]) <= 3e-2


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_build(name, tmp_path, oracle_lib):
    if not oracle_lib.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    make, n = CASES[name]
    ini = make().write(str(tmp_path))
    o = oracle_lib.Oracle(ini)
    ro = o.run(n)
    ref = oracle_lib.ref_harness("steps", ini, n)
    assert ro["iterations"] == ref["iterations"]
    assert np.array_equal(o.state(), ref["state"])
    assert np.array_equal(o.history()["lognorm"], ref["lognorm"])
    dt_o, r_o = oracle_lib.Oracle(ini).residual()
    res = oracle_lib.ref_harness("residual", ini)
    assert np.array_equal(dt_o, res["dt"])
    assert np.array_equal(r_o, res["residual"])


def test_oracle_diverges_where_the_reference_does(tmp_path, oracle_lib):
    from cturbobfm_b200 import cases

    ini = cases.bump2d(ni=96, nj=32, scheme="Roe", muscl=True, limiter="van albada", rk=3, cfl=1.2).write(str(tmp_path))
    r = oracle_lib.Oracle(ini).run(500)
    assert r["status"] == 2 and r["iterations"] == 72
    if oracle_lib.ref_available():
        ref = oracle_lib.ref_harness("steps", ini, 500)
        assert ref["converged"] == 2 and ref["iterations"] == 71  # the diverged iteration is not recorded


def test_viscous_blade_rows_diverge_at_the_first_iteration_like_the_reference(tmp_path, oracle_lib):
    """No-slip walls through Hall blade rows: the body force of a wall node at
    rest is 0/0, so the reference's first iteration already has a NaN energy
    residual; the oracle stops at the same iteration with the same NaN nodes."""
    import numpy as np
    from parity_cases import _viscous
    from cturbobfm_b200 import cases

    ini = _viscous(cases.meridional(ni=24, nj=10), mu=0.01).write(str(tmp_path))
    r = oracle_lib.Oracle(ini).run(5)
    assert r["status"] == 2 and r["iterations"] == 1
    _, res = oracle_lib.Oracle(ini).residual()
    bad = np.isnan(res)
    assert bad[4].any() and not bad[:4].any()
    if oracle_lib.ref_available():
        assert oracle_lib.ref_harness("steps", ini, 5)["converged"] == 2
        assert np.array_equal(np.isnan(oracle_lib.ref_harness("residual", ini)["residual"]), bad)


def test_no_slip_wall_without_viscosity_is_an_inviscid_wall(tmp_path, oracle_lib):
    """Without VISCOSITY_ACTIVE the reference builds an inviscid-wall flux for
    a no_slip_wall patch and never touches its nodes."""
    import dataclasses
    from cturbobfm_b200 import cases

    base = cases.bump2d(ni=24, nj=12)
    ns = cases.bump2d(ni=24, nj=12)
    for m in (2, 3):
        ns.patches[m] = dataclasses.replace(ns.patches[m], spec="no_slip_wall")
    a = oracle_lib.Oracle(base.write(str(tmp_path / "a")))
    ini = ns.write(str(tmp_path / "b"))
    b = oracle_lib.Oracle(ini)
    a.run(10)
    b.run(10)
    assert np.array_equal(a.state(), b.state())
    if oracle_lib.ref_available():
        assert np.array_equal(oracle_lib.ref_harness("steps", ini, 10)["state"], b.state())
