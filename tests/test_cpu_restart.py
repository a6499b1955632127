"""The oracle's restart initialisation (Solver::initializeSolutionFromRestart,
src/solver.cpp:890-1295) against the reference: the golden fixtures of
tests/golden/restart/ (made by the reference build) and, where the reference
build is present, fresh runs of it. The oracle finds the nearest node by
exhaustive search, so it meets the reference exactly wherever no two source
nodes are at exactly the same distance; the fixtures with ties are the GPU
tests' business (the library uses the reference's k-d tree order)."""

import os
import subprocess

import numpy as np
import pytest

import golden_util as gu

NO_TIES = ["annulus_axisymmetric", "annulus_nearest_axi", "bump_standard"]


@pytest.mark.parametrize("name", NO_TIES)
def test_oracle_restart_matches_reference_fixture(name, tmp_path, oracle_lib):
    fx = gu.load_restart(name)
    o = oracle_lib.Oracle(gu.write_restart_case(fx, str(tmp_path)))
    assert np.array_equal(o.state(), fx["init_state"])
    n = int(fx["n_iter"])
    assert o.run(n)["iterations"] == n
    assert np.array_equal(o.state(), fx["state"])


def test_tie_fixtures_hold_ties(tmp_path, oracle_lib):
    """The two refined targets do have nodes half-way between source nodes,
    where a search that takes the first of equal distances differs from the
    reference's k-d tree."""
    for name in ("bump_nearest_ties", "meridional_nearest_ties"):
        fx = gu.load_restart(name)
        d = tmp_path / name
        o = oracle_lib.Oracle(gu.write_restart_case(fx, str(d)))
        differ = (o.state() != fx["init_state"]).any(axis=0)
        assert 0 < differ.sum() < 0.2 * differ.size


def _reference_solution(oracle_lib, case, directory, n_iter):
    case.with_settings(N_ITERATIONS=str(n_iter), SAVE_ITERATIONS_INTERVAL=str(n_iter),
                       OUTPUT_FIELDS_TYPE="secondary").write(directory)
    r = subprocess.run([oracle_lib.REF_CLI, "input.ini"], cwd=directory, capture_output=True, text=True,
                       env=dict(os.environ, OMP_NUM_THREADS="1"), timeout=600)
    assert r.returncode == 0, r.stderr[-400:]
    return os.path.join(directory, "Volume_CSV", "results.csv")


def _jitter(case, seed=7, eps=1e-7):
    rng = np.random.default_rng(seed)
    for a in (case.x, case.y, case.z):
        a *= 1.0 + eps * rng.standard_normal(a.shape)
    return case


def _ref_cases():
    from cturbobfm_b200 import cases

    mer = cases.meridional(ni=16, nj=7, rows=cases.MAP_ROWS, name="mer_src")
    bump = cases.bump2d(ni=24, nj=10, name="bump_src")
    ann = dict(rows=cases.MAP_ROWS, scheme="JST", muscl=False, limiter="None", rk=4, cfl=1.0)
    return {
        "bump_nearest_jittered": (bump, _jitter(cases.bump2d(ni=47, nj=19)), None),
        "bump_nearest_3d_tree": (bump, _jitter(cases.bump2d(ni=35, nj=13)), "nearest_neighbor"),
        "meridional_nearest_jittered": (mer, _jitter(cases.meridional(ni=31, nj=13, rows=cases.MAP_ROWS)), None),
        "annulus_nearest_axisymmetric": (mer, _jitter(cases.annulus3d(ni=21, nj=9, nk=5, **ann)),
                                         "nearest_neighbor_axisymmetric"),
        "annulus_axisymmetric_same_plane": (mer, cases.annulus3d(ni=16, nj=7, nk=7, **ann), "axisymmetric"),
    }


@pytest.mark.parametrize("name", sorted(_ref_cases()))
def test_oracle_restart_matches_reference_build(name, tmp_path, oracle_lib):
    if not oracle_lib.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    source, target, rtype = _ref_cases()[name]
    csv = _reference_solution(oracle_lib, source, str(tmp_path / "src"), 40)
    kw = {"RESTART_SOLUTION": "yes", "RESTART_SOLUTION_FILEPATH": csv}
    if rtype:
        kw["RESTART_TYPE"] = rtype
    ini = target.with_settings(**kw).write(str(tmp_path / "dst"))
    o = oracle_lib.Oracle(ini)
    assert np.array_equal(o.state(), oracle_lib.ref_harness("steps", ini, 0)["state"])
    o.run(5)
    assert np.array_equal(o.state(), oracle_lib.ref_harness("steps", ini, 5)["state"])


def test_oracle_real_gas_restart_matches_reference_build(tmp_path, oracle_lib):
    """FLUID_MODEL = real: temperature from the (rho, e) table, pressure by the
    25-step bisection of FluidReal::computePressure_rho_T and static energy by
    the bisection of computeStaticEnergy_p_rho (src/fluid_real.cpp:227-277)."""
    if not oracle_lib.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    import parity_cases

    src = parity_cases.CASES["co2_bump_jst_rk4"][0]()
    csv = _reference_solution(oracle_lib, src, str(tmp_path / "src"), 30)
    ini = src.with_settings(RESTART_SOLUTION="yes", RESTART_SOLUTION_FILEPATH=csv).write(str(tmp_path / "dst"))
    o = oracle_lib.Oracle(ini)
    assert np.array_equal(o.state(), oracle_lib.ref_harness("steps", ini, 0)["state"])
    o.run(5)
    assert np.array_equal(o.state(), oracle_lib.ref_harness("steps", ini, 5)["state"])


def _restart_ini(tmp_path, text, **kw):
    from cturbobfm_b200 import cases

    tmp_path.mkdir(parents=True, exist_ok=True)
    (tmp_path / "restart.csv").write_text(text)
    s = {"RESTART_SOLUTION": "yes", "RESTART_SOLUTION_FILEPATH": "restart.csv"}
    s.update(kw)
    return cases.bump2d(ni=24, nj=10).with_settings(**s).write(str(tmp_path))


def test_oracle_restart_errors(tmp_path, oracle_lib):
    fx = gu.load_restart("bump_standard")
    text = str(fx["restart_csv"])
    with pytest.raises(oracle_lib.OracleError, match="Failed to open restart file"):
        oracle_lib.Oracle(_restart_ini(tmp_path / "a", text, RESTART_SOLUTION_FILEPATH="missing.csv"))
    coarse = text.replace("NI=24", "NI=12", 1)
    lines = coarse.splitlines()
    coarse = "\n".join(lines[:4 + 12 * 10]) + "\n"
    with pytest.raises(oracle_lib.OracleError, match=r"do not match solver dimensions .* RESTART_TYPE=standard"):
        oracle_lib.Oracle(_restart_ini(tmp_path / "b", coarse, RESTART_TYPE="standard"))
    rows = text.splitlines()
    cells = rows[10].split(",")
    cells[4] = "nan"
    rows[10] = ",".join(cells)
    with pytest.raises(oracle_lib.OracleError, match="NaN or Inf encountered at row index"):
        oracle_lib.Oracle(_restart_ini(tmp_path / "c", "\n".join(rows) + "\n"))
