"""Restart and solution output through the C ABI against the reference.

* RESTART_SOLUTION: the state right after ctbfm_create_from_ini equals the
  reference build's (tests/golden/restart/*.npz) bit for bit: standard,
  axisymmetric and nearest-neighbour restarts, including refined targets
  whose nodes sit half-way between source nodes (the library's k-d tree
  resolves those ties as the reference's does); the state after a few
  iterations matches at 1e-12 relative.
* ctbfm_write_solution: the volume CSV of a case after a few iterations has
  the reference's header and its numbers at 1e-11 relative (derived fields
  such as the total pressure amplify the 1e-12 state difference).
* a written solution restarts the library and the oracle identically (ideal
  gas, real gas, fp32_kahan).
"""

import numpy as np
import pytest

import golden_util as gu

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel_err(a, b):
    scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return (np.abs(a - b).max(axis=1) / scale).max()


@pytest.mark.parametrize("name", [n for n in gu.restart_fixture_names() if not n.startswith("output_")])
def test_restart_matches_reference(name, tmp_path):
    from cturbobfm_b200 import Solver

    fx = gu.load_restart(name)
    n = int(fx["n_iter"])
    with Solver(gu.write_restart_case(fx, str(tmp_path))) as s:
        assert np.array_equal(s.state(), fx["init_state"])
        assert s.step(n) == n
        assert rel_err(s.state(), fx["state"]) <= TOL


def _csv_table(text):
    lines = text.splitlines()
    return lines[:4], np.array([[float(v) for v in l.split(",")] for l in lines[4:] if l.strip()])


@pytest.mark.parametrize("name", gu.restart_fixture_names("output_"))
def test_write_solution_matches_reference_output(name, tmp_path):
    from cturbobfm_b200 import Solver

    fx = gu.load_restart(name)
    n = int(fx["n_iter"])
    ini = gu.write_restart_case(fx, str(tmp_path), OUTPUT_FIELDS_TYPE=str(fx["fields_type"]))
    with Solver(ini) as s:
        assert s.step(n) == n
        path = s.write_solution(str(tmp_path / "solution.csv"))
    head, mine = _csv_table(open(path).read())
    ref_head, ref = _csv_table(str(fx["solution_csv"]))
    assert head == ref_head
    assert mine.shape == ref.shape
    assert np.array_equal(mine[:, :3], ref[:, :3])
    scale = np.maximum(np.abs(ref).max(axis=0), 1e-300)
    assert (np.abs(mine - ref).max(axis=0) / scale).max() <= 1e-11


def _round_trip(tmp_path, case, n_src, n_after, **restart):
    from cturbobfm_b200 import Solver
    from oracle.oracle import Oracle

    with Solver(case.write(str(tmp_path / "src"))) as s:
        s.step(n_src)
        u_src = s.state()
        csv = s.write_solution(str(tmp_path / "solution.csv"))
    kw = {"RESTART_SOLUTION": "yes", "RESTART_SOLUTION_FILEPATH": csv}
    kw.update(restart)
    ini = case.with_settings(**kw).write(str(tmp_path / "dst"))
    o = Oracle(ini)
    with Solver(ini) as s:
        u0 = s.state()
        if case.settings.get("GPU_PRECISION", "fp64") == "fp64":
            assert np.array_equal(u0, o.state())
        s.step(n_after)
        u1 = s.state()
    o.run(n_after)
    return u_src, u0, u1, o.state()


def test_written_solution_restarts_library_and_oracle_alike(tmp_path):
    from cturbobfm_b200 import cases

    u_src, u0, u1, uo = _round_trip(tmp_path, cases.bump2d(ni=48, nj=16), 30, 10)
    assert rel_err(u0, u_src) <= 1e-12  # p(rho, T), e(p, rho) round trip of the written fields
    assert rel_err(u1, uo) <= TOL


def test_real_gas_restart_matches_oracle(tmp_path):
    import parity_cases

    case = parity_cases.CASES["co2_bump_jst_rk4"][0]()
    u_src, u0, u1, uo = _round_trip(tmp_path, case, 20, 5)
    assert rel_err(u0, u_src) <= 1e-3  # the table inversions are approximate
    assert rel_err(u1, uo) <= TOL


def test_fp32_kahan_restart(tmp_path):
    from cturbobfm_b200 import cases

    case = cases.bump2d(ni=48, nj=16).with_settings(GPU_PRECISION="fp32_kahan")
    u_src, u0, u1, uo = _round_trip(tmp_path, case, 30, 10)
    assert rel_err(u0, u_src) <= 1e-6
    assert rel_err(u1, uo) <= 1e-3


def test_restart_errors(tmp_path):
    from cturbobfm_b200 import CtbfmError, Solver, cases

    fx = gu.load_restart("bump_standard")
    good = str(fx["restart_csv"])
    base = cases.bump2d(ni=24, nj=10)

    def ini_with(d, text, **kw):
        d.mkdir()
        (d / "restart.csv").write_text(text)
        s = {"RESTART_SOLUTION": "yes", "RESTART_SOLUTION_FILEPATH": "restart.csv"}
        s.update(kw)
        return base.with_settings(**s).write(str(d))

    with pytest.raises(CtbfmError, match="Failed to open restart file"):
        Solver(ini_with(tmp_path / "a", good, RESTART_SOLUTION_FILEPATH="missing.csv"))
    lines = good.replace("NI=24", "NI=12", 1).splitlines()
    with pytest.raises(CtbfmError, match=r"do not match solver dimensions .* RESTART_TYPE=standard"):
        Solver(ini_with(tmp_path / "b", "\n".join(lines[:4 + 12 * 10]) + "\n", RESTART_TYPE="standard"))
    rows = good.splitlines()
    cells = rows[10].split(",")
    cells[4] = "inf"
    rows[10] = ",".join(cells)
    with pytest.raises(CtbfmError, match="NaN or Inf encountered at row index"):
        Solver(ini_with(tmp_path / "c", "\n".join(rows) + "\n"))
    with pytest.raises(CtbfmError, match="has no \"Density\" column"):
        Solver(ini_with(tmp_path / "d", good.replace("Density", "Dens", 1)))


def test_turbo_bfm_output_is_refused(tmp_path):
    from cturbobfm_b200 import CtbfmError, Solver, cases

    c = cases.meridional(ni=16, nj=7, rows=cases.MAP_ROWS).with_settings(OUTPUT_FIELDS_TYPE="turbo_bfm")
    with Solver(c.write(str(tmp_path))) as s:
        with pytest.raises(CtbfmError, match="turbo_bfm"):
            s.write_solution(str(tmp_path / "x.csv"))
