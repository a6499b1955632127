"""The fp32_kahan working precision against the FP64 oracle: states after a
fixed number of iterations on the parity cases (ideal and real gas), and the
converged mass flow and total-pressure ratio of compressor-map instances.

Tolerances (stated; measured on B200): state 1e-3 relative per field (max
abs difference over max abs value, which inflates the error of near-zero
momentum components) after the parity cases' 5-20 start-up iterations, the
largest observed being 3.6e-4 (CO2 bump, JST); 1e-2 for the fixed-time-step
throttle / Greitzer cases (dt = 2e-7 s changes the state by about 1e-6 per
iteration, the same order as the float cancellation noise of the face
fluxes; observed 7.4e-4 in air, 5.1e-3 in CO2 at 8 MPa); converged mass flow
and PR 1e-4 relative."""

import numpy as np
import pytest

from cturbobfm_b200 import cases
from parity_cases import CASES

pytestmark = pytest.mark.gpu

STATE_TOL = 1e-3
STATE_TOL_FIXED_DT = 1e-2
TURBO_TOL = 1e-4


def rel_err(a, b):
    scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return (np.abs(a - b).max(axis=1) / scale).max()


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp32_kahan_state_tracks_the_oracle(name, tmp_path, oracle_lib):
    from cturbobfm_b200 import Solver

    make, n = CASES[name]
    c = make()
    ini = c.write(str(tmp_path / "fp64"))
    o = oracle_lib.Oracle(ini)
    o.run(n)
    ini32 = c.with_settings(GPU_PRECISION="fp32_kahan").write(str(tmp_path / "fp32"))
    with Solver(ini32) as s:
        assert s.info().precision == 1
        assert s.step(n) == n
        err = rel_err(s.state(), o.state())
    print(f"{name}: fp32_kahan state error {err:.2e}")
    fixed_dt = c.settings.get("TIME_STEP_METHOD") == "fixed"
    assert err <= (STATE_TOL_FIXED_DT if fixed_dt else STATE_TOL)


@pytest.mark.parametrize("m", [0, 1])
def test_converged_map_instance_matches_the_oracle(m, tmp_path, oracle_lib):
    from cturbobfm_b200 import Solver

    # small compressor-map instances (64 x 24 and 72 x 26) so the oracle converges in seconds
    c = cases.meridional(ni=64 + 8 * m, nj=24 + 2 * m, p_ratio=1.05 + 0.05 * m, speed=0.95, cfl=2.2, drop=3,
                         rows=cases.MAP_ROWS, ramp=2000, n_iter=20000, name=f"m{m}")
    ini = c.write(str(tmp_path / "fp64"))
    o = oracle_lib.Oracle(ini)
    r = o.run(20000)
    assert r["converged"] == 1
    ref = o.history()["turbo"][-1]
    ini32 = c.with_settings(GPU_PRECISION="fp32_kahan").write(str(tmp_path / "fp32"))
    with Solver(ini32) as s:
        s.solve()
        assert s.status == 1
        tb = s.turbo()[1]
        its = s.iteration
    e_mf = abs(tb[0] - ref[0]) / abs(ref[0])
    e_pr = abs(tb[1] - ref[1]) / abs(ref[1])
    print(f"map instance {m}: oracle {r['iterations']} its, fp32 {its} its; mass flow {e_mf:.2e}, PR {e_pr:.2e}")
    assert e_mf <= TURBO_TOL and e_pr <= TURBO_TOL
