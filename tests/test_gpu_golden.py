"""GPU runs of the reference's regression cases against the golden fixtures
the reference build produced (tests/golden/): fixed-length runs at 1e-12
relative, runs to the convergence test (same iteration count), and the
reference's own regression gate on the converged fields."""

import numpy as np
import pytest

import golden_util as gu

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return (np.abs(a - b).max(axis=1) / scale).max()


@pytest.mark.parametrize("name", gu.fixture_names())
def test_gpu_matches_golden_iterations(name, tmp_path):
    from cturbobfm_b200 import Solver

    fx = gu.load(name)
    n = int(fx["n_iter"])
    ini = gu.write_case(fx, str(tmp_path), n)
    with Solver(ini) as s:
        assert s.step(n) == n
        assert rel_err(s.state(), fx["state"]) <= 1e-12
        h = s.history()
    assert np.abs(h["lognorm"] - fx["lognorm"]).max() <= 1e-10


@pytest.mark.parametrize("name", [n for n in gu.fixture_names() if "conv_state" in gu.load(n)])
def test_gpu_converges_like_reference(name, tmp_path):
    from cturbobfm_b200 import Solver

    fx = gu.load(name)
    ini = gu.write_case(fx, str(tmp_path), 200000)
    with Solver(ini) as s:
        done = s.solve()
        assert s.status == 1
        assert done == int(fx["conv_iterations"])
        u = s.state()
    assert rel_err(u, fx["conv_state"]) <= 1e-10
    if "shipped_Density" in fx:
        settings = {l.split("=", 1)[0].strip(): l.split("=", 1)[1].strip() for l in str(fx["ini"]).splitlines()}
        rho, p, t = gu.primitive_fields(u, float(settings["FLUID_GAMMA"]), float(settings["FLUID_R_CONSTANT"]))
        for mine, key in ((rho, "Density"), (p, "Pressure"), (t, "Temperature")):
            assert gu.l2_relative(mine, fx["shipped_" + key]) <= 3e-2
