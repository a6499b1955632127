"""A case created from memory (ctbfm_create: settings, grid arrays and
patches, no files) runs bit for bit as the same case written as input.ini +
grid CSV + boundaries.csv and created by ctbfm_create_from_ini, on every
parity case; the server takes in-memory requests (ctbfm_server_submit_case)
with the same results as ini requests."""

import os
import time

import numpy as np
import pytest

from cturbobfm_b200 import cases
from parity_cases import CASES

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(CASES))
def test_in_memory_case_runs_as_the_ini(name, tmp_path):
    from cturbobfm_b200 import Solver

    make, n = CASES[name]
    case = make()
    ini = case.write(str(tmp_path / "ini"))
    with Solver(ini) as a:
        a.step(n)
        ref, hist = a.state(), a.history()["lognorm"]
    with Solver.from_case(case, str(tmp_path / "mem")) as b:
        assert b.info().device_bytes > 0
        assert b.step(n) == n
        assert np.array_equal(b.state(), ref)
        assert np.array_equal(b.history()["lognorm"], hist)


def test_in_memory_arrays_may_be_released_after_creation(tmp_path):
    from cturbobfm_b200 import Solver

    case = cases.bump2d(ni=30, nj=14)
    ini = case.write(str(tmp_path))
    with Solver(ini) as a:
        a.step(30)
        ref = a.state()
    x, y = case.x.copy(), case.y.copy()
    s = Solver.from_case(case)
    case.x[...] = np.nan  # the library holds its own copy
    case.y[...] = np.nan
    try:
        s.step(30)
        assert np.array_equal(s.state(), ref)
    finally:
        s.close()
        case.x[...], case.y[...] = x, y


def _serve(submit, n_req):
    from cturbobfm_b200 import Server

    out = {}
    with Server(chunk=100, host_threads=2) as srv:
        ids = [submit(srv, q) for q in range(n_req)]
        t0 = time.time()
        while len(out) < n_req and time.time() - t0 < 300:
            srv.pump()
            for r in srv.results():
                out[r["id"]] = r
    return [out[i] for i in ids]


def test_server_in_memory_requests_equal_ini_requests(tmp_path):
    makers = [lambda: cases.bump2d(ni=30, nj=14).with_settings(N_ITERATIONS="400"),
              lambda: CASES["meridional_hall"][0]().with_settings(N_ITERATIONS="300"),
              lambda: CASES["meridional_chima"][0]().with_settings(N_ITERATIONS="300")]
    inis = []
    for q, m in enumerate(makers):
        inis.append(m().write(str(tmp_path / f"ini{q}")))
    by_ini = _serve(lambda srv, q: srv.submit(inis[q]), len(makers))
    by_mem = _serve(lambda srv, q: srv.submit_case(makers[q](), str(tmp_path / f"mem{q}")), len(makers))
    for a, b in zip(by_ini, by_mem):
        assert a["error"] == 0 and b["error"] == 0, (a["message"], b["message"])
        assert a["iterations"] == b["iterations"] > 0
        assert np.array_equal(np.asarray(a["massflow"]), np.asarray(b["massflow"]))
        assert np.array_equal(np.asarray(a["turbo"]), np.asarray(b["turbo"]))
    assert os.path.exists(tmp_path / "mem2")  # the Chima table was written for the in-memory request
