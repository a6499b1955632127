"""The Spalart-Allmaras model (TURBULENCE_MODEL = SA) on the GPU against the
CPU oracle, which reproduces the reference build bit for bit on these cases
(tests/test_cpu_oracle.py): the working variable nu hat after n iterations
(read from the volume CSV's "Nu Tilde" column) and the state over a longer
run, 1e-12 relative per field; and SA members in a batch with other members
bit for bit as alone."""

import os

import numpy as np
import pytest

from cturbobfm_b200 import cases
from parity_cases import CASES

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12
SA_CASES = [n for n in sorted(CASES) if "_sa" in n]


def rel_err(a, b):
    a, b = np.atleast_2d(a), np.atleast_2d(b)
    scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return (np.abs(a - b).max(axis=1) / scale).max()


def _csv_column(path, name):
    lines = open(path).read().splitlines()
    header = [h.strip() for h in lines[3].split(",")]
    col = header.index(name)
    return np.array([float(l.split(",")[col]) for l in lines[4:]])


@pytest.mark.parametrize("name", SA_CASES)
def test_nu_hat_matches_oracle(name, tmp_path, oracle_lib):
    from cturbobfm_b200 import Solver

    make, n = CASES[name]
    ini = make().write(str(tmp_path))
    o = oracle_lib.Oracle(ini)
    o.run(n)
    with Solver(ini) as s:
        assert s.step(n) == n
        csv = s.write_solution(str(tmp_path / "out.csv"))
    nu = _csv_column(csv, "Nu Tilde")
    ref = o.nuhat()
    assert np.abs(ref).max() > 0
    assert rel_err(nu, ref) <= REL_TOL


def test_long_sa_run_matches_oracle(tmp_path, oracle_lib):
    """200 iterations of the SA bump channel (JST, RK4, Sutherland air)."""
    from cturbobfm_b200 import Solver

    make, _ = CASES["bump_sa"]
    ini = make().write(str(tmp_path))
    o = oracle_lib.Oracle(ini)
    o.run(200)
    with Solver(ini) as s:
        assert s.step(200) == 200
        assert rel_err(s.state(), o.state()) <= REL_TOL
        assert np.abs(s.history()["lognorm"] - o.history()["lognorm"]).max() <= 1e-10


def test_sa_members_in_a_batch_equal_their_solo_runs(tmp_path):
    from cturbobfm_b200 import Batch, Solver

    makers = [CASES["bump_sa"][0], CASES["sector45_sa"][0], lambda: cases.bump2d(ni=30, nj=14)]
    inis = []
    for m, make in enumerate(makers):
        d = tmp_path / f"c{m}"
        os.makedirs(d)
        inis.append(make().write(str(d)))
    solo = []
    for ini in inis:
        with Solver(ini) as s:
            s.step(12)
            solo.append(s.state())
    solvers = [Solver(ini) for ini in inis]
    try:
        with Batch(solvers) as b:
            b.step(12)
        for s, ref in zip(solvers, solo):
            assert np.array_equal(s.state(), ref)
    finally:
        for s in solvers:
            s.close()
