"""Serving (ctbfm_server_*): requests arriving while others run are admitted
into the running batches, and each result is the same alone and in the mix
(bit for bit: every member computes on its own, and scheduling decisions
depend only on the member's own iteration count)."""

import os

import numpy as np
import pytest

from cturbobfm_b200 import cases

pytestmark = pytest.mark.gpu


def _req(name, ni, nj, pr, sp, prec="fp32_kahan", drop=3):
    return cases.meridional(ni=ni, nj=nj, p_ratio=pr, speed=sp, cfl=2.2, drop=drop, rows=cases.MAP_ROWS,
                            ramp=2000, precision=prec, n_iter=20000, name=name)


def _write(c, root):
    d = os.path.join(root, c.name)
    os.makedirs(d)
    return c.write(d)


def _drain(server, expect):
    out = {}
    for _ in range(10000):
        server.pump()
        for r in server.results():
            out[r["id"]] = r
        if len(out) == expect:
            return out
    raise AssertionError("server did not finish")


def test_results_are_the_same_alone_and_in_the_mix(tmp_path):
    from cturbobfm_b200 import Server, Solver

    a = _write(_req("a", 64, 24, 1.05, 0.95), str(tmp_path))
    others = [_write(_req("b", 96, 32, 1.1, 0.9), str(tmp_path)),
              _write(_req("c", 80, 28, 1.0, 1.0, prec="fp64"), str(tmp_path)),
              _write(_req("d", 72, 40, 1.15, 0.92), str(tmp_path)),
              _write(cases.bump2d(ni=48, nj=16, n_iter=3000, name="e").with_settings(GPU_PRECISION="fp32_kahan"),
                     str(tmp_path))]
    with Server(chunk=100) as s:
        ida = s.submit(a)
        alone = _drain(s, 1)[ida]
    assert alone["status"] == 1 and alone["error"] == 0
    # the same operating point on the plain drop-in path
    with Solver(a) as p:
        p.solve()
        assert p.status == 1
        assert p.iteration == alone["iterations"]
        assert np.array_equal(p.turbo()[1], np.array(alone["turbo"]))
    # in the mix: two requests first, A after two rounds, the rest later
    with Server(chunk=100) as s:
        ids = [s.submit(others[0]), s.submit(others[1])]
        s.pump()
        s.pump()
        ida = s.submit(a)
        s.pump()
        ids += [s.submit(others[2]), s.submit(others[3])]
        res = _drain(s, 5)
    mixed = res[ida]
    assert mixed["status"] == alone["status"]
    assert mixed["iterations"] == alone["iterations"]
    assert mixed["turbo"] == alone["turbo"] and mixed["massflow"] == alone["massflow"]
    assert all(res[i]["error"] == 0 for i in ids)
    assert res[ids[1]]["precision"] == 0  # the fp64 request stays fp64
    assert all(r["t_admit"] >= r["t_submit"] and r["t_done"] >= r["t_admit"] for r in res.values())


def test_budget_admits_one_solve_at_a_time(tmp_path):
    from cturbobfm_b200 import Server, Solver

    inis = [_write(_req(f"r{m}", 64, 24, 1.0 + 0.05 * m, 0.95), str(tmp_path)) for m in range(3)]
    # a solve's device slab is sized like the previous solve of its precision
    # (the first one of a process grows its slabs): measure the second
    for _ in range(2):
        with Solver(inis[0]) as p:
            one = int(p.info().device_bytes)
    with Server(budget_bytes=int(one * 1.5), chunk=200) as s:
        ids = [s.submit(i) for i in inis]
        res = _drain(s, 3)
    order = sorted(res.values(), key=lambda r: r["t_admit"])
    assert [r["id"] for r in order] == ids  # arrival order
    for prev, nxt in zip(order, order[1:]):
        assert nxt["t_admit"] >= prev["t_done"]  # admitted only once the previous solve left


def test_stalled_fp32_solve_continues_in_fp64_deterministically(tmp_path):
    from cturbobfm_b200 import Server

    ini = _write(_req("s", 64, 24, 1.05, 0.95), str(tmp_path))
    out = []
    for _ in range(2):
        with Server(chunk=50, stall_window=50) as s:
            rid = s.submit(ini)
            out.append(_drain(s, 1)[rid])
    assert out[0]["precision"] == 0  # promoted
    assert out[0]["status"] == 1
    assert out[0] == {**out[1], "t_submit": out[0]["t_submit"], "t_admit": out[0]["t_admit"],
                      "t_done": out[0]["t_done"], "id": out[0]["id"]}


def test_a_bad_request_fails_alone(tmp_path):
    from cturbobfm_b200 import Server

    good = _write(_req("g", 64, 24, 1.05, 0.95), str(tmp_path))
    with Server(chunk=200) as s:
        bad = s.submit(str(tmp_path / "missing" / "input.ini"))
        ok = s.submit(good)
        res = _drain(s, 2)
    assert res[bad]["error"] == 1 and res[bad]["status"] == -1
    assert res[ok]["error"] == 0 and res[ok]["status"] == 1


def test_node_limit_admits_in_arrival_order(tmp_path):
    from cturbobfm_b200 import Server

    inis = [_write(_req(f"n{m}", 64, 24, 1.0 + 0.05 * m, 0.95), str(tmp_path)) for m in range(3)]
    with Server(chunk=200, max_active_nodes=int(64 * 24 * 1.5)) as s:
        ids = [s.submit(i) for i in inis]
        res = _drain(s, 3)
    order = sorted(res.values(), key=lambda r: r["t_admit"])
    assert [r["id"] for r in order] == ids
    for prev, nxt in zip(order, order[1:]):
        assert nxt["t_admit"] >= prev["t_done"]
    assert all(r["status"] == 1 for r in res.values())


def _pressures_scaled(c, f):
    """The same flow with every pressure (initial state, inlet total and
    outlet static pressure) multiplied by f: an ideal-gas Euler solution
    scales with it, density and energy with it, velocities and temperatures
    unchanged."""
    import dataclasses

    st = dict(c.settings)
    st["INIT_PRESSURE"] = repr(float(st["INIT_PRESSURE"]) * f)
    patches = []
    for p in c.patches:
        parts = [x.strip() for x in p.spec.split(",")]
        if parts[0] in ("inlet", "outlet"):
            parts[1] = repr(float(parts[1]) * f)
        patches.append(dataclasses.replace(p, spec=", ".join(parts)))
    return dataclasses.replace(c, settings=st, patches=patches)


def test_diverged_fp32_solve_is_run_again_in_fp64(tmp_path):
    """A request whose fp32_kahan solve diverges while the FP64 solve
    converges: the bump channel with its pressures scaled by 1e36, so that
    the energy (about 2.5e41) overflows float at once while FP64 solves the
    scaled flow. A server allowed to move float solves to FP64
    (stall_window > 0) runs it again from its initial state in FP64, and the
    result is that of the plain FP64 solve."""
    from cturbobfm_b200 import Server, SolverDiverged, Solver

    c = _pressures_scaled(cases.bump2d(ni=48, nj=20), 1e36).with_settings(
        GPU_PRECISION="fp32_kahan", RESIDUALS_DROP_CONVERGENCE="2", N_ITERATIONS="10000")
    ini32 = _write(c, str(tmp_path / "f32"))
    with Solver(ini32) as s:
        with pytest.raises(SolverDiverged):
            s.solve()
    ini64 = _write(c.with_settings(GPU_PRECISION="fp64"), str(tmp_path / "f64"))
    with Solver(ini64) as s:
        s.solve()
        assert s.status == 1
        it64 = s.iteration
        mf64, tp64 = s.turbo()
    with Server(chunk=200) as srv:  # stall_window 0: the divergence is the result
        rid = srv.submit(ini32)
        r = _drain(srv, 1)[rid]
    assert r["status"] == 2 and r["precision"] == 1
    with Server(chunk=200, stall_window=100000) as srv:
        rid = srv.submit(ini32)
        r = _drain(srv, 1)[rid]
    assert r["status"] == 1 and r["precision"] == 0
    assert r["iterations"] == it64
    assert np.array_equal(np.array(r["turbo"]), tp64)
    assert np.array_equal(np.array(r["massflow"]), mf64)


def test_warm_started_request_is_the_same_alone_and_in_the_mix(tmp_path):
    """A request that restarts from another operating point's converged
    solution (RESTART_SOLUTION, nearest-neighbour mapping onto its own grid)
    converges faster than cold and gives the same result alone, in a mix, and
    on the plain drop-in path."""
    from cturbobfm_b200 import Server, Solver

    nominal = _req("n", 64, 24, 1.1, 0.95, prec="fp64")
    with Solver(_write(nominal, str(tmp_path))) as s:
        s.solve()
        assert s.status == 1
        csv = s.write_solution(str(tmp_path / "nominal.csv"))
    cold = _req("w", 80, 28, 1.05, 0.95)
    warm = cold.with_settings(RESTART_SOLUTION="yes", RESTART_SOLUTION_FILEPATH=csv,
                              RESTART_TYPE="nearest_neighbor_axisymmetric", OUTLET_PRESSURE_RAMP_ITERATIONS="0")
    ini_cold = _write(cold, str(tmp_path / "cold"))
    ini = _write(warm, str(tmp_path / "warm"))
    with Solver(ini_cold) as p:
        p.solve()
        cold_its = p.iteration
    with Solver(ini) as p:
        p.solve()
        assert p.status == 1
        plain = (p.iteration, list(p.turbo()[1]))
    assert plain[0] < cold_its
    with Server(chunk=100) as s:
        rid = s.submit(ini)
        alone = _drain(s, 1)[rid]
    other = _write(_req("o", 96, 32, 1.1, 0.9), str(tmp_path))
    with Server(chunk=100) as s:
        first = s.submit(other)
        s.pump()
        rid = s.submit(ini)
        mixed = _drain(s, 2)[rid]
    for r in (alone, mixed):
        assert r["status"] == 1
        assert r["iterations"] == plain[0]
        assert r["turbo"] == plain[1]
    assert first >= 0


def test_float_solve_moves_to_fp64_within_an_order_of_its_drop(tmp_path):
    """promote_orders = 1: a fp32_kahan request is paused on the device once
    its best residual drop is within one order of RESIDUALS_DROP_CONVERGENCE,
    its FP64 side built while the next chunk runs, and it converges in FP64;
    the same request gives the same result alone and beside another one, and
    the server statistics count the move."""
    from cturbobfm_b200 import Server

    a = _req("a", 64, 24, 1.05, 0.95, drop=4)
    b = _req("b", 72, 26, 1.10, 0.90, drop=4)
    ina, inb = _write(a, str(tmp_path)), _write(b, str(tmp_path))
    with Server(chunk=100, promote_orders=1.0) as srv:
        ra = srv.submit(ina)
        alone = _drain(srv, 1)[ra]
        st = srv.stats()
    assert alone["status"] == 1 and alone["precision"] == 0 and alone["error"] == 0
    assert st["promotions"] == 1 and st["rounds"] >= 1 and st["wait_s"] > 0
    with Server(chunk=100, promote_orders=1.0) as srv:
        ra, rb = srv.submit(ina), srv.submit(inb)
        mix = _drain(srv, 2)
    assert mix[ra]["iterations"] == alone["iterations"]
    assert np.array_equal(np.array(mix[ra]["turbo"]), np.array(alone["turbo"]))
    assert mix[rb]["status"] == 1 and mix[rb]["precision"] == 0
