"""The synthetic case generator writes the reference's file formats."""

import numpy as np

from cturbobfm_b200 import cases


def test_grid_round_trip(tmp_path):
    c = cases.annulus3d(ni=10, nj=5, nk=7)
    c.write(str(tmp_path))
    shape, cols = cases.read_grid_csv(str(tmp_path / "grid.csv"))
    assert shape == (10, 5, 7)
    assert np.array_equal(cols["x"], c.x) and np.array_equal(cols["z"], c.z)
    assert np.array_equal(cols["blockage"], c.fields["blockage"])
    # periodic duplicates: k = 0 and k = nk - 1 coincide exactly
    assert np.array_equal(c.y[:, :, 0], c.y[:, :, -1]) and np.array_equal(c.z[:, :, 0], c.z[:, :, -1])


def test_boundaries_file(tmp_path):
    c = cases.bump2d(ni=12, nj=6)
    c.write(str(tmp_path))
    rows = [l.strip() for l in open(tmp_path / "boundaries.csv") if "=" not in l]
    assert rows[0].startswith("PATCH_NAME")
    assert "OUTFLOW,12,12,0,6,0,1" in rows


def test_compressor_map_is_seeded():
    a = cases.compressor_map(n=8)
    b = cases.compressor_map(n=8)
    assert [x.shape for x in a] == [x.shape for x in b]
    assert all(64 <= x.shape[0] <= 256 and 24 <= x.shape[1] <= 96 for x in a)
    assert [x.settings["ROTATIONAL_SPEED_SCALING_FACTOR"] for x in a] == \
           [x.settings["ROTATIONAL_SPEED_SCALING_FACTOR"] for x in b]


def test_serving_requests_are_seeded_and_mixed():
    a = cases.serving_requests(40, 20.0)
    b = cases.serving_requests(40, 20.0)
    assert [t for t, _ in a] == [t for t, _ in b]
    assert [c.shape for _, c in a] == [c.shape for _, c in b]
    times = [t for t, _ in a]
    assert all(t2 > t1 for t1, t2 in zip(times, times[1:]))
    n3d = sum(c.shape[2] > 1 for _, c in a)
    assert 0 < n3d < 40
    for _, c in a:
        ni, nj, nk = c.shape
        if nk > 1:
            assert 96 <= ni <= 160 and 32 <= nj <= 48 and 32 <= nk <= 64
        else:
            assert 64 <= ni <= 256 and 24 <= nj <= 96
        assert c.settings["RESIDUALS_DROP_CONVERGENCE"] == "3"


def test_synthetic_co2_table_is_consistent(tmp_path):
    import numpy as np

    from cturbobfm_b200 import fluid_table as ft

    t = ft.generate(n_rho=20, n_e=20, n_p=16, n_T=16, n_s=16)
    for key in ("rho_e", "p_T", "p_s"):
        assert np.isfinite(t[key][4]).all()
    # the (p, T) table inverts the equation of state
    p0, p1, T0, T1, pt = t["p_T"]
    P = np.linspace(p0, p1, pt.shape[0])
    T = np.linspace(T0, T1, pt.shape[1])
    for i in (0, 7, 15):
        for j in (0, 9, 15):
            rho = pt[i, j, 0]
            assert abs(ft.pressure_rho_T(rho, T[j]) - P[i]) <= 1e-6 * P[i]
    # above the critical temperature the sound speed is real and positive
    assert (pt[:, T > ft.T_CRIT, 2] > 0).all()
    path = ft.write(str(tmp_path / "t.lut"), n_rho=8, n_e=8, n_p=8, n_T=8, n_s=8)
    text = open(path).read()
    for marker in ("# SECTION: RHO_E", "# SECTION: P_T", "# SECTION: P_S", "NOMINAL_GAMMA:", "E_MAX:", "T_MAX:", "S_MAX:"):
        assert marker in text
