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
