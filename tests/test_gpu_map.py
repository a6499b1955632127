"""The compressor-map front-end on the GPU against the reference build's own
files (tests/golden/map/): a speed line of P_, PREQ_ and KT_ folders run as
one batch writes turbo.csv and residuals.csv with the reference's rows,
header and time column (values at the reference's 6 significant digits),
the final volume CSV under the reference's file name, and the same
characteristics.csv."""

import os

import numpy as np
import pytest

import map_util

pytestmark = pytest.mark.gpu


def test_speed_line_matches_reference_files(tmp_path):
    from cturbobfm_b200 import compressor_map as cm

    fx, meta = map_util.write_inputs(str(tmp_path))
    res = cm.run_cases(str(tmp_path), verbose=False)
    assert set(res) == {"KT_0.9", "P_1.02", "PREQ_1.05"}  # P_1.10 has no input.ini
    for m in meta:
        if not m["volume_files"]:
            continue
        d = tmp_path / m["name"]
        for f in ("turbo.csv", "residuals.csv"):
            head, mine = map_util.table((d / f).read_text(encoding="utf-8"))
            ref_head, ref = map_util.table(str(fx[m["name"] + "/out_" + f]))
            assert head == ref_head
            assert mine.shape == ref.shape, (m["name"], f)
            cols = slice(None) if f == "residuals.csv" else slice(0, 4)
            close = np.isclose(mine[:, cols], ref[:, cols], rtol=2e-5, atol=1e-9).all(axis=1)
            rows = np.flatnonzero(~close)
            assert close.all(), (m["name"], f, rows[:5].tolist(), ref[rows[:3]].tolist(), mine[rows[:3]].tolist())
            if f == "turbo.csv":
                # (PR^k - 1) / (TR - 1) amplifies the last-bit pow difference by 1 / |TR - 1|
                eta, eta_ref, tr = mine[:, 4], ref[:, 4], ref[:, 3]
                bound = 2e-5 * np.abs(eta_ref) + 1e-9 + 1e-10 * np.abs(eta_ref) / np.maximum(np.abs(tr - 1), 1e-12)
                bad = np.abs(eta - eta_ref) > bound
                assert not bad.any(), (m["name"], np.flatnonzero(bad)[:5], ref[bad][:3], mine[bad][:3])
        assert os.path.basename(res[m["name"]]["solution"]) == m["volume_files"][-1]
    mine = cm.write_characteristics(cm.read_solutions(str(tmp_path), verbose=False), str(tmp_path / "mine.csv"))
    ref_dir = tmp_path / "ref"
    map_util.write_reference_outputs(str(ref_dir))
    os.rmdir(ref_dir / "P_1.10")
    ref = cm.write_characteristics(cm.read_solutions(str(ref_dir)), str(tmp_path / "ref.csv"))
    a = map_util.table(open(mine).read())[1]
    b = map_util.table(open(ref).read())[1]
    assert np.allclose(a, b, rtol=2e-5, atol=2e-6)
