"""ctbfm_create and ctbfm_server_submit_case without a GPU: a case held in
memory (settings, grid arrays, boundary patches) passes the same host checks
as the same case written as input.ini + grid CSV + boundaries.csv and read by
ctbfm_create_from_ini, and fails them with the same status and message;
malformed descriptions are argument errors."""

import ctypes
import time

import pytest

from parity_cases import CASES


@pytest.fixture(scope="module")
def lib():
    import os

    from cturbobfm_b200 import build, solver

    if not os.path.exists(solver.LIB_PATH):
        build.build()
    return solver.load_library()


def _create(lib, case, directory=None):
    from cturbobfm_b200 import solver

    desc, keep = solver.case_desc(case, directory)
    h = ctypes.c_void_p()
    rc = lib.ctbfm_create(ctypes.byref(desc), ctypes.byref(h))
    msg = lib.ctbfm_last_error()
    if h.value:
        lib.ctbfm_destroy(h)
    del keep
    return rc, msg


def _create_from_ini(lib, case, directory):
    h = ctypes.c_void_p()
    rc = lib.ctbfm_create_from_ini(case.write(str(directory)).encode(), ctypes.byref(h))
    msg = lib.ctbfm_last_error()
    if h.value:
        lib.ctbfm_destroy(h)
    return rc, msg


@pytest.mark.parametrize("name", sorted(CASES))
def test_every_parity_case_passes_the_host_checks_in_memory(lib, tmp_path, name):
    """Every setting, patch and grid field of the parity cases is accepted from
    memory; without a GPU the first CUDA call is what fails."""
    rc, msg = _create(lib, CASES[name][0](), str(tmp_path))
    if rc != 0:
        assert rc == 2 and msg.startswith(b"cudaGetDevice"), (rc, msg)


def _bump():
    from cturbobfm_b200 import cases

    return cases.bump2d(ni=12, nj=6)


def _mutations():
    import dataclasses

    from cturbobfm_b200 import cases

    bump = _bump()
    bad_patch = dataclasses.replace(bump, patches=[dataclasses.replace(bump.patches[0], i_min=5, i_max=7)]
                                    + bump.patches[1:])
    no_blockage = cases.meridional(ni=24, nj=10)
    no_blockage = dataclasses.replace(no_blockage, fields={k: v for k, v in no_blockage.fields.items()
                                                           if k != "blockage"})
    return {
        "topology": bump.with_settings(TOPOLOGY="4D"),
        "scheme": bump.with_settings(CONVECTION_SCHEME="AUSM"),
        "cfl": bump.with_settings(CFL="abc"),
        "implicit": bump.with_settings(TIME_INTEGRATION_TYPE="2"),
        "greitzer": bump.with_settings(ENABLE_GREITZER_MODELING="yes"),
        "precision": bump.with_settings(GPU_PRECISION="fp16"),
        "fusion": bump.with_settings(GPU_STAGE_FUSION="sometimes"),
        "patch_range": bad_patch,
        "patch_type": dataclasses.replace(bump, patches=[dataclasses.replace(bump.patches[0], spec="porous_wall")]
                                          + bump.patches[1:]),
        "patch_value": dataclasses.replace(bump, patches=[dataclasses.replace(bump.patches[0], spec="inlet, 1e5, x")]
                                           + bump.patches[1:]),
        "no_blockage": no_blockage,
        "topology_vs_grid": bump.with_settings(TOPOLOGY="3D"),
    }


@pytest.mark.parametrize("which", sorted(_mutations()))
def test_invalid_cases_fail_as_from_an_ini(lib, tmp_path, which):
    case = _mutations()[which]
    rc_ini, msg_ini = _create_from_ini(lib, case, tmp_path / "ini")
    rc_mem, msg_mem = _create(lib, case)
    assert rc_ini == 1
    assert rc_mem == rc_ini
    if which == "no_blockage":  # the ini path names the grid file
        assert msg_mem.startswith(b"blockage not found in:") and msg_ini.startswith(b"blockage not found in:")
    else:
        assert msg_mem == msg_ini


def test_a_patch_without_its_setting(lib):
    import dataclasses

    from cturbobfm_b200 import cases

    bump = _bump()
    extra = dataclasses.replace(bump, patches=bump.patches + [cases.Patch("ghost", 0, 0, 0, 5, 0, 0, "")])
    from cturbobfm_b200 import solver

    desc, keep = solver.case_desc(extra)
    # the case_desc helper writes every patch's spec under its name; drop the ghost's
    n = desc.n_settings
    keys = [desc.keys[q] for q in range(n) if desc.keys[q] != b"ghost"]
    vals = [desc.values[q] for q in range(n) if desc.keys[q] != b"ghost"]
    desc.keys = (ctypes.c_char_p * len(keys))(*keys)
    desc.values = (ctypes.c_char_p * len(vals))(*vals)
    desc.n_settings = len(keys)
    h = ctypes.c_void_p()
    assert lib.ctbfm_create(ctypes.byref(desc), ctypes.byref(h)) == 1
    assert b'Missing value for key "ghost" in configuration.' in lib.ctbfm_last_error()
    del keep


def test_grid_fields_named_twice_or_as_coordinates(lib):
    import dataclasses

    bump = _bump()
    for name in ("x", "z"):
        case = dataclasses.replace(bump, fields={name: bump.x})
        rc, msg = _create(lib, case)
        assert rc == 1 and b"given twice" in msg


def test_malformed_descriptions_are_argument_errors(lib):
    from cturbobfm_b200 import solver

    h = ctypes.c_void_p()
    assert lib.ctbfm_create(None, ctypes.byref(h)) == 4
    desc, keep = solver.case_desc(_bump())
    assert lib.ctbfm_create(ctypes.byref(desc), None) == 4

    def expect(field, value, message):
        d, k = solver.case_desc(_bump())
        setattr(d, field, value)
        assert lib.ctbfm_create(ctypes.byref(d), ctypes.byref(h)) == 4, field
        assert message in lib.ctbfm_last_error()
        assert not h.value

    expect("ni", 0, b"at least 1")
    expect("nk", -3, b"at least 1")
    expect("ni", 1 << 40, b"too large")
    expect("x", None, b"null grid coordinates")
    expect("n_fields", -1, b"negative count")
    expect("n_settings", -2, b"negative count")
    expect("patches", None, b"null patch array")
    expect("keys", None, b"null settings arrays")
    d, k = solver.case_desc(_bump())
    d.keys[0] = None
    assert lib.ctbfm_create(ctypes.byref(d), ctypes.byref(h)) == 4
    assert b"null setting key or value" in lib.ctbfm_last_error()
    d, k = solver.case_desc(_bump())
    d.patches[0].name = None
    assert lib.ctbfm_create(ctypes.byref(d), ctypes.byref(h)) == 4
    assert b"null patch name" in lib.ctbfm_last_error()
    assert lib.ctbfm_server_submit_case(None, ctypes.byref(desc), None) == 4
    del keep


def test_side_files_need_a_directory():
    from cturbobfm_b200 import solver

    with pytest.raises(ValueError, match="pass a directory"):
        solver.case_desc(CASES["meridional_chima"][0]())


def test_server_reports_a_bad_in_memory_request_without_device_work(lib):
    from cturbobfm_b200 import Server

    with Server(chunk=10, host_threads=2) as s:
        # a grid that contradicts TOPOLOGY fails in the host preparation, before any device call
        rid = s.submit_case(_bump().with_settings(TOPOLOGY="3D"))
        res = []
        for _ in range(2000):
            active, waiting = s.pump()
            res += s.results()
            if res:
                break
            time.sleep(0.005)
        assert active == 0 and waiting == 0
    assert len(res) == 1 and res[0]["id"] == rid
    assert res[0]["error"] == 1 and res[0]["status"] == -1
    assert "TOPOLOGY does not match the grid's NK" in res[0]["message"]
