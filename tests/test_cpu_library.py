"""The C ABI boundary without a GPU: libctbfm.so loads, exports every function
include/ctbfm.h declares (and the Python binding knows each signature), and
configuration errors come back as status codes with the reference's messages
before any device work."""

import ctypes
import os
import re
import time

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "ctbfm.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ctbfm_[a-z_0-9]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from cturbobfm_b200 import build, solver

    if not os.path.exists(solver.LIB_PATH):
        build.build()
    return solver.load_library()


def test_every_declared_symbol_is_exported(lib):
    from cturbobfm_b200 import solver

    names = declared_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
        assert name in solver.SIGNATURES, name


def test_version(lib):
    assert b"sm_100a" in lib.ctbfm_version()


def test_missing_input_file_is_a_config_error(lib, tmp_path):
    h = ctypes.c_void_p()
    rc = lib.ctbfm_create_from_ini(str(tmp_path / "nope.ini").encode(), ctypes.byref(h))
    assert rc == 1
    assert b"Failed to load configuration file" in lib.ctbfm_last_error()
    assert not h.value


@pytest.mark.parametrize("key,value,message", [
    ("TOPOLOGY", "4D", "Invalid value for key \"TOPOLOGY\""),
    ("CONVECTION_SCHEME", "AUSM", "Invalid value for key \"CONVECTION_SCHEME\""),
    ("FLUX_LIMITER", "vanalbada", "Invalid value for key \"FLUX_LIMITER\""),
    ("TIME_INTEGRATION_TYPE", "2", "Implicit time integration"),
    ("TIME_STEP_METHOD", "adaptive", "Invalid value for key \"TIME_STEP_METHOD\""),
    ("BFM_MODEL", "Correlations", "Not found value for key \"LEADING_EDGE_INDEX\""),
    ("BFM_MODEL", "Chima", "Not found value for key \"CHIMA_SCALING_FUNCTIONS_FILEPATH\""),
    ("INIT_DIRECTION", "1, 0", "INIT_DIRECTION must have 3 components"),
    ("ENABLE_GREITZER_MODELING", "yes", "Greitzer modeling is only compatible with fixed time step method"),
    ("INLET_REFERENCE_FRAME", "polar", "Invalid value for key \"INLET_REFERENCE_FRAME\""),
    ("GPU_PRECISION", "fp16", "Invalid value for key \"GPU_PRECISION\""),
    ("FLUID_MODEL", "vdw", "Invalid value for key \"FLUID_MODEL\""),
])
def test_invalid_settings_are_rejected(lib, tmp_path, key, value, message):
    from cturbobfm_b200 import cases

    ini = cases.bump2d(ni=12, nj=6).with_settings(**{key: value}).write(str(tmp_path))
    h = ctypes.c_void_p()
    rc = lib.ctbfm_create_from_ini(ini.encode(), ctypes.byref(h))
    assert rc == 1
    assert message.encode() in lib.ctbfm_last_error()


def test_null_arguments(lib):
    assert lib.ctbfm_create_from_ini(None, None) == 4
    assert lib.ctbfm_step(None, 1, None) == 4
    assert lib.ctbfm_batch_create(None, 0, None) == 4
    assert lib.ctbfm_batch_step(None, 1, None) == 4
    assert lib.ctbfm_batch_enqueue(None, 1) == 4
    assert lib.ctbfm_batch_status(None, None, None, None, None) == 4
    assert lib.ctbfm_promote_fp64(None) == 4
    arr = (ctypes.c_void_p * 2)(None, None)
    out = ctypes.c_void_p()
    assert lib.ctbfm_batch_create(arr, 2, ctypes.byref(out)) == 4
    assert out.value is None
    lib.ctbfm_batch_destroy(None)
    assert lib.ctbfm_server_submit(None, b"x", None) == 4
    assert lib.ctbfm_server_pump(None, None, None) == 4
    assert lib.ctbfm_server_results(None, None, 0, None) == 4
    lib.ctbfm_server_destroy(None)
    assert lib.ctbfm_server_set_promotion(None, 1.0) == 4
    assert lib.ctbfm_server_get_stats(None, None) == 4


def test_server_promotion_and_statistics_arguments(lib):
    import ctypes

    from cturbobfm_b200 import Server, solver

    with Server(chunk=10, host_threads=1) as s:
        assert lib.ctbfm_server_set_promotion(s._h, -1.0) == 4
        assert lib.ctbfm_server_set_promotion(s._h, float("nan")) == 4
        assert lib.ctbfm_server_set_promotion(s._h, 0.5) == 0
        assert lib.ctbfm_server_get_stats(s._h, None) == 4
        st = s.stats()  # nothing pumped yet
        assert st["rounds"] == 0 and st["rebuilds"] == 0 and st["promotions"] == 0
        assert all(st[k] == 0.0 for k, _ in solver.ServerStats._fields_ if k.endswith("_s"))
    with Server(chunk=10, host_threads=1, promote_orders=1.0) as s:
        assert s.stats()["rounds"] == 0


def test_server_reports_a_bad_request_without_device_work(lib, tmp_path):
    from cturbobfm_b200 import Server

    with Server(chunk=10, host_threads=2) as s:
        rid = s.submit(str(tmp_path / "missing" / "input.ini"))
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
    assert res[0]["message"]


def test_real_gas_table_errors_come_back_as_config_errors(lib, tmp_path):
    import os
    from cturbobfm_b200 import cases

    c = cases.with_real_gas(cases.bump2d(ni=12, nj=6), pt=8.0e6, tt=320.0, p_init=7.6e6, t_init=315.0,
                            table={"n_rho": 8, "n_e": 8, "n_p": 8, "n_T": 8, "n_s": 8})
    ini = c.write(str(tmp_path / "a"))
    os.remove(os.path.join(str(tmp_path / "a"), "fluid_table_CO2.lut"))
    h = ctypes.c_void_p()
    assert lib.ctbfm_create_from_ini(ini.encode(), ctypes.byref(h)) == 1
    assert b"FluidReal: Could not open table file at:" in lib.ctbfm_last_error()
    ini = c.with_settings(STOP_ON_TABLE_OUT_OF_BOUNDS="yes").write(str(tmp_path / "b"))
    assert lib.ctbfm_create_from_ini(ini.encode(), ctypes.byref(h)) == 1
    assert b"STOP_ON_TABLE_OUT_OF_BOUNDS" in lib.ctbfm_last_error()


def _viscous_bump(walls="no_slip_wall, 0, 0, 0", **settings):
    import dataclasses

    from cturbobfm_b200 import cases

    c = cases.bump2d(ni=12, nj=6)
    for m in (2, 3):
        c.patches[m] = dataclasses.replace(c.patches[m], spec=walls)
    kw = dict(VISCOSITY_ACTIVE="yes", FLUID_MU_CONSTANT="1e-3", FLUID_CP="1004.675", FLUID_PRANDTL_NUMBER="0.72")
    kw.update(settings)
    return c.with_settings(**{k: v for k, v in kw.items() if v is not None})


@pytest.mark.parametrize("walls,settings,message", [
    ("no_slip_wall, 0, 0, 0", {"TURBULENCE_ACTIVE": "yes"}, "Not found value for key \"TURBULENCE_MODEL\""),
    ("no_slip_wall, 0, 0, 0", {"TURBULENCE_ACTIVE": "yes", "TURBULENCE_MODEL": "kOmega"},
     "Invalid value for key \"TURBULENCE_MODEL\""),
    ("no_slip_wall, 0, 0, 0", {"TURBULENCE_ACTIVE": "yes", "TURBULENCE_MODEL": "SA", "RESTART_SOLUTION": "yes"},
     "restarted Spalart-Allmaras field"),
    ("no_slip_wall, 0, 0, 0", {"FLUID_VISCOSITY_MODEL": "Power"}, "Unknown ViscosityModel: Power"),
    ("no_slip_wall, 0, 0, 0", {"FLUID_CP": None}, "Not found value for key \"FLUID_CP\""),
    ("no_slip_wall, 0, 0, 0", {"FLUID_PRANDTL_NUMBER": None}, "Not found value for key \"FLUID_PRANDTL_NUMBER\""),
    ("no_slip_wall, 0, 0, 0", {"FLUID_VISCOSITY_MODEL": "Sutherland", "FLUID_MU_CONSTANT": None},
     "Not found value for key \"FLUID_SUTHERLAND_MU_REF\""),
    ("no_slip_wall, 0, 0, 0", {"FLUID_VISCOSITY_MODEL": "Constant", "FLUID_MU_CONSTANT": None},
     "Missing constant viscosity value"),
    ("no_slip_wall", {}, "needs the wall velocity"),
    ("no_slip_wall, 10, 0, 0", {}, "moving walls"),
    ("no_slip_wall, 0, 0, 0", {"GPU_STAGE_FUSION": "persistent"},
     "GPU_STAGE_FUSION = persistent runs ideal-gas inviscid cases"),
])
def test_viscous_settings_are_checked_before_device_work(lib, tmp_path, walls, settings, message):
    """Viscous runs: the transport keys and the no-slip walls are read with
    the reference's keys and messages when the solver is created, before any
    device call."""
    ini = _viscous_bump(walls, **settings).write(str(tmp_path))
    h = ctypes.c_void_p()
    rc = lib.ctbfm_create_from_ini(ini.encode(), ctypes.byref(h))
    assert rc == 1
    assert message.encode() in lib.ctbfm_last_error()
