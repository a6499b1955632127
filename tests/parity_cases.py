"""Small operating points shared by the oracle-pinning and GPU parity tests.
Each entry: name -> (case factory, iterations). Sizes are chosen so the CPU
oracle finishes in well under a second per case."""

import dataclasses

from cturbobfm_b200 import cases


def _throttle(greitzer: bool):
    c = cases.meridional(ni=48, nj=16, bfm_model="Hall-Thollet")
    c.patches[1] = dataclasses.replace(c.patches[1], spec="throttle, 0.5")
    kw = dict(TIME_STEP_METHOD="fixed", FIXED_TIME_STEP="2e-7")
    if greitzer:
        kw.update(ENABLE_GREITZER_MODELING="yes", GREITZER_PLENUM_VOLUME="0.05")
    return c.with_settings(**kw)


def _sector(angle_deg: float, nk: int = 9):
    """3-D annular sector with periodic k faces at the given angle and a
    cylindrical-frame swirling inlet (no BFM)."""
    import math
    import numpy as np

    c = cases.annulus3d(ni=20, nj=8, nk=nk, scheme="JST", muscl=False, rk=4, bfm_model="None")
    ni, nj = c.shape[0], c.shape[1]
    th = np.linspace(0.0, math.radians(angle_deg), nk)
    r = np.sqrt(c.y ** 2 + c.z ** 2)
    c.y[:] = r * np.cos(th)[None, None, :]
    c.z[:] = r * np.sin(th)[None, None, :]
    c.fields.clear()
    c.patches[0] = dataclasses.replace(c.patches[0], spec="inlet, 101325.0, 288.15, 1, 0, 0.3")
    c.patches[1] = dataclasses.replace(c.patches[1], spec="radial_equilibrium, 95000")
    c.patches[4] = dataclasses.replace(c.patches[4], spec=f"periodic, 0, 0, {angle_deg}")
    c.patches[5] = dataclasses.replace(c.patches[5], spec=f"periodic, 1, 0, {angle_deg}")
    s = dict(c.settings)
    s["BFM_ACTIVE"] = "no"
    s["INLET_REFERENCE_FRAME"] = "cylindrical"
    return dataclasses.replace(c, settings=s)


def _co2(case):
    """The same operating point in CO2 from the synthetic real-gas table:
    inlet 8 MPa / 320 K, initial and outlet 7.6 MPa / 315 K."""
    return cases.with_real_gas(case, pt=8.0e6, tt=320.0, p_init=7.6e6, t_init=315.0, table={"n_rho": 24, "n_e": 24, "n_p": 20, "n_T": 20, "n_s": 20})


def _bump_bc(inlet: str, outlet: str, **kw):
    """The bump channel with other inlet / outlet boundary conditions."""
    c = cases.bump2d(ni=24, nj=12, **kw)
    c.patches[0] = dataclasses.replace(c.patches[0], spec=inlet)
    c.patches[1] = dataclasses.replace(c.patches[1], spec=outlet)
    return c


def _bump_farfield():
    ps, ts = cases.static_state(101325.0, 288.15, 0.5)
    ff = f"farfield, 0.5, {ps!r}, {ts!r}, 1, 0, 0"
    return _bump_bc(ff, ff)


def _bump_farfield_supersonic():
    ps, ts = cases.static_state(101325.0, 288.15, 1.6)
    ff = f"farfield, 1.6, {ps!r}, {ts!r}, 1, 0, 0"
    return _bump_bc(ff, ff, mach=1.6, cfl=1.0)


def _bump_supersonic():
    ps, ts = cases.static_state(101325.0, 288.15, 1.6)
    u = 1.6 * (1.4 * 287.05 * ts) ** 0.5
    return _bump_bc(f"inlet_supersonic, {ps!r}, {ts!r}, {u!r}, 0, 0", "outlet_supersonic", mach=1.6, cfl=1.0)


def _mass_flow(spec: str, **settings):
    c = cases.meridional(ni=24, nj=10, rows=cases.MAP_ROWS)
    c.patches[1] = dataclasses.replace(c.patches[1], spec=spec)
    return c.with_settings(**settings) if settings else c


def _sector_mass_flow():
    c = _sector(45.0)
    c.patches[1] = dataclasses.replace(c.patches[1], spec="mass_flow, 8.0")
    return c


def _co2_farfield():
    ff = "farfield, 0.3, 7600000.0, 315.0, 1, 0, 0"
    c = _co2(cases.bump2d(ni=24, nj=12, mach=0.3))
    c.patches[0] = dataclasses.replace(c.patches[0], spec=ff)
    c.patches[1] = dataclasses.replace(c.patches[1], spec=ff)
    return c


def _chima():
    """Chima body force on the rotor row alone, with synthetic angular-momentum
    and entropy rises and scaling functions over the mass flow."""
    import numpy as np

    c = cases.meridional(ni=24, nj=10, rows=[cases.MAP_ROWS[0]], bfm_model="Chima")
    inside = c.fields["bladePresent"][:, 0, 0] > 0
    idx = np.nonzero(inside)[0]
    blade = c.fields["bladePresent"] > 0
    c.fields["deltaAngularMomentum"] = np.where(blade, 40.0 * c.y / 0.3, 0.0)
    c.fields["deltaEntropy"] = np.where(blade, 6.0, 0.0)
    table = "MassFlow,PhiTurn,PhiLoss\n" + "".join(
        f"{m!r},{t!r},{l!r}\n" for m, t, l in ((20.0, 0.8, 1.2), (40.0, 1.0, 1.0), (60.0, 1.1, 0.9), (90.0, 1.2, 0.8)))
    c = c.with_settings(LEADING_EDGE_INDEX=str(int(idx[0])), TRAILING_EDGE_INDEX=str(int(idx[-1])),
                        CHIMA_SCALING_FUNCTIONS_FILEPATH="chima.csv")
    return dataclasses.replace(c, files={"chima.csv": table})


def _correlations():
    """Correlations body force on the rotor row alone."""
    import numpy as np

    c = cases.meridional(ni=24, nj=10, rows=[cases.MAP_ROWS[0]], bfm_model="Correlations")
    idx = np.nonzero(c.fields["bladePresent"][:, 0, 0] > 0)[0]
    c.fields["bladeCamberCurvature"] = np.full_like(c.x, 2.0)
    return c.with_settings(LEADING_EDGE_INDEX=str(int(idx[0])), TRAILING_EDGE_INDEX=str(int(idx[-1])),
                           KN_CORRELATION_BFM_COEFFICIENT="0.8")


def _edges(c):
    """LEADING_EDGE_INDEX / TRAILING_EDGE_INDEX of the first blade row."""
    import numpy as np

    idx = np.nonzero(c.fields["bladePresent"][:, 0, 0] > 0)[0]
    return dict(LEADING_EDGE_INDEX=str(int(idx[0])), TRAILING_EDGE_INDEX=str(int(idx[-1])))


def _lift_drag(c):
    """Lift-Drag body force (src/source_bfm_lift_drag.cpp:3-88): design
    relative flow angle beta0 and profile-loss coefficient Kp0 per node,
    varying over the span so that both signs of (beta0 - beta) occur."""
    import numpy as np

    blade = c.fields["bladePresent"] > 0
    span = (c.fields["bladeMetalAngle"] - c.fields["bladeMetalAngle"].min())
    c.fields["liftDragBeta0"] = np.where(blade, np.deg2rad(-62.0) + 0.8 * span, 0.0)
    c.fields["liftDragKpEtamax"] = np.where(blade, 0.02 + 0.01 * span, 0.0)
    s = dict(BFM_MODEL="Lift-Drag")
    s.update(_edges(c))
    return c.with_settings(**s)


def _stall_fields(c, name, lo, hi):
    """A per-node deviation-angle field varying linearly over j from lo to
    hi (radians) inside the blade rows, so that some nodes are beyond it."""
    import numpy as np

    nj = c.shape[1]
    ramp = np.linspace(lo, hi, nj)[None, :, None]
    c.fields[name] = np.where(c.fields["bladePresent"] > 0, np.broadcast_to(ramp, c.x.shape), 0.0)


def _stalled(bfm_model):
    """STALLED_BFM_ACTIVE (src/source_bfm_base.cpp:178-185,
    src/source_bfm_thollet.cpp:79-84): nodes whose deviation exceeds
    deviationAngleStall take the camber normal as force direction (and no
    Thollet viscous force)."""
    c = cases.meridional(ni=24, nj=10, rows=cases.MAP_ROWS, bfm_model=bfm_model)
    _stall_fields(c, "deviationAngleStall", -0.05, 0.05)
    return c.with_settings(STALLED_BFM_ACTIVE="yes")


def _thollet_off_design():
    """HALL_THOLLET_OFF_DESIGN_ACTIVE (src/source_bfm_thollet.cpp:85-110):
    the off-design loss pi K_mach |delta - delta_pivot|^(2 K_d), together with
    the stalled-node rule."""
    c = _stalled("Hall-Thollet")
    _stall_fields(c, "deviationAnglePivot", -0.1, 0.1)
    return c.with_settings(HALL_THOLLET_OFF_DESIGN_ACTIVE="yes", HALL_THOLLET_COEFFICIENT_KD="1.3")


def _perturbation(c, center, radius):
    """PERTURBATION_BODY_FORCE (src/source_bfm_base.cpp:215-243): a Gaussian
    bump of the body force in space and time around `center`, active over the
    physical time the run covers."""
    return c.with_settings(PERTURBATION_BODY_FORCE="yes", PERTURBATION_CENTER=", ".join(repr(v) for v in center),
                           PERTURBATION_RADIAL_EXTENSION=repr(radius), PERTURBATION_SCALING_FACTOR="0.5",
                           PERTURBATION_TIME_START="0.0", PERTURBATION_TIME_DURATION="0.002")


def _viscous(c, mu=None, walls=(2, 3), **settings):
    """Laminar viscous run (VISCOSITY_ACTIVE) with the J-face walls made
    no-slip walls at rest: Sutherland's law for air when mu is None, else a
    constant viscosity (large, so that the viscous terms weigh in after a few
    iterations on these coarse grids)."""
    for m in walls:
        c.patches[m] = dataclasses.replace(c.patches[m], spec="no_slip_wall, 0, 0, 0")
    kw = dict(VISCOSITY_ACTIVE="yes", FLUID_CP="1004.675", FLUID_PRANDTL_NUMBER="0.72")
    if mu is None:
        kw.update(FLUID_VISCOSITY_MODEL="Sutherland", FLUID_SUTHERLAND_MU_REF="1.716e-5",
                  FLUID_SUTHERLAND_T_REF="273.15", FLUID_SUTHERLAND_S="110.4")
    else:
        kw.update(FLUID_MU_CONSTANT=repr(mu))
    kw.update(settings)
    return c.with_settings(**kw)


def _sa(c, **settings):
    """The Spalart-Allmaras model (TURBULENCE_MODEL = SA,
    src/turbulence_model_sa.cpp) on a viscous run."""
    return c.with_settings(TURBULENCE_ACTIVE="yes", TURBULENCE_MODEL="SA", **settings)


def _co2_viscous():
    c = _co2(cases.bump2d(ni=24, nj=12, mach=0.3))
    return _viscous(c, mu=5e-3, FLUID_CP="1200.0", FLUID_PRANDTL_NUMBER="0.9")


CASES = {
    "bump_jst_rk4": (lambda: cases.bump2d(ni=24, nj=12), 20),
    "bump_roe_vanalbada_rk3": (lambda: cases.bump2d(ni=24, nj=12, scheme="Roe", muscl=True, limiter="van albada", rk=3, cfl=0.8), 20),
    "bump_roe_vanleer_rk3": (lambda: cases.bump2d(ni=24, nj=12, scheme="Roe", muscl=True, limiter="van leer", rk=3, cfl=0.8), 20),
    "bump_roe_minmod_rk3": (lambda: cases.bump2d(ni=24, nj=12, scheme="Roe", muscl=True, limiter="min mod", rk=3, cfl=0.8), 20),
    "bump_roe_first_order": (lambda: cases.bump2d(ni=24, nj=12, scheme="Roe", rk=4, cfl=0.8), 20),
    "bump_global_dt": (lambda: cases.bump2d(ni=24, nj=12).with_settings(TIME_STEP_METHOD="global", CFL="1.0"), 20),
    "bump_outlet_ramp": (lambda: cases.bump2d(ni=24, nj=12).with_settings(OUTLET_PRESSURE_RAMP_ITERATIONS="10"), 20),
    "meridional_hall": (lambda: cases.meridional(ni=24, nj=10), 20),
    "meridional_thollet_radial_eq": (lambda: cases.meridional(ni=48, nj=16, bfm_model="Hall-Thollet", outlet="radial_equilibrium", p_ratio=1.0), 20),
    "meridional_throttle": (lambda: _throttle(False), 20),
    "meridional_greitzer": (lambda: _throttle(True), 20),
    "annulus_roe_hall": (lambda: cases.annulus3d(ni=20, nj=8, nk=9), 10),
    "annulus_jst_thollet": (lambda: cases.annulus3d(ni=40, nj=12, nk=17, scheme="JST", muscl=False, rk=4, bfm_model="Hall-Thollet"), 5),
    "sector45_jst_cylindrical_inlet": (lambda: _sector(45.0), 10),
    "co2_bump_jst_rk4": (lambda: _co2(cases.bump2d(ni=24, nj=12, mach=0.3)), 20),
    "co2_bump_roe_minmod_rk3": (lambda: _co2(cases.bump2d(ni=24, nj=12, scheme="Roe", muscl=True, limiter="min mod", rk=3, cfl=0.8, mach=0.3)), 20),
    "co2_meridional_hall": (lambda: _co2(cases.meridional(ni=24, nj=10, rows=cases.MAP_ROWS)), 20),
    "co2_meridional_greitzer": (lambda: _co2(_throttle(True)), 20),
    "co2_annulus_roe_hall": (lambda: _co2(cases.annulus3d(ni=20, nj=8, nk=9, rows=cases.MAP_ROWS)), 5),
    "bump_farfield": (_bump_farfield, 20),
    "bump_farfield_supersonic": (_bump_farfield_supersonic, 20),
    "bump_supersonic_in_out": (_bump_supersonic, 20),
    "bump_transparent_jst": (lambda: _bump_bc("inlet, 101325.0, 288.15, 1, 0, 0", "transparent"), 20),
    "bump_transparent_roe_muscl": (lambda: _bump_bc("inlet, 101325.0, 288.15, 1, 0, 0", "transparent", scheme="Roe",
                                                    muscl=True, limiter="van albada", rk=3, cfl=0.8), 20),
    "meridional_mass_flow_radial": (lambda: _mass_flow("mass_flow, 70.0"), 20),
    "meridional_mass_flow_uniform": (lambda: _mass_flow("mass_flow, 70.0, 101325.0, 0.1, 0",
                                                        MASS_FLOW_MAX_PRESSURE_CHANGE="0.05"), 20),
    "sector45_mass_flow": (_sector_mass_flow, 10),
    "co2_bump_farfield": (_co2_farfield, 20),
    "meridional_chima": (_chima, 20),
    "meridional_correlations": (_correlations, 20),
    "bump_viscous_sutherland": (lambda: _viscous(cases.bump2d(ni=24, nj=12)), 20),
    "bump_viscous_roe_muscl": (lambda: _viscous(cases.bump2d(ni=24, nj=12, scheme="Roe", muscl=True, limiter="van albada",
                                                             rk=3, cfl=0.8), mu=0.02), 20),
    "bump_viscous_supersonic_inlet": (lambda: _viscous(_bump_supersonic(), mu=0.01), 20),
    "bump_viscous_global_dt": (lambda: _viscous(cases.bump2d(ni=24, nj=12), mu=0.05, TIME_STEP_METHOD="global", CFL="1.0"), 20),
    "meridional_viscous_duct": (lambda: _viscous(cases.meridional(ni=24, nj=10, p_ratio=0.95), mu=0.01,
                                                 BFM_ACTIVE="no", BLOCKAGE_ACTIVE="no"), 20),
    "sector45_viscous": (lambda: _viscous(_sector(45.0), mu=0.01), 10),
    "annulus_viscous_roe": (lambda: _viscous(cases.annulus3d(ni=20, nj=8, nk=9, bfm_model="None"),
                                             BFM_ACTIVE="no", BLOCKAGE_ACTIVE="no"), 10),
    "co2_bump_viscous": (_co2_viscous, 20),
    "bump_sa": (lambda: _sa(_viscous(cases.bump2d(ni=24, nj=12))), 20),
    "bump_sa_roe_relaxed": (lambda: _sa(_viscous(cases.bump2d(ni=24, nj=12, scheme="Roe", muscl=True,
                                                              limiter="van albada", rk=3, cfl=0.8)),
                                        TURBULENCE_NU_TILDE_RATIO="5.0", IMPLICIT_UNDER_RELAXATION="0.8"), 20),
    "meridional_sa_duct": (lambda: _sa(_viscous(cases.meridional(ni=24, nj=10, p_ratio=0.95), BFM_ACTIVE="no",
                                                BLOCKAGE_ACTIVE="no"), TURBULENCE_EDDY_VISCOSITY_RATIO="0.5"), 20),
    "sector45_sa": (lambda: _sa(_viscous(_sector(45.0)), TURBULENT_PRANDTL_NUMBER="0.9"), 10),
    "meridional_lift_drag": (lambda: _lift_drag(cases.meridional(ni=24, nj=10, rows=cases.MAP_ROWS)), 20),
    "meridional_hall_stalled": (lambda: _stalled("Hall"), 20),
    "meridional_thollet_off_design_stalled": (_thollet_off_design, 20),
    "meridional_hall_perturbation": (lambda: _perturbation(cases.meridional(ni=24, nj=10, rows=cases.MAP_ROWS),
                                                           (0.25, 0.3, 0.0), 0.06), 20),
    "annulus_lift_drag_perturbation": (lambda: _perturbation(_lift_drag(cases.annulus3d(ni=20, nj=8, nk=9,
                                                                                        rows=cases.MAP_ROWS)),
                                                             (0.25, 0.0, 0.3), 0.08), 10),
}
