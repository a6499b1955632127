"""Synthetic CTurboBFM cases: structured grids, BFM input fields, boundary patches
and input.ini settings, written in the reference's file formats.

File formats follow the reference:
  * grid CSV: ``NI=``/``NJ=``/``NK=`` header lines, a ``x,y,z[,field...]``
    header, then one row per node in i-major, k-fastest order
    (src/input.cpp:14-82);
  * ``boundaries.csv``: lines containing ``=`` are skipped, a header line
    containing ``PATCH_NAME``, then ``NAME,I_MIN,I_MAX,J_MIN,J_MAX,K_MIN,K_MAX``
    in node indices (src/solver.cpp:232-294);
  * ``input.ini``: ``KEY = value`` lines, ``;`` comments (src/config.cpp:15-44).

The workloads are seeded synthetic stand-ins for the reference's validation
geometries; no data set is involved.
"""

from __future__ import annotations

import dataclasses
import math
import os
from typing import Dict, List, Optional, Tuple

import numpy as np

# Names of the per-node input fields the grid CSV may carry
# (include/types.hpp:1036-1078). Only the ones the hot path reads are used.
BFM_FIELDS = (
    "blockage",
    "normalAxial",
    "normalRadial",
    "normalTangential",
    "rpm",
    "streamwiseLength",
    "bladePresent",
    "numberBlades",
    "bladeMetalAngle",
    "bladeGasPathAngle",
    "bladeLeanAngle",
)


@dataclasses.dataclass
class Patch:
    name: str
    i_min: int
    i_max: int
    j_min: int
    j_max: int
    k_min: int
    k_max: int
    spec: str  # right-hand side of the INI patch line, e.g. "inlet, 101325, 288.15, 1, 0, 0"

    @property
    def kind(self) -> str:
        return self.spec.split(",")[0].strip().lower()

    @property
    def values(self) -> List[float]:
        parts = [p.strip() for p in self.spec.split(",")[1:]]
        return [float(p) for p in parts if p]


@dataclasses.dataclass
class Case:
    """One operating point: grid, fields, patches and solver settings."""

    name: str
    x: np.ndarray  # (NI, NJ, NK) float64
    y: np.ndarray
    z: np.ndarray
    fields: Dict[str, np.ndarray]
    patches: List[Patch]
    settings: Dict[str, str]
    # keyword arguments of fluid_table.write for FLUID_MODEL = real (the table
    # is written next to input.ini under FLUID_TABLE_FILE)
    table: Optional[Dict] = None
    # further input files written next to input.ini (name -> text), e.g. the
    # Chima scaling functions
    files: Optional[Dict[str, str]] = None

    @property
    def shape(self) -> Tuple[int, int, int]:
        return tuple(int(s) for s in self.x.shape)  # type: ignore[return-value]

    @property
    def n_nodes(self) -> int:
        ni, nj, nk = self.shape
        return ni * nj * nk

    @property
    def n_stages(self) -> int:
        ti = self.settings.get("TIME_INTEGRATION_TYPE", "0").strip().lower()
        return 3 if ti in ("1", "rk3", "explicit_rk3", "runge_kutta_3") else 4

    def with_settings(self, **kw: str) -> "Case":
        s = dict(self.settings)
        s.update({k: str(v) for k, v in kw.items()})
        return dataclasses.replace(self, settings=s)

    # -- file output ------------------------------------------------------
    def write_side_files(self, directory: str) -> None:
        """Writes the input files the settings name besides the grid and the
        boundaries (the fluid table, ``files``) into ``directory``."""
        os.makedirs(directory, exist_ok=True)
        for name, text in (self.files or {}).items():
            with open(os.path.join(directory, name), "w") as f:
                f.write(text)
        if self.table is not None:
            from . import fluid_table

            fluid_table.write(os.path.join(directory, self.settings["FLUID_TABLE_FILE"]), **self.table)

    def write(self, directory: str) -> str:
        """Writes grid.csv, boundaries.csv and input.ini; returns the ini path."""
        os.makedirs(directory, exist_ok=True)
        ni, nj, nk = self.shape
        names = ["x", "y", "z"] + list(self.fields.keys())
        cols = [self.x, self.y, self.z] + [self.fields[n] for n in self.fields]
        data = np.stack([c.reshape(-1) for c in cols], axis=1)
        with open(os.path.join(directory, "grid.csv"), "w") as f:
            f.write(f"NDIMENSIONS={3 if nk > 1 else 2}\nNI={ni}\nNJ={nj}\nNK={nk}\n")
            f.write(",".join(names) + "\n")
            np.savetxt(f, data, fmt="%.17g", delimiter=",")
        with open(os.path.join(directory, "boundaries.csv"), "w") as f:
            f.write(f"NI={ni}\nNJ={nj}\nNK={nk}\n")
            f.write("PATCH_NAME,I_MIN,I_MAX,J_MIN,J_MAX,K_MIN,K_MAX\n")
            for p in self.patches:
                f.write(f"{p.name},{p.i_min},{p.i_max},{p.j_min},{p.j_max},{p.k_min},{p.k_max}\n")
        settings = dict(self.settings)
        settings["GRID_FILE"] = "grid.csv"
        settings["BOUNDARY_CONDITIONS_FILEPATH"] = "boundaries.csv"
        for p in self.patches:
            settings[p.name] = p.spec
        self.write_side_files(directory)
        ini = os.path.join(directory, "input.ini")
        with open(ini, "w") as f:
            f.write("[CFD]\n")
            for k, v in settings.items():
                f.write(f"{k} = {v}\n")
        return ini


def _base_settings(topology: str) -> Dict[str, str]:
    return {
        "SOLUTION_NAME": "results",
        "RESTART_SOLUTION": "no",
        "KIND_SOLVER": "Euler",
        "TOPOLOGY": topology,
        "FLUID_GAMMA": "1.4",
        "FLUID_NAME": "Air",
        "FLUID_MODEL": "Ideal",
        "FLUID_R_CONSTANT": "287.05",
        "INIT_DIRECTION": "1, 0, 0",
        "SAVE_UNSTEADY": "no",
        "SAVE_ITERATIONS_INTERVAL": "1000000",
        "HISTORY_BUFFER_SIZE": "1000000",
        "RESIDUALS_DROP_CONVERGENCE": "16",
        "TIME_INTEGRATION_TYPE": "0",
        "TIME_STEP_METHOD": "local",
        "CONVECTION_SCHEME": "JST",
        "MUSCL_RECONSTRUCTION": "no",
        "FLUX_LIMITER": "None",
        "OUTPUT_FIELDS_TYPE": "primary",
    }


def static_state(pt: float, tt: float, mach: float, gamma: float = 1.4) -> Tuple[float, float]:
    """Isentropic static pressure and temperature for a Mach number."""
    f = 1.0 + 0.5 * (gamma - 1.0) * mach * mach
    return pt * f ** (-gamma / (gamma - 1.0)), tt / f


def _tanh_cluster(n: int, beta: float) -> np.ndarray:
    """Two-sided tanh clustering of n points on [0, 1]."""
    s = np.linspace(-1.0, 1.0, n)
    return 0.5 * (1.0 + np.tanh(beta * s) / math.tanh(beta))


def bump2d(ni: int = 192, nj: int = 64, n_iter: int = 5000, cfl: float = 2.0,
           scheme: str = "JST", muscl: bool = False, limiter: str = "None",
           rk: int = 4, mach: float = 0.5, name: str = "bump2d") -> Case:
    """Circular-arc bump channel: length 3, height 1, 10%-thick arc on the lower
    wall between x = 1 and x = 2; uniform in x, two-sided tanh wall clustering
    (beta = 2) in y; total-condition inlet, static outlet for inlet Mach, walls."""
    radius = (0.25 + 0.01) / 0.2
    xs = np.linspace(0.0, 3.0, ni)
    yb = np.where((xs >= 1.0) & (xs <= 2.0),
                  np.sqrt(np.maximum(radius ** 2 - (xs - 1.5) ** 2, 0.0)) - (radius - 0.1), 0.0)
    eta = _tanh_cluster(nj, 2.0)
    x = np.repeat(xs[:, None], nj, axis=1)
    y = yb[:, None] + (1.0 - yb[:, None]) * eta[None, :]
    z = np.zeros_like(x)
    x, y, z = (a[:, :, None].copy() for a in (x, y, z))
    pt, tt = 101325.0, 288.15
    ps, ts = static_state(pt, tt, mach)
    s = _base_settings("2D")
    s.update({
        "INIT_MACH_NUMBER": f"{mach!r}",
        "INIT_TEMPERATURE": f"{ts!r}",
        "INIT_PRESSURE": f"{ps!r}",
        "CFL": f"{cfl!r}",
        "N_ITERATIONS": str(n_iter),
        "TIME_INTEGRATION_TYPE": "0" if rk == 4 else "1",
        "CONVECTION_SCHEME": scheme,
        "MUSCL_RECONSTRUCTION": "yes" if muscl else "no",
        "FLUX_LIMITER": limiter,
    })
    patches = [
        Patch("INFLOW", 0, 0, 0, nj, 0, 1, f"inlet, {pt!r}, {tt!r}, 1, 0, 0"),
        Patch("OUTFLOW", ni, ni, 0, nj, 0, 1, f"outlet, {ps!r}"),
        Patch("LOWER_WALL", 0, ni, 0, 0, 0, 1, "inviscid_wall"),
        Patch("UPPER_WALL", 0, ni, nj, nj, 0, 1, "inviscid_wall"),
    ]
    return Case(name, x, y, z, {}, patches, s)


def _row_fields(xs: np.ndarray, rs: np.ndarray, rows, nk: int) -> Dict[str, np.ndarray]:
    """BFM input fields for blade rows given as (x_le, x_te, kappa_hub_deg,
    kappa_tip_deg, rpm, n_blades, max_blockage_loss) tuples. Blockage is
    b = 1 - loss * sin^2(pi * xi) with xi the chordwise fraction, so its
    gradient is non-zero inside a row; the metal angle varies linearly from hub
    to tip; the camber normal is (-sin k, 0, cos k) in (axial, radial,
    tangential) components."""
    ni, nj = xs.size, rs.size
    shape = (ni, nj, nk)
    f = {n: np.zeros(shape) for n in BFM_FIELDS}
    f["blockage"][:] = 1.0
    span = (rs - rs[0]) / (rs[-1] - rs[0])
    for (x_le, x_te, k_hub, k_tip, rpm, nb, loss) in rows:
        inside = (xs >= x_le) & (xs <= x_te)
        if not inside.any():
            continue
        xi = (xs - x_le) / (x_te - x_le)
        kappa = np.deg2rad(k_hub + (k_tip - k_hub) * span)  # (nj,)
        for i in np.nonzero(inside)[0]:
            f["blockage"][i] = 1.0 - loss * math.sin(math.pi * xi[i]) ** 2
            f["bladePresent"][i] = 1.0
            f["numberBlades"][i] = nb
            f["rpm"][i] = rpm
            f["streamwiseLength"][i] = xs[i] - x_le
            f["bladeMetalAngle"][i] = kappa[:, None]
            f["normalAxial"][i] = -np.sin(kappa)[:, None]
            f["normalTangential"][i] = np.cos(kappa)[:, None]
    return f


def annulus3d(ni: int = 160, nj: int = 48, nk: int = 64, n_iter: int = 10000,
              cfl: float = 1.2, scheme: str = "Roe", muscl: bool = True,
              limiter: str = "van albada", rk: int = 3, bfm_model: str = "Hall",
              rpm: float = 10000.0, p_ratio: float = 1.15, mach: float = 0.3,
              name: str = "annulus3d", rows=None, speed: Optional[float] = None,
              drop: Optional[int] = None, ramp: Optional[int] = None,
              precision: Optional[str] = None, scale: float = 1.0) -> Case:
    """Full-annulus axial rotor + stator: hub radius 0.20 m, tip 0.40 m, axial
    length 0.6 m; rotor at 0.2-0.3 m (blockage loss 0.4, metal angle magnitude
    50 deg at hub to 60 deg at tip, negative in the solver's sign convention
    for positive rpm), stator at 0.35-0.45 m. k = 0 and k = nk - 1 are 360
    degree periodic duplicates (identical coordinates). ``rows`` replaces the
    blade rows (MAP_ROWS for the serving workload); ``speed``, ``drop``,
    ``ramp`` and ``precision`` set ROTATIONAL_SPEED_SCALING_FACTOR,
    RESIDUALS_DROP_CONVERGENCE, OUTLET_PRESSURE_RAMP_ITERATIONS and
    GPU_PRECISION. ``scale`` multiplies every length (grid and blade-row
    positions)."""
    xs = np.linspace(0.0, 0.6, ni) * scale
    rs = np.linspace(0.20, 0.40, nj) * scale
    th = np.array([2.0 * math.pi * k / (nk - 1) for k in range(nk - 1)] + [0.0])
    X = np.broadcast_to(xs[:, None, None], (ni, nj, nk)).copy()
    R = np.broadcast_to(rs[None, :, None], (ni, nj, nk))
    T = np.broadcast_to(th[None, None, :], (ni, nj, nk))
    Y = R * np.cos(T)
    Z = R * np.sin(T)
    if rows is None:
        rows = [(0.2, 0.3, -50.0, -60.0, rpm, 24, 0.4),
                (0.35, 0.45, 10.0, 15.0, 0.0, 30, 0.3)]
    rows = [(r[0] * scale, r[1] * scale) + tuple(r[2:]) for r in rows]
    fields = _row_fields(xs, rs, rows, nk)
    pt, tt = 101325.0, 288.15
    ps, ts = static_state(pt, tt, mach)
    s = _base_settings("3D")
    s.update({
        "BFM_ACTIVE": "yes",
        "BLOCKAGE_ACTIVE": "yes",
        "BFM_MODEL": bfm_model,
        "HALL_THOLLET_COEFFICIENT_KN": "1.0",
        "HALL_THOLLET_COEFFICIENT_KF": "1.0",
        "HALL_THOLLET_COEFFICIENT_KD": "1.0",
        "HALL_THOLLET_OFF_DESIGN_ACTIVE": "no",
        "FLUID_KINEMATIC_VISCOSITY": "1.48E-5",
        "INIT_MACH_NUMBER": f"{mach!r}",
        "INIT_TEMPERATURE": f"{ts!r}",
        "INIT_PRESSURE": f"{ps!r}",
        "CFL": f"{cfl!r}",
        "N_ITERATIONS": str(n_iter),
        "TIME_INTEGRATION_TYPE": "0" if rk == 4 else "1",
        "CONVECTION_SCHEME": scheme,
        "MUSCL_RECONSTRUCTION": "yes" if muscl else "no",
        "FLUX_LIMITER": limiter,
        "TURBO_DIRECTION": "i",
    })
    if speed is not None:
        s["ROTATIONAL_SPEED_SCALING_FACTOR"] = f"{speed!r}"
    if drop is not None:
        s["RESIDUALS_DROP_CONVERGENCE"] = str(drop)
    if ramp is not None:
        s["OUTLET_PRESSURE_RAMP_ITERATIONS"] = str(ramp)
    if precision is not None:
        s["GPU_PRECISION"] = precision
    patches = [
        Patch("INFLOW", 0, 0, 0, nj, 0, nk, f"inlet, {pt!r}, {tt!r}, 1, 0, 0"),
        Patch("OUTFLOW", ni, ni, 0, nj, 0, nk, f"outlet, {p_ratio * pt!r}"),
        Patch("HUB", 0, ni, 0, 0, 0, nk, "inviscid_wall"),
        Patch("SHROUD", 0, ni, nj, nj, 0, nk, "inviscid_wall"),
        Patch("PER1", 0, ni, 0, nj, 0, 0, "periodic, 0, 0, 360.0"),
        Patch("PER2", 0, ni, 0, nj, nk, nk, "periodic, 1, 0, 360.0"),
    ]
    return Case(name, X, Y, Z, fields, patches, s)


# Blade rows (x_le, x_te, kappa_hub_deg, kappa_tip_deg, rpm, n_blades,
# max_blockage_loss) of the rotor/stator stage of annulus3d.
STAGE_ROWS = [(0.2, 0.3, -50.0, -60.0, 10000.0, 24, 0.4),
              (0.35, 0.45, 10.0, 15.0, 0.0, 30, 0.3)]
# The compressor-map stage: the same rows with 30-40 degree rotor metal angles
# and 0.1 blockage loss. The annulus3d stage diverges in axisymmetric form
# (the oracle and the reference alike) at every back pressure of the map; this
# one converges over p_out/pt_in 1.00-1.20 and speed 85-100 %.
MAP_ROWS = [(0.2, 0.3, -30.0, -40.0, 10000.0, 24, 0.1),
            (0.35, 0.45, 10.0, 15.0, 0.0, 30, 0.1)]


def meridional(ni: int = 96, nj: int = 32, n_iter: int = 20000, cfl: float = 1.3,
               p_ratio: float = 1.15, speed: float = 1.0, bfm_model: str = "Hall",
               outlet: str = "outlet", drop: int = 8, mach: float = 0.3,
               scheme: str = "JST", rk: int = 4, name: str = "meridional",
               rows=None, ramp: Optional[int] = None, precision: Optional[str] = None) -> Case:
    """Axisymmetric meridional plane of a rotor/stator stage (nk = 1; the
    solver builds a 1 degree wedge around it). ``rows`` defaults to the
    annulus3d stage; ``ramp`` sets OUTLET_PRESSURE_RAMP_ITERATIONS and
    ``precision`` GPU_PRECISION."""
    xs = np.linspace(0.0, 0.6, ni)
    rs = np.linspace(0.20, 0.40, nj)
    X = np.broadcast_to(xs[:, None, None], (ni, nj, 1)).copy()
    Y = np.broadcast_to(rs[None, :, None], (ni, nj, 1)).copy()
    Z = np.zeros_like(X)
    fields = _row_fields(xs, rs, STAGE_ROWS if rows is None else rows, 1)
    pt, tt = 101325.0, 288.15
    ps, ts = static_state(pt, tt, mach)
    s = _base_settings("axisymmetric")
    s.update({
        "BFM_ACTIVE": "yes",
        "BLOCKAGE_ACTIVE": "yes",
        "BFM_MODEL": bfm_model,
        "HALL_THOLLET_COEFFICIENT_KN": "1.0",
        "HALL_THOLLET_COEFFICIENT_KF": "1.0",
        "HALL_THOLLET_COEFFICIENT_KD": "1.0",
        "HALL_THOLLET_OFF_DESIGN_ACTIVE": "no",
        "FLUID_KINEMATIC_VISCOSITY": "1.48E-5",
        "ROTATIONAL_SPEED_SCALING_FACTOR": f"{speed!r}",
        "INIT_MACH_NUMBER": f"{mach!r}",
        "INIT_TEMPERATURE": f"{ts!r}",
        "INIT_PRESSURE": f"{ps!r}",
        "CFL": f"{cfl!r}",
        "N_ITERATIONS": str(n_iter),
        "RESIDUALS_DROP_CONVERGENCE": str(drop),
        "TIME_INTEGRATION_TYPE": "0" if rk == 4 else "1",
        "CONVECTION_SCHEME": scheme,
        "TURBO_OUTPUT": "yes",
        "TURBO_DIRECTION": "i",
    })
    if ramp is not None:
        s["OUTLET_PRESSURE_RAMP_ITERATIONS"] = str(ramp)
    if precision is not None:
        s["GPU_PRECISION"] = precision
    if outlet == "outlet":
        out_spec = f"outlet, {p_ratio * pt!r}"
    elif outlet == "radial_equilibrium":
        out_spec = f"radial_equilibrium, {p_ratio * pt!r}"
    else:
        raise ValueError(outlet)
    patches = [
        Patch("INFLOW", 0, 0, 0, nj, 0, 1, f"inlet, {pt!r}, {tt!r}, 1, 0, 0"),
        Patch("OUTFLOW", ni, ni, 0, nj, 0, 1, out_spec),
        Patch("HUB", 0, ni, 0, 0, 0, 1, "inviscid_wall"),
        Patch("SHROUD", 0, ni, nj, nj, 0, 1, "inviscid_wall"),
    ]
    return Case(name, X, Y, Z, fields, patches, s)


def compressor_map(n: int = 256, seed: int = 20261203, ni_range=(64, 256),
                   nj_range=(24, 96), p_ratio_range=(1.00, 1.20),
                   speed_range=(0.85, 1.00), n_iter: int = 40000, drop: int = 3,
                   cfl: float = 2.2, ramp: int = 2000,
                   precision: Optional[str] = "fp32_kahan") -> List[Case]:
    """The batched compressor-map workload: n axisymmetric meridional
    instances of the MAP_ROWS stage with independently drawn grid sizes,
    back-pressure ratios and shaft-speed scalings from a seeded PCG64
    generator (draw order per instance: NI, NJ, p_out/pt_in, speed). Each
    runs JST + RK4 with local time steps at CFL 2.2, the outlet pressure
    ramped over 2000 iterations, to a residual drop of 3 orders."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for m in range(n):
        ni = int(rng.integers(ni_range[0], ni_range[1] + 1))
        nj = int(rng.integers(nj_range[0], nj_range[1] + 1))
        pr = float(rng.uniform(*p_ratio_range))
        sp = float(rng.uniform(*speed_range))
        out.append(meridional(ni=ni, nj=nj, n_iter=n_iter, p_ratio=pr, speed=sp, cfl=cfl,
                              drop=drop, name=f"map{m:03d}", rows=MAP_ROWS, ramp=ramp,
                              precision=precision))
    return out


def greitzer_plenum_volume(B: float, speed: float, r_hub: float = 0.20, r_tip: float = 0.40, length: float = 0.6,
                           rpm: float = 10000.0, tt: float = 288.15, gamma: float = 1.4, rgas: float = 287.05) -> float:
    """GREITZER_PLENUM_VOLUME for a Greitzer B parameter. The reference has no
    B key; this library maps B = U / (2 a) sqrt(V_p / (A_c L_c)) with U the
    blade speed at the mean radius, a the inlet stagnation sound speed, A_c
    the annulus area and L_c the machine length, so
    V_p = (2 a B / U)^2 A_c L_c."""
    U = rpm * speed * 2.0 * math.pi / 60.0 * 0.5 * (r_hub + r_tip)
    a = math.sqrt(gamma * rgas * tt)
    Ac = math.pi * (r_tip ** 2 - r_hub ** 2)
    return (2.0 * a * B / U) ** 2 * Ac * length


def throttle_request(ni: int, nj: int, kt: float, B: float, speed: float, name: str = "throttle",
                     precision: Optional[str] = "fp32_kahan", n_iter: int = 40000) -> Case:
    """An axisymmetric compressor-map request on a throttle with the Greitzer
    plenum (ENABLE_GREITZER_MODELING, fixed time step): throttle coefficient
    kt, B parameter mapped by greitzer_plenum_volume, time step
    dt = 1.2 / ((u + a) / dx + a / dr) with u + a = 440 m/s, a = 340 m/s on the
    grid's spacings; JST, RK4, residual drop 3 orders."""
    c = meridional(ni=ni, nj=nj, p_ratio=1.0, speed=speed, cfl=2.2, drop=3, rows=MAP_ROWS, n_iter=n_iter,
                   name=name, precision=precision)
    c.patches[1] = dataclasses.replace(c.patches[1], spec=f"throttle, {kt!r}")
    dx, dr = 0.6 / (ni - 1), 0.2 / (nj - 1)
    dt = 1.2 / (440.0 / dx + 340.0 / dr)
    return c.with_settings(TIME_STEP_METHOD="fixed", FIXED_TIME_STEP=repr(dt), ENABLE_GREITZER_MODELING="yes",
                           GREITZER_PLENUM_VOLUME=repr(greitzer_plenum_volume(B, speed)))


def serving_requests(n: int, rate: float, seed: int = 20261203, frac_3d: float = 0.3,
                     precision: Optional[str] = "fp32_kahan", frac_throttle: float = 0.2) -> List[Tuple[float, Case]]:
    """The serving workload: n operating-point requests with Poisson arrival
    times at `rate` per second, drawn from a seeded PCG64 generator (per
    request: inter-arrival gap, kind, then sizes, back pressure and speed).
    A fraction 1 - frac_3d are axisymmetric instances of the compressor map
    (NI x NJ ~ U{64..256} x U{24..96}), of which a fraction frac_throttle are
    throttle requests with the Greitzer plenum (throttle_request on NI x NJ ~
    U{64..128} x U{24..48}: kt ~ U[0.8, 1.0], B ~ U[0.1, 0.5], speed ~
    U[0.85, 0.90]; finer grids, kt 1.2 and speeds from about 0.93 on the
    finer of these grids diverge from the impulsive throttled start at any
    time step, in the oracle as on the GPU);
    the rest are 3-D annuli of the same stage
    with NI x NJ x NK ~ U{96..160} x U{32..48} x U{32..64} (JST + RK4, CFL
    2.2). Static-outlet requests: p_out/pt_in ~ U[1.00,1.20], outlet ramp 2000
    iterations. All: speed ~ U[0.85,1.00], residual drop 3 orders."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    t = 0.0
    for m in range(n):
        t += float(rng.exponential(1.0 / rate))
        is3d = bool(rng.uniform() < frac_3d)
        if is3d:
            ni, nj, nk = int(rng.integers(96, 161)), int(rng.integers(32, 49)), int(rng.integers(32, 65))
        else:
            ni, nj, nk = int(rng.integers(64, 257)), int(rng.integers(24, 97)), 1
        pr = float(rng.uniform(1.00, 1.20))
        sp = float(rng.uniform(0.85, 1.00))
        throttle = (not is3d) and bool(rng.uniform() < frac_throttle)
        if throttle:
            kt, B = float(rng.uniform(0.8, 1.0)), float(rng.uniform(0.1, 0.5))
            ni, nj = 64 + (ni - 64) // 3, 24 + (nj - 24) // 3  # U{64..128} x U{24..48}
            sp = 0.85 + (sp - 0.85) / 3.0  # U[0.85, 0.90]
            out.append((t, throttle_request(ni, nj, kt, B, sp, name=f"req{m:04d}", precision=precision)))
            continue
        if is3d:
            c = annulus3d(ni=ni, nj=nj, nk=nk, cfl=2.2, scheme="JST", muscl=False, limiter="None", rk=4,
                          p_ratio=pr, rows=MAP_ROWS, speed=sp, drop=3, ramp=2000, precision=precision,
                          n_iter=40000, name=f"req{m:04d}")
        else:
            c = meridional(ni=ni, nj=nj, n_iter=40000, p_ratio=pr, speed=sp, cfl=2.2, drop=3,
                           name=f"req{m:04d}", rows=MAP_ROWS, ramp=2000, precision=precision)
        out.append((t, c))
    return out


def with_real_gas(case: Case, pt: float, tt: float, p_init: float, t_init: float, p_out: Optional[float] = None,
                  table: Optional[Dict] = None) -> Case:
    """The same operating point in FLUID_MODEL = real with the synthetic CO2
    table of fluid_table (1e5-1e7 Pa, 200-600 K, 60 x 60 per section unless
    `table` says otherwise): inlet total conditions (pt, tt), initial static
    state (p_init, t_init), outlet static pressure p_out (default p_init)."""
    s = dict(case.settings)
    s.update({"FLUID_MODEL": "real", "FLUID_NAME": "CO2", "FLUID_TABLE_FILE": "fluid_table_CO2.lut",
              "INIT_PRESSURE": f"{p_init!r}", "INIT_TEMPERATURE": f"{t_init!r}"})
    for k in ("FLUID_GAMMA", "FLUID_R_CONSTANT"):
        s.pop(k, None)
    patches = []
    for p in case.patches:
        kind = p.kind
        if kind == "inlet":
            rest = p.spec.split(",")[3:]
            p = dataclasses.replace(p, spec=", ".join([f"inlet, {pt!r}, {tt!r}"] + [r.strip() for r in rest]))
        elif kind in ("outlet", "radial_equilibrium"):
            p = dataclasses.replace(p, spec=f"{kind}, {(p_init if p_out is None else p_out)!r}")
        patches.append(p)
    return dataclasses.replace(case, settings=s, patches=patches, table=dict(table or {}))


def realgas_annulus(ni: int = 256, nj: int = 96, nk: int = 128, n_iter: int = 10000, cfl: float = 1.0,
                    precision: Optional[str] = None, p_out: float = 8.2e6, table: Optional[Dict] = None) -> Case:
    """The real-gas workload: a compact CO2 rotor/stator annulus (annulus3d
    geometry scaled by 1/4: hub 0.05 m, tip 0.10 m, length 0.15 m; MAP_ROWS
    blade rows with the rotor at 15000 rpm), Hall body force, Roe + MUSCL
    min mod, RK3, local time step at CFL 1.0, on the synthetic CO2 table of
    fluid_table (60 x 60 per section, 1e5-1e7 Pa, 200-600 K). Inlet total
    8.0 MPa / 310 K, initial state 7.6 MPa / 305 K at Mach 0.3, outlet static
    p_out."""
    rows = [(0.2, 0.3, -30.0, -40.0, 15000.0, 24, 0.1), (0.35, 0.45, 10.0, 15.0, 0.0, 30, 0.1)]
    c = annulus3d(ni=ni, nj=nj, nk=nk, n_iter=n_iter, cfl=cfl, scheme="Roe", muscl=True, limiter="min mod", rk=3,
                  bfm_model="Hall", rows=rows, precision=precision, scale=0.25, name="realgas_annulus")
    return with_real_gas(c, pt=8.0e6, tt=310.0, p_init=7.6e6, t_init=305.0, p_out=p_out, table=table)


def viscous_annulus(ni: int = 160, nj: int = 48, nk: int = 64, n_iter: int = 10000,
                    precision: Optional[str] = None, viscous: bool = True) -> Case:
    """The laminar viscous workload: the annulus3d duct (hub 0.20 m, tip
    0.40 m, length 0.6 m, 360 degree periodic; JST, RK4, CFL 1.2: Roe +
    MUSCL RK3 diverges on this duct within about 100 iterations, with or
    without viscosity) without blade rows, static outlet at 0.95 of the inlet total
    pressure, hub and shroud as no-slip walls at rest,
    Sutherland's law for air (mu_ref 1.716e-5 Pa s at 273.15 K, S 110.4 K),
    cp 1004.675 J/(kg K), Pr 0.72. ``viscous=False`` gives the same duct with
    inviscid walls (the baseline of the viscous terms' cost)."""
    c = annulus3d(ni=ni, nj=nj, nk=nk, n_iter=n_iter, bfm_model="None", p_ratio=0.95, scheme="JST", muscl=False,
                  limiter="None", rk=4, precision=precision, name="viscous_annulus")
    c = c.with_settings(BFM_ACTIVE="no", BLOCKAGE_ACTIVE="no")
    if not viscous:
        return c
    for m in (2, 3):
        c.patches[m] = dataclasses.replace(c.patches[m], spec="no_slip_wall, 0, 0, 0")
    return c.with_settings(VISCOSITY_ACTIVE="yes", FLUID_VISCOSITY_MODEL="Sutherland",
                           FLUID_SUTHERLAND_MU_REF="1.716e-5", FLUID_SUTHERLAND_T_REF="273.15",
                           FLUID_SUTHERLAND_S="110.4", FLUID_CP="1004.675", FLUID_PRANDTL_NUMBER="0.72")


def read_grid_csv(path: str) -> Tuple[Tuple[int, int, int], Dict[str, np.ndarray]]:
    """Reads a grid CSV in the reference's format (src/input.cpp:14-82)."""
    ni = nj = nk = None
    with open(path) as f:
        while True:
            line = f.readline()
            if not line:
                raise ValueError("no x,y,z header in " + path)
            if line.startswith("NI="):
                ni = int(line[3:])
            elif line.startswith("NJ="):
                nj = int(line[3:])
            elif line.startswith("NK="):
                nk = int(line[3:])
            elif line.startswith("x,y,z"):
                names = line.strip().split(",")
                break
        data = np.loadtxt(f, delimiter=",", ndmin=2)
    shape = (ni, nj, nk)
    return shape, {n: data[:, c].reshape(shape).copy() for c, n in enumerate(names)}
