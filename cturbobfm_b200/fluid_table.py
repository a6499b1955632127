"""Synthetic real-gas look-up tables in the reference's ``.lut`` format.

The reference loads a thermodynamic table for ``FLUID_MODEL = real``
(``FluidReal::loadTable``, src/fluid_real.cpp:12-208) that its own script
fills from CoolProp. CoolProp is not available here, so this module writes a
table of the same layout from a van der Waals equation of state with a
constant ideal-gas heat capacity, fitted to CO2's critical point:

    p = rho R T / (1 - b rho) - a rho^2          e = cv T - a rho
    s = cv ln(T / T0) + R ln((1/rho - b) / (1/rho0 - b))
    c^2 = (dp/drho)_e + p / rho^2 (dp/de)_rho  (clipped below at 1e-3 R T)

with a = 27 R^2 Tc^2 / (64 pc), b = R Tc / (8 pc). The equation is explicit
in (rho, e); (p, T) takes the stable root of the cubic (lowest Gibbs energy
among the mechanically stable roots) and (p, s) a bisection in rho along the
isentrope. The numbers are a stand-in with the right structure (a critical
point inside the table, strongly non-ideal compressibility near it), not
CO2 data.

Sections (all uniform grids, first index outer):
  RHO_E  p T a s mu kappa dp_drho dp_de     over (rho, e)
  P_T    rho e a s                           over (p, T)
  P_S    rho T e                             over (p, s)
"""

from __future__ import annotations

import math
import os
from typing import Dict

import numpy as np

# CO2 constants used for the fit
MOLAR_MASS = 0.0440098        # kg/mol
R_GAS = 8.314462618 / MOLAR_MASS
T_CRIT = 304.1282             # K
P_CRIT = 7.3773e6             # Pa
CV = 700.0                    # J/(kg K), constant ideal-gas part
A_VDW = 27.0 * R_GAS ** 2 * T_CRIT ** 2 / (64.0 * P_CRIT)
B_VDW = R_GAS * T_CRIT / (8.0 * P_CRIT)
RHO_CRIT = 1.0 / (3.0 * B_VDW)
T_REF, RHO_REF = 298.15, 1.8  # entropy origin
MU, KAPPA = 2.0e-5, 2.0e-2    # constant transport properties


def pressure_rho_T(rho, T):
    return rho * R_GAS * T / (1.0 - B_VDW * rho) - A_VDW * rho * rho


def energy_rho_T(rho, T):
    return CV * T - A_VDW * rho


def temperature_rho_e(rho, e):
    return (e + A_VDW * rho) / CV


def entropy_rho_T(rho, T):
    return CV * np.log(T / T_REF) + R_GAS * np.log((1.0 / rho - B_VDW) / (1.0 / RHO_REF - B_VDW))


def derivatives_rho_e(rho, e):
    """(dp/drho)_e and (dp/de)_rho."""
    d = 1.0 - B_VDW * rho
    dp_de = rho * R_GAS / (CV * d)
    dp_drho = R_GAS * ((e + 2.0 * A_VDW * rho) * d + rho * (e + A_VDW * rho) * B_VDW) / (CV * d * d) \
        - 2.0 * A_VDW * rho
    return dp_drho, dp_de


def sound_speed_rho_e(rho, e):
    T = temperature_rho_e(rho, e)
    p = pressure_rho_T(rho, T)
    dp_drho, dp_de = derivatives_rho_e(rho, e)
    c2 = dp_drho + p / (rho * rho) * dp_de
    return np.sqrt(np.maximum(c2, 1e-3 * R_GAS * np.maximum(T, 1.0)))


def density_p_T(p: float, T: float) -> float:
    """Stable root of a b rho^3 - a rho^2 + (R T + p b) rho - p = 0."""
    roots = np.roots([A_VDW * B_VDW, -A_VDW, R_GAS * T + p * B_VDW, -p])
    best, best_g = None, None
    for r in roots:
        if abs(r.imag) > 1e-9 * max(1.0, abs(r.real)):
            continue
        rho = float(r.real)
        if not (0.0 < rho < 1.0 / B_VDW):
            continue
        e = energy_rho_T(rho, T)
        dp_drho, dp_de = derivatives_rho_e(rho, e)
        c2 = dp_drho + p / (rho * rho) * dp_de
        if c2 <= 0.0 and best is not None:
            continue
        g = e + p / rho - T * float(entropy_rho_T(rho, T))
        if best is None or g < best_g:
            best, best_g = rho, g
    if best is None:
        raise ValueError(f"no density for p={p}, T={T}")
    return best


def density_p_s(p: float, s: float, rho_lo: float, rho_hi: float) -> float:
    """rho on the isentrope s where p(rho, T(rho, s)) = p (bisection)."""
    def T_of(rho):
        return T_REF * math.exp((s - R_GAS * math.log((1.0 / rho - B_VDW) / (1.0 / RHO_REF - B_VDW))) / CV)

    def f(rho):
        return float(pressure_rho_T(rho, T_of(rho))) - p

    lo, hi = rho_lo, rho_hi
    flo, fhi = f(lo), f(hi)
    if flo >= 0.0:
        return lo
    if fhi <= 0.0:
        return hi
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if f(mid) < 0.0:
            lo = mid
        else:
            hi = mid
        if hi - lo <= 1e-13 * hi:
            break
    return 0.5 * (lo + hi)


def generate(p_min: float = 1.0e5, p_max: float = 1.0e7, T_min: float = 200.0, T_max: float = 600.0,
             n_rho: int = 60, n_e: int = 60, n_p: int = 60, n_T: int = 60, n_s: int = 60) -> Dict:
    """All three sections as arrays (the table the reference would load)."""
    P = np.linspace(p_min, p_max, n_p)
    T = np.linspace(T_min, T_max, n_T)
    pt = np.zeros((n_p, n_T, 4))
    for i, p in enumerate(P):
        for j, t in enumerate(T):
            rho = density_p_T(float(p), float(t))
            e = float(energy_rho_T(rho, t))
            pt[i, j] = (rho, e, float(sound_speed_rho_e(rho, e)), float(entropy_rho_T(rho, t)))
    rho_min, rho_max = float(pt[:, :, 0].min()), float(pt[:, :, 0].max())
    e_min, e_max = float(pt[:, :, 1].min()), float(pt[:, :, 1].max())
    s_min, s_max = float(pt[:, :, 3].min()), float(pt[:, :, 3].max())

    rho_g = np.linspace(rho_min, rho_max, n_rho)
    e_g = np.linspace(e_min, e_max, n_e)
    R_, E_ = np.meshgrid(rho_g, e_g, indexing="ij")
    T_re = temperature_rho_e(R_, E_)
    p_re = pressure_rho_T(R_, T_re)
    dpr, dpe = derivatives_rho_e(R_, E_)
    re = np.stack([p_re, T_re, sound_speed_rho_e(R_, E_), entropy_rho_T(R_, np.maximum(T_re, 1e-3)),
                   np.full_like(R_, MU), np.full_like(R_, KAPPA), dpr, dpe], axis=-1)

    S = np.linspace(s_min, s_max, n_s)
    ps = np.zeros((n_p, n_s, 3))
    lo, hi = 0.5 * rho_min, min(0.999 / B_VDW, 1.5 * rho_max)
    for i, p in enumerate(P):
        for j, s in enumerate(S):
            rho = density_p_s(float(p), float(s), lo, hi)
            t = T_REF * math.exp((s - R_GAS * math.log((1.0 / rho - B_VDW) / (1.0 / RHO_REF - B_VDW))) / CV)
            ps[i, j] = (rho, t, float(energy_rho_T(rho, t)))
    return {"rho_e": (rho_min, rho_max, e_min, e_max, re), "p_T": (p_min, p_max, T_min, T_max, pt),
            "p_s": (p_min, p_max, s_min, s_max, ps)}


def write(path: str, name: str = "CO2", **kw) -> str:
    """Writes the table in the reference's .lut layout; returns the path."""
    t = generate(**kw)
    fmt = "%.17g"
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        f.write("# Synthetic van der Waals table (CO2 critical point), written by cturbobfm_b200.fluid_table\n")
        f.write(f"FLUID_NAME: {name}\n")
        f.write(f"MOLAR_MASS: {MOLAR_MASS!r}\n")
        f.write(f"GAS_CONSTANT: {R_GAS!r}\n")
        f.write(f"CRITICAL_PRESSURE: {P_CRIT!r}\n")
        f.write(f"CRITICAL_TEMPERATURE: {T_CRIT!r}\n")
        f.write(f"CRITICAL_DENSITY: {RHO_CRIT!r}\n")
        f.write(f"NOMINAL_GAMMA: {(CV + R_GAS) / CV!r}\n\n")
        for sec, keys, cols in (("RHO_E", ("N_RHO", "N_E", "RHO_MIN", "RHO_MAX", "E_MIN", "E_MAX"), "rho_e"),
                                ("P_T", ("N_P", "N_T", "P_MIN", "P_MAX", "T_MIN", "T_MAX"), "p_T"),
                                ("P_S", ("N_P", "N_S", "P_MIN", "P_MAX", "S_MIN", "S_MAX"), "p_s")):
            xmin, xmax, ymin, ymax, data = t[cols]
            f.write(f"# SECTION: {sec}\n")
            vals = (data.shape[0], data.shape[1], xmin, xmax, ymin, ymax)
            for k, v in zip(keys, vals):
                f.write(f"{k}: {v if isinstance(v, int) else repr(float(v))}\n")
            for i in range(data.shape[0]):
                for j in range(data.shape[1]):
                    f.write(" ".join(fmt % x for x in data[i, j]) + "\n")
            f.write("\n")
    return path
