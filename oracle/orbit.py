"""FP64 numpy restatement of the reference's input formation: broadcast
Kepler orbits and clocks, the GLONASS RK4 integrator and the Sagnac range
model.

Test infrastructure only: imported by tests/ as the checker of the device
kernels (pf_broadcast_orbits, pf_sat_positions*, pf_sagnac).  The product
never imports it.  Pinned against tests/golden/orbit_golden.json, outputs of
the reference's own CPU path (tests/golden/make_orbit_golden.py).
"""
from __future__ import annotations

import math

import numpy as np

WEEK = 604800.0

# (mu, omega_e, relativistic F) per system (python/gnss_gpu/ephemeris.py:36-63)
CONSTS = {
    "G": (3.986005e14, 7.2921151467e-5, -4.442807633e-10),
    "E": (3.986004418e14, 7.2921151467e-5, -4.442807309e-10),
    "J": (3.986005e14, 7.2921151467e-5, -4.442807633e-10),
    "C": (3.986004418e14, 7.292115e-5, -4.442807309e-10),
}


def rx_seconds_of_week(system: str, t: float) -> float:
    """gnss_time_scales.py:50-63: BDT = GPST - 14 s, GLONASS UTC scale = GPST - 18 s, folded."""
    off = {"C": 14.0, "R": 18.0}.get(system)
    if off is None:
        return float(t)
    v = float(t) - off
    while v < 0.0:
        v += WEEK
    while v >= WEEK:
        v -= WEEK
    return v


def _wrap(dt):
    dt = np.where(dt > WEEK / 2.0, dt - WEEK, dt)
    return np.where(dt < -WEEK / 2.0, dt + WEEK, dt)


def kepler(rec: dict, system: str, times) -> tuple[np.ndarray, np.ndarray]:
    """Positions [E, 3] and clocks [E] of one Kepler record (a mapping with the
    EphemerisParams field names; tgd is the delay to subtract) at GPST
    seconds of week ``times`` (ephemeris.py:428-512, ephemeris.cu:24-104)."""
    mu, om, F = CONSTS.get(system, CONSTS["G"])
    t = np.asarray([rx_seconds_of_week(system, x) for x in np.atleast_1d(times)], np.float64)
    a = rec["sqrt_a"] ** 2
    n = math.sqrt(mu / a ** 3) + rec["delta_n"]
    e = rec["e"]
    tk = _wrap(t - rec["toe"])
    M = rec["M0"] + n * tk
    E = M.copy()
    live = np.ones_like(E, bool)
    for _ in range(10):  # Newton on Kepler's equation, per element until |dE| < 1e-15
        dE = (M - E + e * np.sin(E)) / (1.0 - e * np.cos(E))
        E = np.where(live, E + dE, E)
        live &= ~(np.abs(dE) < 1e-15)
        if not live.any():
            break
    sE, cE = np.sin(E), np.cos(E)
    den = 1.0 - e * cE
    v = np.arctan2(math.sqrt(1.0 - e * e) * sE / den, (cE - e) / den)
    phi = v + rec["omega"]
    s2, c2 = np.sin(2.0 * phi), np.cos(2.0 * phi)
    u = phi + (rec["cuc"] * c2 + rec["cus"] * s2)
    r = a * (1.0 - e * cE) + (rec["crc"] * c2 + rec["crs"] * s2)
    inc = rec["i0"] + rec["idot"] * tk + (rec["cic"] * c2 + rec["cis"] * s2)
    xp, yp = r * np.cos(u), r * np.sin(u)
    Om = rec["omega0"] + (rec["omega_dot"] - om) * tk - om * rec["toe"]
    pos = np.stack([xp * np.cos(Om) - yp * np.cos(inc) * np.sin(Om),
                    xp * np.sin(Om) + yp * np.cos(inc) * np.cos(Om),
                    yp * np.sin(inc)], axis=-1)
    dt = _wrap(t - rec["toc"])
    clk = rec["af0"] + rec["af1"] * dt + rec["af2"] * dt * dt + F * e * rec["sqrt_a"] * sE - rec["tgd"]
    return pos, clk


# GLONASS PZ-90 constants (orbit_glonass.py:26-36)
GLO_RE, GLO_MU, GLO_J2, GLO_OMGE = 6378136.0, 3.9860044e14, 1.0826257e-3, 7.292115e-5


def _glo_deriv(x, acc):
    """orbit_glonass.py:67-92."""
    r2 = float(x[0] * x[0] + x[1] * x[1] + x[2] * x[2])
    if r2 <= 0.0 or not math.isfinite(r2):
        return np.zeros(6)
    r3 = r2 * math.sqrt(r2)
    w2 = GLO_OMGE * GLO_OMGE
    at = 1.5 * GLO_J2 * GLO_MU * GLO_RE ** 2 / r2 / r3
    bt = 5.0 * x[2] * x[2] / r2
    ct = -GLO_MU / r3 - at * (1.0 - bt)
    return np.array([x[3], x[4], x[5],
                     (ct + w2) * x[0] + 2.0 * GLO_OMGE * x[4] + acc[0],
                     (ct + w2) * x[1] - 2.0 * GLO_OMGE * x[3] + acc[1],
                     (ct - 2.0 * at) * x[2] + acc[2]])


def glonass(state: dict, t: float, step: float = 60.0) -> tuple[np.ndarray, float]:
    """Position and clock of a GLONASS state (keys toe, pos, vel, acc, tau_n,
    gamma_n) at GPST second of week t: fixed RK4 steps plus a residual step
    (orbit_glonass.py:95-170)."""
    el = rx_seconds_of_week("R", t) - state["toe"]
    el = float(_wrap(np.float64(el)))
    x = np.array(list(state["pos"]) + list(state["vel"]), np.float64)
    acc = np.asarray(state["acc"], np.float64)
    rem = el
    base = -step if rem < 0.0 else step
    while abs(rem) > 1.0e-9:
        h = base if abs(rem) >= abs(base) else rem
        k1 = _glo_deriv(x, acc)
        k2 = _glo_deriv(x + k1 * (h / 2.0), acc)
        k3 = _glo_deriv(x + k2 * (h / 2.0), acc)
        k4 = _glo_deriv(x + k3 * h, acc)
        x = x + (k1 + 2.0 * k2 + 2.0 * k3 + k4) * (h / 6.0)
        rem -= h
    return x[:3].copy(), -state["tau_n"] + state["gamma_n"] * el


C_LIGHT = 299792458.0
OMEGA_E = 7.2921151467e-5


def sagnac(rx, sat) -> tuple[np.ndarray, np.ndarray]:
    """Rotated satellites [n, 3] and ranges [n] (range_model.py:12-40)."""
    rx = np.asarray(rx, np.float64).reshape(3)
    sat = np.asarray(sat, np.float64).reshape(-1, 3)
    th = OMEGA_E * (np.linalg.norm(rx - sat, axis=1) / C_LIGHT)
    rot = sat.copy()
    rot[:, 0] = sat[:, 0] * np.cos(th) + sat[:, 1] * np.sin(th)
    rot[:, 1] = -sat[:, 0] * np.sin(th) + sat[:, 1] * np.cos(th)
    return rot, np.linalg.norm(rx - rot, axis=1)
