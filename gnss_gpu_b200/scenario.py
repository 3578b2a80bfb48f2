"""Seeded synthetic GNSS workloads standing in for the reference's datasets.

The reference's accuracy numbers come from UrbanNav / PPC / GSDC recordings
that are not available here; these generators produce the shapes and value
distributions of the benchmark configurations instead:

* single_filter(...)  -- one receiver moving at constant velocity, GPS-like
  satellites at 26,560 km with azimuth U[0, 2pi), elevation U[15, 85] deg,
  azimuth drift 0.008 deg/s, pseudorange = range + clock + N(0, sigma) and a
  fraction of satellites per epoch NLOS with +Exp(mean) bias.  8 satellites
  and one clock (the 10,000-particle CPU case), or 32 satellites in four
  constellations with one clock each (the 1,000,000-particle case).
* batched(...)        -- many independent trajectories (random heading, speed
  U[0, 20] m/s, start within 5 km of the anchor) with log-uniform particle
  counts and a satellite count drawn per filter and epoch.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

WGS84_A = 6378137.0
WGS84_F = 1.0 / 298.257223563
WGS84_E2 = WGS84_F * (2.0 - WGS84_F)
ORBIT_R = 26_560_000.0
ANCHOR_LLA = (35.63, 139.78, 40.0)  # degrees, degrees, metres


def lla_to_ecef(lat_deg, lon_deg, h):
    lat, lon = np.radians(lat_deg), np.radians(lon_deg)
    s = np.sin(lat)
    n = WGS84_A / np.sqrt(1.0 - WGS84_E2 * s * s)
    return np.array([(n + h) * np.cos(lat) * np.cos(lon),
                     (n + h) * np.cos(lat) * np.sin(lon),
                     (n * (1.0 - WGS84_E2) + h) * s])


def enu_rotation_lla(lat_deg, lon_deg):
    lat, lon = np.radians(lat_deg), np.radians(lon_deg)
    sl, cl, so, co = np.sin(lat), np.cos(lat), np.sin(lon), np.cos(lon)
    return np.array([[-so, co, 0.0], [-sl * co, -sl * so, cl], [cl * co, cl * so, sl]])


def enu_rotation_ecef(p):
    """ECEF -> local ENU rotation (rows E, N, U) at an ECEF point."""
    x, y, z = p
    lon = np.arctan2(y, x)
    rho = np.hypot(x, y)
    lat = np.arctan2(z, rho * (1.0 - WGS84_E2))
    for _ in range(8):
        s = np.sin(lat)
        nr = WGS84_A / np.sqrt(1.0 - WGS84_E2 * s * s)
        h = rho / np.cos(lat) - nr
        lat = np.arctan2(z, rho * (1.0 - WGS84_E2 * nr / (nr + h)))
    return enu_rotation_lla(np.degrees(lat), np.degrees(lon))


def sat_positions(rx_ecef, rot, az, el):
    """Satellites on the sphere of radius ORBIT_R along the receiver's
    line of sight u(az, el): |rx + rho u| = ORBIT_R."""
    u_enu = np.stack([np.cos(el) * np.sin(az), np.cos(el) * np.cos(az), np.sin(el)], axis=-1)
    u = u_enu @ rot  # ENU -> ECEF (rot rows are E, N, U)
    b = u @ rx_ecef
    c = rx_ecef @ rx_ecef - ORBIT_R ** 2
    rho = -b + np.sqrt(b * b - c)
    return rx_ecef + rho[..., None] * u


@dataclass
class Trajectory:
    truth_ecef: np.ndarray      # (E, 3)
    truth_clk: np.ndarray       # (E, n_clk)
    disp_enu: np.ndarray        # (E, 3) known displacement per epoch, local frame
    sats: list                  # per epoch (S_t, 3)
    pr: list                    # per epoch (S_t,)
    clk_idx: list               # per epoch (S_t,)
    nlos: list                  # per epoch (S_t,) bool
    anchor: np.ndarray          # (3,) start ECEF
    rot: np.ndarray             # (3, 3) ECEF -> ENU at the start


def single_filter(n_epochs=100, n_const=1, sats_per_const=8, speed_east=10.0, dt=1.0,
                  clk0=3000.0, clk_drift=0.5, sigma_pr=3.0, nlos_count=None, nlos_frac=None,
                  nlos_mean=15.0, seed=0, start_enu=(0.0, 0.0, 0.0), heading=None, speed=None,
                  sat_count=None, lla=ANCHOR_LLA):
    """One trajectory.  nlos_count satellites (or nlos_frac of them) per epoch
    get a +Exp(nlos_mean) bias.  sat_count(rng, t) may pick a per-epoch
    satellite count from the pool."""
    rng = np.random.default_rng(seed)
    base = lla_to_ecef(*lla)
    rot = enu_rotation_lla(lla[0], lla[1])
    start = base + np.asarray(start_enu, dtype=np.float64) @ rot
    n_pool = n_const * sats_per_const
    az0 = rng.uniform(0.0, 2.0 * np.pi, n_pool)
    el = np.radians(rng.uniform(15.0, 85.0, n_pool))
    drift = np.radians(0.008) * dt
    if heading is None:
        vel_enu = np.array([speed_east, 0.0, 0.0])
    else:
        vel_enu = (speed or 0.0) * np.array([np.sin(heading), np.cos(heading), 0.0])
    clk_off = clk0 + rng.uniform(-50.0, 50.0, n_const) * (n_const > 1)
    truth, tclk, disp, sats, prs, cidx, nl = [], [], [], [], [], [], []
    for t in range(n_epochs):
        p_enu = np.asarray(start_enu, dtype=np.float64) + vel_enu * dt * (t + 1)
        p = base + p_enu @ rot
        az = az0 + drift * (t + 1)
        sp = sat_positions(p, rot, az, el)
        c = clk_off + clk_drift * (t + 1)
        ci = np.repeat(np.arange(n_const), sats_per_const)
        s_all = n_pool if sat_count is None else int(sat_count(rng, t))
        sel = np.arange(n_pool) if s_all >= n_pool else np.sort(rng.choice(n_pool, s_all, replace=False))
        sp, ci = sp[sel], ci[sel]
        rng_true = np.linalg.norm(sp - p, axis=1)
        pr = rng_true + c[ci] + rng.normal(0.0, sigma_pr, len(sel))
        is_nlos = np.zeros(len(sel), bool)
        k = nlos_count if nlos_count is not None else int(round((nlos_frac or 0.0) * len(sel)))
        if k:
            idx = rng.choice(len(sel), min(k, len(sel)), replace=False)
            is_nlos[idx] = True
            pr[idx] += rng.exponential(nlos_mean, len(idx))
        truth.append(p)
        tclk.append(c)
        disp.append(vel_enu * dt)
        sats.append(sp)
        prs.append(pr)
        cidx.append(ci.astype(np.int32))
        nl.append(is_nlos)
    return Trajectory(np.array(truth), np.array(tclk), np.array(disp), sats, prs, cidx, nl, start, rot)


def config0(seed=0):
    """Plain PF, CPU-runnable: 8 satellites, one clock, 100 epochs, 10,000 particles."""
    return single_filter(n_epochs=100, n_const=1, sats_per_const=8, nlos_count=2, seed=seed)


def config1(n_epochs=1000, seed=1):
    """Drop-in at scale: 32 satellites (4 constellations x 8), 4 clocks, 25 % NLOS."""
    return single_filter(n_epochs=n_epochs, n_const=4, sats_per_const=8, nlos_frac=0.25, seed=seed)


def batched(n_filters=256, n_epochs=600, n_min=1_000, n_max=100_000, s_min=6, s_max=40, seed=2):
    """Independent trajectories with log-uniform particle counts."""
    rng = np.random.default_rng(seed)
    n_part = np.exp(rng.uniform(np.log(n_min), np.log(n_max), n_filters)).astype(np.int64)
    trajs = []
    for f in range(n_filters):
        r = rng.uniform(0.0, 5000.0)
        th = rng.uniform(0.0, 2.0 * np.pi)
        start = (r * np.sin(th), r * np.cos(th), 0.0)
        trajs.append(single_filter(
            n_epochs=n_epochs, n_const=1, sats_per_const=s_max, heading=rng.uniform(0, 2 * np.pi),
            speed=rng.uniform(0.0, 20.0), nlos_frac=0.25, start_enu=start, seed=seed * 100_003 + f,
            sat_count=lambda g, t: g.integers(s_min, s_max + 1)))
    return n_part, trajs
