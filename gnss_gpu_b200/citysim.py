"""Box-building city simulator for the learned NLOS likelihood.

A city is a square of `size` metres in the local E/N frame of the anchor,
cut into `cell`-metre blocks.  Each block holds a building with probability
`occupancy`: an axis-aligned box with footprint U[20, 60] m on each side
(centred in the block, so the block edges are always street) and height
log-uniform in [10, 150] m.  Receivers drive along the block edges (the
street grid) at 1.5 m above ground.

A satellite is blocked (NLOS) at a receiver position when the ray from the
receiver toward the satellite hits any box before it climbs above the
tallest building.  The ray walks the block grid cell by cell (Amanatides and
Woo's traversal) and is tested against the box of every occupied cell with
the slab method.  Blocked satellites get a pseudorange bias +Exp(mean 20 m)
and C/N0 ~ N(35, 5) dB-Hz; line-of-sight ones C/N0 ~ N(45, 4).

Everything is vectorised NumPy and seeded; the GPU never runs this code.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import scenario as S

RX_HEIGHT = 1.5


@dataclass
class City:
    size: float
    cell: float
    n: int                  # blocks per side
    occ: np.ndarray         # (n, n) bool, [ix, iy]
    box: np.ndarray         # (n, n, 4) x0, x1, y0, y1 (local E/N, m)
    height: np.ndarray      # (n, n) m
    hmax: float


def make_city(seed: int, size: float = 2000.0, cell: float = 80.0, occupancy: float = 0.4) -> City:
    rng = np.random.default_rng(seed)
    n = int(round(size / cell))
    occ = rng.random((n, n)) < occupancy
    w = rng.uniform(20.0, 60.0, (n, n))
    d = rng.uniform(20.0, 60.0, (n, n))
    h = np.exp(rng.uniform(np.log(10.0), np.log(150.0), (n, n)))
    cx = (np.arange(n)[:, None] + 0.5) * cell + np.zeros((n, n))
    cy = (np.arange(n)[None, :] + 0.5) * cell + np.zeros((n, n))
    box = np.stack([cx - w / 2, cx + w / 2, cy - d / 2, cy + d / 2], axis=-1)
    h = np.where(occ, h, 0.0)
    return City(size, cell, n, occ, box, h, float(h.max()) if occ.any() else 0.0)


def los_blocked(city: City, p: np.ndarray, az: np.ndarray, el: np.ndarray) -> np.ndarray:
    """True where the ray from p (R, 3) local E/N/U toward azimuth az,
    elevation el (radians, el > 0) hits a building."""
    p = np.asarray(p, np.float64).reshape(-1, 3)
    az = np.broadcast_to(np.asarray(az, np.float64), (len(p),))
    el = np.broadcast_to(np.asarray(el, np.float64), (len(p),))
    dx = np.cos(el) * np.sin(az)
    dy = np.cos(el) * np.cos(az)
    dz = np.sin(el)
    t_end = np.maximum(city.hmax - p[:, 2], 0.0) / dz  # above every roof afterwards
    c = city.cell
    ix = np.floor(p[:, 0] / c).astype(np.int64)
    iy = np.floor(p[:, 1] / c).astype(np.int64)
    sx = np.where(dx > 0, 1, -1)
    sy = np.where(dy > 0, 1, -1)
    big = 1e30
    with np.errstate(divide="ignore", invalid="ignore"):
        inv_dx = np.where(np.abs(dx) > 1e-12, 1.0 / dx, big)
        inv_dy = np.where(np.abs(dy) > 1e-12, 1.0 / dy, big)
    t_max_x = np.where(np.abs(dx) > 1e-12, ((ix + (sx > 0)) * c - p[:, 0]) * inv_dx, big)
    t_max_y = np.where(np.abs(dy) > 1e-12, ((iy + (sy > 0)) * c - p[:, 1]) * inv_dy, big)
    t_dx = np.where(np.abs(dx) > 1e-12, c * np.abs(inv_dx), big)
    t_dy = np.where(np.abs(dy) > 1e-12, c * np.abs(inv_dy), big)
    blocked = np.zeros(len(p), bool)
    t_cur = np.zeros(len(p))
    alive = t_end > 0
    steps = los_steps(city)
    for _ in range(steps):
        if not alive.any():
            break
        inside = alive & (ix >= 0) & (ix < city.n) & (iy >= 0) & (iy < city.n)
        if inside.any():
            k = np.nonzero(inside)[0]
            bx, by = ix[k], iy[k]
            occ = city.occ[bx, by]
            k = k[occ]
            if len(k):
                b = city.box[ix[k], iy[k]]
                h = city.height[ix[k], iy[k]]
                t0x = (b[:, 0] - p[k, 0]) * inv_dx[k]
                t1x = (b[:, 1] - p[k, 0]) * inv_dx[k]
                t0y = (b[:, 2] - p[k, 1]) * inv_dy[k]
                t1y = (b[:, 3] - p[k, 1]) * inv_dy[k]
                # rays parallel to a slab: inside it or never
                par_x = np.abs(dx[k]) <= 1e-12
                par_y = np.abs(dy[k]) <= 1e-12
                inx = (p[k, 0] >= b[:, 0]) & (p[k, 0] <= b[:, 1])
                iny = (p[k, 1] >= b[:, 2]) & (p[k, 1] <= b[:, 3])
                lo_x = np.where(par_x, np.where(inx, -big, big), np.minimum(t0x, t1x))
                hi_x = np.where(par_x, np.where(inx, big, -big), np.maximum(t0x, t1x))
                lo_y = np.where(par_y, np.where(iny, -big, big), np.minimum(t0y, t1y))
                hi_y = np.where(par_y, np.where(iny, big, -big), np.maximum(t0y, t1y))
                lo_z = (0.0 - p[k, 2]) / dz[k]
                hi_z = (h - p[k, 2]) / dz[k]
                t_in = np.maximum(np.maximum(lo_x, lo_y), np.maximum(lo_z, 0.0))
                t_out = np.minimum(np.minimum(hi_x, hi_y), hi_z)
                blocked[k] |= t_in <= t_out
        # step to the next cell
        go_x = t_max_x < t_max_y
        t_cur = np.where(go_x, t_max_x, t_max_y)
        ix = np.where(go_x, ix + sx, ix)
        iy = np.where(go_x, iy, iy + sy)
        t_max_x = np.where(go_x, t_max_x + t_dx, t_max_x)
        t_max_y = np.where(go_x, t_max_y, t_max_y + t_dy)
        alive = alive & ~blocked & (t_cur <= t_end)
    return blocked


def los_steps(city: City) -> int:
    """Cells a ray may cross in los_blocked before it is declared clear."""
    return int(np.ceil(2.0 * (city.hmax / np.tan(np.radians(5.0))) / city.cell)) + 4


def los_blocked_device(city: City, p: np.ndarray, az: np.ndarray, el: np.ndarray) -> np.ndarray:
    """los_blocked on the GPU (pf_city_los): the same DDA in FP64 with the
    same rounding, so the flags equal the host's.  The city's arrays stay on
    the device (cached on the City object)."""
    import ctypes as C

    import torch

    from . import _native as N

    p = np.asarray(p, np.float64).reshape(-1, 3)
    az = np.broadcast_to(np.asarray(az, np.float64), (len(p),))
    el = np.broadcast_to(np.asarray(el, np.float64), (len(p),))
    d = np.stack([np.cos(el) * np.sin(az), np.cos(el) * np.cos(az), np.sin(el)], axis=1)
    out = np.zeros(len(p), bool)
    if len(p) == 0:
        return out
    dev = torch.device("cuda", torch.cuda.current_device())
    cache = getattr(city, "_dev", None)
    if cache is None or cache[0] != dev:
        cache = (dev, torch.from_numpy(np.ascontiguousarray(city.occ, dtype=np.uint8)).to(dev),
                 torch.from_numpy(np.ascontiguousarray(city.box, dtype=np.float64)).to(dev),
                 torch.from_numpy(np.ascontiguousarray(city.height, dtype=np.float64)).to(dev))
        city._dev = cache
    _, d_occ, d_box, d_h = cache
    d_p = torch.from_numpy(np.ascontiguousarray(p)).to(dev)
    d_d = torch.from_numpy(np.ascontiguousarray(d)).to(dev)
    d_b = torch.empty(len(p), dtype=torch.uint8, device=dev)
    ptr = lambda x: C.c_void_p(x.data_ptr())  # noqa: E731
    N.check(N.load().pf_city_los(ptr(d_occ), ptr(d_box), ptr(d_h), int(city.n), float(city.cell),
                                 float(city.hmax), los_steps(city), ptr(d_p), ptr(d_d), len(p), ptr(d_b),
                                 C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))
    out[:] = d_b.cpu().numpy() != 0
    return out


@dataclass
class CityTrajectory:
    """A drive through one city plus its GNSS observations."""
    city: City
    truth_enu: np.ndarray       # (E, 3)
    truth_ecef: np.ndarray      # (E, 3)
    truth_clk: np.ndarray       # (E, 1)
    disp_enu: np.ndarray        # (E, 3) displacement of epoch t (from t-1)
    sats: list                  # per epoch (S, 3) ECEF
    az: list                    # per epoch (S,) radians, at the true position
    el: list
    pr: list                    # per epoch (S,)
    cn0: list                   # per epoch (S,) dB-Hz
    nlos: list                  # per epoch (S,) bool
    bias: list                  # per epoch (S,) m (0 for LOS)
    anchor: np.ndarray          # (3,) ECEF of the city origin
    rot: np.ndarray             # (3, 3) ECEF -> ENU


def drive_many(city: City, n_traj: int, n_epochs: int, seed: int, n_sat: int = 24, speed=(5.0, 15.0),
               dt: float = 1.0, sigma_pr: float = 3.0, nlos_mean: float = 20.0, clk0: float = 3000.0,
               clk_drift: float = 0.5, lla=S.ANCHOR_LLA, sat_range=None) -> list:
    """n_traj receivers drive along the street grid of one city (turning at
    random at intersections), each with its own GPS-like constellation:
    azimuth U[0, 2 pi), elevation U[15, 85] deg, azimuth drift 0.008 deg/s.
    sat_range = (lo, hi) draws the number of satellites of every epoch
    uniformly from lo..hi out of a pool of n_sat (all n_sat otherwise).
    The ray tracing of every epoch is one call for all receivers."""
    rng = np.random.default_rng(seed)
    base = S.lla_to_ecef(*lla)
    rot = S.enu_rotation_lla(lla[0], lla[1])
    c = city.cell
    R = n_traj
    g = rng.integers(2, city.n - 2, (R, 2))
    pos = np.column_stack([g[:, 0] * c, g[:, 1] * c, np.full(R, RX_HEIGHT)])
    heading = rng.integers(0, 4, R)  # 0 E, 1 N, 2 W, 3 S
    dirs = np.array([[1.0, 0.0], [0.0, 1.0], [-1.0, 0.0], [0.0, -1.0]])
    v = rng.uniform(speed[0], speed[1], R)
    az0 = rng.uniform(0.0, 2.0 * np.pi, (R, n_sat))
    el_s = np.radians(rng.uniform(15.0, 85.0, (R, n_sat)))
    drift = np.radians(0.008) * dt
    rec = [dict(truth=[], disp=[], sats=[], az=[], el=[], pr=[], cn0=[], nlos=[], bias=[], clk=[]) for _ in range(R)]
    for t in range(n_epochs):
        new = pos.copy()
        new[:, :2] += dirs[heading] * (v * dt)[:, None]
        cross = (np.floor(pos[:, :2] / c) != np.floor(new[:, :2] / c)).any(axis=1)
        out = ~((new[:, 0] >= c) & (new[:, 0] <= city.size - c) & (new[:, 1] >= c) & (new[:, 1] <= city.size - c))
        turn = cross | out
        if turn.any():
            snapped = np.clip(np.round(new[turn, :2] / c) * c, c, city.size - c)
            new[turn, :2] = snapped
            # a new heading other than straight back
            step = rng.integers(1, 4, int(turn.sum()))
            back = (heading[turn] + 2) % 4
            heading[turn] = (back + step) % 4
        d = new - pos
        pos = new
        # satellites of this epoch
        sel = []
        for r in range(R):
            if sat_range is None:
                sel.append(np.arange(n_sat))
            else:
                k = int(rng.integers(sat_range[0], sat_range[1] + 1))
                sel.append(np.sort(rng.choice(n_sat, min(k, n_sat), replace=False)))
        az = [np.mod(az0[r, sel[r]] + drift * (t + 1), 2 * np.pi) for r in range(R)]
        el = [el_s[r, sel[r]] for r in range(R)]
        m = np.array([len(a) for a in az])
        blk_all = los_blocked(city, np.repeat(pos, m, axis=0), np.concatenate(az), np.concatenate(el))
        o = 0
        clk = clk0 + clk_drift * (t + 1)
        for r in range(R):
            blk = blk_all[o:o + m[r]]
            o += m[r]
            p_ecef = base + pos[r] @ rot
            sp = S.sat_positions(p_ecef, rot, az[r], el[r])
            b = np.where(blk, rng.exponential(nlos_mean, m[r]), 0.0)
            pr = np.linalg.norm(sp - p_ecef, axis=1) + clk + rng.normal(0.0, sigma_pr, m[r]) + b
            cn0 = np.where(blk, rng.normal(35.0, 5.0, m[r]), rng.normal(45.0, 4.0, m[r]))
            q = rec[r]
            q["truth"].append(pos[r].copy())
            q["disp"].append(d[r])
            q["sats"].append(sp)
            q["az"].append(az[r])
            q["el"].append(np.array(el[r], copy=True))
            q["pr"].append(pr)
            q["cn0"].append(cn0)
            q["nlos"].append(blk)
            q["bias"].append(b)
            q["clk"].append([clk])
    out = []
    for q in rec:
        te = np.array(q["truth"])
        out.append(CityTrajectory(city, te, base + te @ rot, np.array(q["clk"]), np.array(q["disp"]), q["sats"],
                                  q["az"], q["el"], q["pr"], q["cn0"], q["nlos"], q["bias"], base, rot))
    return out


def drive(city: City, n_epochs: int, seed: int, **kw) -> CityTrajectory:
    """One receiver (drive_many with n_traj = 1)."""
    return drive_many(city, 1, n_epochs, seed, **kw)[0]


def sat_az_el(rot: np.ndarray, p_ecef: np.ndarray, sats: np.ndarray):
    """Azimuth and elevation (radians) of satellites seen from p."""
    u = sats - p_ecef
    u = u / np.linalg.norm(u, axis=1, keepdims=True)
    e = u @ rot.T
    return np.mod(np.arctan2(e[:, 0], e[:, 1]), 2 * np.pi), np.arcsin(np.clip(e[:, 2], -1.0, 1.0))


def city_triangles(city: City, anchor_ecef, rot) -> np.ndarray:
    """The city's buildings as a triangle mesh (T, 3, 3) in ECEF: per
    building four walls and a roof, two triangles each.  anchor_ecef is the
    city origin, rot the ECEF -> local E/N/U rotation."""
    ix, iy = np.nonzero(city.occ)
    x0, x1 = city.box[ix, iy, 0], city.box[ix, iy, 1]
    y0, y1 = city.box[ix, iy, 2], city.box[ix, iy, 3]
    h = city.height[ix, iy]
    z = np.zeros_like(h)
    # corners: 0..3 at the ground, 4..7 at the roof (x0y0, x1y0, x1y1, x0y1)
    cx = np.stack([x0, x1, x1, x0, x0, x1, x1, x0], axis=1)
    cy = np.stack([y0, y0, y1, y1, y0, y0, y1, y1], axis=1)
    cz = np.stack([z, z, z, z, h, h, h, h], axis=1)
    corners = np.stack([cx, cy, cz], axis=-1)                   # (B, 8, 3) local
    faces = np.array([[0, 1, 5], [0, 5, 4], [1, 2, 6], [1, 6, 5], [2, 3, 7], [2, 7, 6], [3, 0, 4], [3, 4, 7],
                      [4, 5, 6], [4, 6, 7]])
    tri_local = corners[:, faces, :].reshape(-1, 3, 3)
    return np.asarray(anchor_ecef, dtype=np.float64) + tri_local @ np.asarray(rot, dtype=np.float64)
