"""Device parity of the input-formation kernels (pf_sat_positions*,
pf_broadcast_orbits, pf_sagnac) against the reference's own outputs
(tests/golden/orbit_golden.json) and the FP64 oracle (oracle/orbit.py).

Tolerance: FP64 on both sides; the device contracts multiply-adds and uses
its own sin/cos/atan2, so positions agree to 1e-6 m (orbit radius ~2.7e7 m)
and clocks to 1e-15 s; GLONASS after up to 30 RK4 steps to 1e-6 m, and a
GLONASS state integrated over days (thousands of RK4 steps) to 1e-12
relative.
"""
from __future__ import annotations

import json
from datetime import datetime
from pathlib import Path

import numpy as np
import pytest

from oracle import orbit as O

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
GOLD = json.loads((ROOT / "tests" / "golden" / "orbit_golden.json").read_text())


def nav_of(d: dict):
    from gnss_gpu_b200.nav_rinex import NavMessage

    return NavMessage(prn=d["prn"], toc=datetime.fromisoformat(d["toc"]), system=d["system"],
                      **{k: v for k, v in d.items() if k not in ("prn", "toc", "system")})


def test_compute_satellite_position_matches_reference():
    """The reference binding's entry points on the PRN 01 record
    (tests/test_ephemeris.py:515-542 of the reference)."""
    from gnss_gpu_b200 import _gnss_gpu_ephemeris as E
    from gnss_gpu_b200.ephemeris import _pack

    c = GOLD["kepler"][0]
    assert c["nav"]["system"] == "G" and c["apply_group_delay"]
    params = _pack([nav_of(c["nav"])])["kepler"]
    flat = np.frombuffer(params.tobytes(), np.float64)
    for t, p_ref, c_ref in zip(c["times"], c["pos"], c["clk"]):
        pos, clk = E.compute_satellite_position(flat, t, 1)
        assert pos.shape == (1, 3) and clk.shape == (1,)
        np.testing.assert_allclose(pos[0], p_ref, rtol=0, atol=1e-6)
        assert abs(clk[0] - c_ref) <= 1e-15
    pos_b, clk_b = E.compute_satellite_position_batch(flat, c["times"], 1)
    assert pos_b.shape == (len(c["times"]), 1, 3)
    np.testing.assert_allclose(pos_b[:, 0], c["pos"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(clk_b[:, 0], c["clk"], rtol=0, atol=1e-15)
    # batch equals single, element for element
    for k, t in enumerate(c["times"]):
        pos, clk = E.compute_satellite_position(flat, t, 1)
        assert np.array_equal(pos[0], pos_b[k, 0]) and clk[0] == clk_b[k, 0]


def test_broadcast_orbits_every_kepler_case():
    """G/E/J/C constants, BDT offset, Galileo BGD choice, group delay on/off,
    week crossover: every case of the fixture in one launch."""
    from gnss_gpu_b200.ephemeris import _pack, broadcast_orbits

    cases = GOLD["kepler"]
    recs = np.concatenate([_pack([nav_of(c["nav"])], [c["obs_code"]], c["apply_group_delay"]) for c in cases])
    T = max(len(c["times"]) for c in cases)
    # one row of times per (case, time) pair: epoch e = (case, k), column = case
    times, idx = [], []
    for j, c in enumerate(cases):
        for t in c["times"]:
            times.append(t)
            row = np.full(len(cases), -1, np.int32)
            row[j] = j
            idx.append(row)
    pos, clk = broadcast_orbits(recs, times, np.stack(idx))
    e = 0
    for j, c in enumerate(cases):
        for k in range(len(c["times"])):
            np.testing.assert_allclose(pos[e, j], c["pos"][k], rtol=0, atol=1e-6)
            assert abs(clk[e, j] - c["clk"][k]) <= 1e-15, (j, k)
            assert np.isnan(pos[e]).sum() == 3 * (len(cases) - 1)  # index -1 -> NaN
            e += 1
    assert T >= 4


def test_broadcast_orbits_glonass():
    from gnss_gpu_b200.ephemeris import _pack, broadcast_orbits

    for c in GOLD["glonass"]:
        recs = _pack([nav_of(c["nav"])])
        pos, clk = broadcast_orbits(recs, c["times"])
        np.testing.assert_allclose(pos[:, 0], c["pos"], rtol=0, atol=1e-6)
        np.testing.assert_allclose(clk[:, 0], c["clk"], rtol=0, atol=1e-18)


def test_ephemeris_compute_and_batch_match_reference():
    """Ephemeris.compute / compute_batch (ephemeris.py:277-412): selection,
    dropped BeiDou GEO and unknown PRNs, re-selection per epoch."""
    from gnss_gpu_b200 import Ephemeris

    msgs = {}
    for k, recs in GOLD["selection"]["records"].items():
        msgs[int(k) if k.isdigit() else k] = [nav_of(r) for r in recs]
    eph = Ephemeris(msgs)
    c = GOLD["selection"]["compute"]
    pos, clk, used = eph.compute(c["time"], c["prns"], obs_codes=c["obs_codes"])
    assert used == c["used"]
    np.testing.assert_allclose(pos, c["pos"], rtol=1e-12, atol=1e-6)
    np.testing.assert_allclose(clk, c["clk"], rtol=0, atol=1e-15)
    b = GOLD["selection"]["batch"]
    pos, clk, used = eph.compute_batch(b["times"], b["prns"])
    assert used == b["used"]
    np.testing.assert_allclose(pos, b["pos"], rtol=1e-12, atol=1e-6)
    np.testing.assert_allclose(clk, b["clk"], rtol=0, atol=1e-15)
    # empty inputs keep the reference's shapes
    p0, c0, u0 = eph.compute_batch([], b["prns"])
    assert p0.shape == (0, 0, 3) and c0.shape == (0, 0) and u0 == []
    p0, c0, u0 = eph.compute(c["time"], [17])
    assert p0.shape == (0, 3) and u0 == []


def test_compute_single_group_delay_and_invalid():
    """tests/test_ephemeris.py:139-151 of the reference: omitting the group
    delay changes the clock by exactly tgd; an invalid record raises."""
    from gnss_gpu_b200 import Ephemeris
    from gnss_gpu_b200.nav_rinex import NavMessage

    nav = nav_of(GOLD["kepler"][0]["nav"])
    eph = Ephemeris({1: [nav]})
    t = nav.toe + 123.0
    p1, c1 = eph.compute_single(nav, t)
    p2, c2 = eph.compute_single(nav, t, apply_group_delay=False)
    assert np.array_equal(p1, p2)
    assert np.isclose(c2 - c1, nav.tgd)
    with pytest.raises(ValueError):
        eph.compute_single(NavMessage(prn=2, toc=nav.toc, sqrt_a=0.0), t)


def test_broadcast_orbits_large_batch_matches_oracle():
    """600 epochs x 48 records with random per-epoch record choice across
    four Kepler systems, against the oracle record by record."""
    from gnss_gpu_b200 import _native as N
    from gnss_gpu_b200.ephemeris import broadcast_orbits

    rng = np.random.default_rng(3)
    n_rec, n_epoch, n_sat = 48, 600, 32
    recs = np.zeros(n_rec, N.BROADCAST_DTYPE)
    systems = rng.choice([ord("G"), ord("E"), ord("J"), ord("C")], n_rec)
    recs["system"] = systems
    k = recs["kepler"]
    k["sqrt_a"] = rng.uniform(5150.0, 6500.0, n_rec)
    k["e"] = rng.uniform(0.0, 0.02, n_rec)
    for f, lo, hi in (("i0", 0.9, 1.0), ("omega0", -3.1, 3.1), ("omega", -3.1, 3.1), ("M0", -3.1, 3.1),
                      ("delta_n", 3e-9, 5e-9), ("omega_dot", -9e-9, -7e-9), ("idot", -1e-10, 1e-10),
                      ("cuc", -5e-6, 5e-6), ("cus", -5e-6, 5e-6), ("crc", 150.0, 300.0), ("crs", -50.0, 50.0),
                      ("cic", -2e-7, 2e-7), ("cis", -2e-7, 2e-7), ("af0", -1e-4, 1e-4), ("af1", -1e-11, 1e-11),
                      ("tgd", -1e-8, 1e-8)):
        k[f] = rng.uniform(lo, hi, n_rec)
    k["toe"] = rng.choice([0.0, 7200.0, 302400.0, 597600.0], n_rec)
    k["toc"] = k["toe"]
    times = rng.uniform(0.0, 604800.0, n_epoch)
    idx = rng.integers(0, n_rec, (n_epoch, n_sat)).astype(np.int32)
    pos, clk = broadcast_orbits(recs, times, idx)
    worst_p = worst_c = 0.0
    for r in range(n_rec):
        e_, s_ = np.nonzero(idx == r)
        if e_.size == 0:
            continue
        rec = {f: float(k[f][r]) for f in N.EPHEMERIS_FIELDS}
        p_o, c_o = O.kepler(rec, chr(systems[r]), times[e_])
        worst_p = max(worst_p, float(np.abs(pos[e_, s_] - p_o).max()))
        worst_c = max(worst_c, float(np.abs(clk[e_, s_] - c_o).max()))
    assert worst_p <= 1e-6 and worst_c <= 1e-15, (worst_p, worst_c)


def test_sagnac_matches_reference_and_batch():
    from gnss_gpu_b200 import range_model as R

    s = GOLD["sagnac"]
    np.testing.assert_allclose(R.rotate_satellites_sagnac(s["rx"], s["sat"]), s["rot"], rtol=0, atol=1e-7)
    np.testing.assert_allclose(R.geometric_ranges_sagnac(s["rx"], s["sat"]), s["range"], rtol=0, atol=1e-7)
    rng = np.random.default_rng(1)
    rx = np.asarray(s["rx"]) + rng.normal(0, 1000.0, (50, 3))
    sat = rng.normal(0, 1.5e7, (50, 12, 3))
    rot, dist = R.sagnac_batch(rx, sat)
    for e in range(0, 50, 7):
        r_o, d_o = O.sagnac(rx[e], sat[e])
        np.testing.assert_allclose(rot[e], r_o, rtol=0, atol=1e-7)
        np.testing.assert_allclose(dist[e], d_o, rtol=0, atol=1e-7)
    r0, d0 = R.sagnac_batch(np.zeros((0, 3)), np.zeros((0, 4, 3)))
    assert r0.shape == (0, 4, 3) and d0.shape == (0, 4)


def _glonass_records(n, rng):
    from gnss_gpu_b200 import _native as N

    recs = np.zeros(n, N.BROADCAST_DTYPE)
    recs["system"] = ord("R")
    g = recs["glonass"]
    for r in range(n):
        ang = rng.uniform(0, 2 * np.pi)
        inc = rng.uniform(1.0, 1.2)
        rad = rng.uniform(2.54e7, 2.56e7)
        v = np.sqrt(3.9860044e14 / rad)
        g["toe"][r] = rng.choice([900.0, 302400.0, 603900.0])
        pos = np.array([rad * np.cos(ang), rad * np.sin(ang), 0.0])
        v_in = np.array([-v * np.sin(ang) * np.cos(inc), v * np.cos(ang) * np.cos(inc), v * np.sin(inc)])
        g["pos"][r] = pos
        g["vel"][r] = v_in - np.cross([0.0, 0.0, 7.292115e-5], pos)  # earth-fixed velocity of a circular orbit
        g["acc"][r] = rng.normal(0, 2e-6, 3)
        g["tau_n"][r], g["gamma_n"][r] = rng.normal(0, 1e-5), rng.normal(0, 1e-12)
    return recs


def test_glonass_batch_matches_oracle():
    """GLONASS states integrated from toe over up to +-2 h (more steps than the
    device's state table holds, so walks continue past it), week crossover
    included, against the oracle's RK4 walk from toe."""
    from gnss_gpu_b200.ephemeris import broadcast_orbits

    rng = np.random.default_rng(17)
    recs = _glonass_records(6, rng)
    n_epoch = 120
    times = np.empty(n_epoch)
    idx = np.empty((n_epoch, 6), np.int32)
    for e in range(n_epoch):
        times[e] = (recs["glonass"]["toe"][e % 6] + 18.0 + rng.uniform(-7200.0, 7200.0)) % 604800.0
        idx[e] = (np.arange(6) + e) % 6
    pos, clk = broadcast_orbits(recs, times, idx)
    g = recs["glonass"]
    for e in range(0, n_epoch, 3):
        for s in range(6):
            r = idx[e, s]
            st = {"toe": float(g["toe"][r]), "pos": g["pos"][r], "vel": g["vel"][r], "acc": g["acc"][r],
                  "tau_n": float(g["tau_n"][r]), "gamma_n": float(g["gamma_n"][r])}
            p_o, c_o = O.glonass(st, float(times[e]))
            # FP64 on both sides, the device contracting multiply-adds: up to
            # 120 RK4 steps agree to 1e-12 of the orbit radius
            assert np.abs(pos[e, s] - p_o).max() <= 1e-6 + 1e-12 * np.linalg.norm(p_o)
            assert abs(clk[e, s] - c_o) <= 1e-15


def test_glonass_state_table_equals_walk_from_toe():
    """The shared state table changes nothing: with a record table too large
    for it (the kernel then walks every epoch from toe) the positions are
    the same bit for bit."""
    from gnss_gpu_b200 import _native as N
    from gnss_gpu_b200.ephemeris import broadcast_orbits

    rng = np.random.default_rng(23)
    recs = _glonass_records(8, rng)
    times = (recs["glonass"]["toe"][0] + 18.0 + np.linspace(-5000.0, 5000.0, 257)) % 604800.0
    idx = np.tile(np.arange(8, dtype=np.int32), (times.size, 1))
    pos_a, clk_a = broadcast_orbits(recs, times, idx)
    big = np.zeros(200_000, N.BROADCAST_DTYPE)  # 200K records: no room for the state table
    big[:8] = recs
    big["system"][8:] = ord("G")
    pos_b, clk_b = broadcast_orbits(big, times, idx)
    assert np.array_equal(pos_a, pos_b) and np.array_equal(clk_a, clk_b)
