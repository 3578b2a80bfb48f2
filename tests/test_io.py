"""CPU tests of the file formats around the filter: RINEX observation
reading, NMEA reading and NMEA writing, against the reference's own outputs
(tests/golden/io_golden.json, made by make_io_golden.py from the
reference's io/rinex.py, io/nmea.py and io/nmea_writer.py).  No device call."""
from __future__ import annotations

import json
import math
from datetime import date, datetime
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLD = json.loads((ROOT / "tests" / "golden" / "io_golden.json").read_text())


@pytest.mark.parametrize("name", ["v3", "v2"])
def test_rinex_obs_matches_reference(tmp_path, name):
    from gnss_gpu_b200.rinex_obs import read_rinex_obs

    g = GOLD["rinex_obs"][name]
    p = tmp_path / "x.obs"
    p.write_text(g["text"])
    obs = read_rinex_obs(p)
    h = obs.header
    assert (h.version, h.sat_system, h.marker_name, h.interval) == (
        g["header"]["version"], g["header"]["sat_system"], g["header"]["marker_name"], g["header"]["interval"])
    assert h.approx_position.tolist() == g["header"]["approx_position"]
    assert h.obs_types == g["header"]["obs_types"]
    assert len(obs.epochs) == len(g["epochs"])
    for e, r in zip(obs.epochs, g["epochs"]):
        assert e.time.isoformat() == r["time"]
        assert e.satellites == r["satellites"]
        assert e.observations == r["observations"]
    times, pr, sats = obs.pseudoranges("C1C" if name == "v3" else "C1")
    ref = g["pseudoranges"]
    assert [t.isoformat() for t in times] == ref["times"] and sats == ref["sats"]
    want = np.array([[np.nan if v is None else v for v in row] for row in ref["pr"]])
    np.testing.assert_array_equal(pr, want)


def test_rinex_obs_without_the_code_gives_empty(tmp_path):
    from gnss_gpu_b200.rinex_obs import read_rinex_obs

    p = tmp_path / "x.obs"
    p.write_text(GOLD["rinex_obs"]["v3"]["text"])
    times, pr, sats = read_rinex_obs(p).pseudoranges("C7X")
    assert times == [] and pr.size == 0 and sats == []


def test_nmea_parse_matches_reference(tmp_path):
    from gnss_gpu_b200.nmea import parse_nmea

    p = tmp_path / "x.nmea"
    p.write_text(GOLD["nmea"]["text"])
    msgs = parse_nmea(p)
    ref = GOLD["nmea"]["messages"]
    assert [type(m).__name__ for m in msgs] == [r["type"] for r in ref]
    for m, r in zip(msgs, ref):
        for k, v in r.items():
            if k == "type":
                continue
            got = getattr(m, k)
            assert (got.isoformat() if isinstance(got, datetime) else got) == v, k


def test_nmea_writer_matches_reference():
    from gnss_gpu_b200.nmea import NMEAWriter, positions_to_nmea

    g = GOLD["writer"]
    w = NMEAWriter()
    t = datetime(2024, 1, 15, 23, 59, 59, 990000)
    sats = [(1, 45, 120, 42), (5, 12, 300, 35), (12, 78, 15, 48), (17, 5, 200, 28), (24, 33, 95, 40), (30, 60, 250, 44)]
    assert w.gga(51.4778, -0.0014, 46.5, time_utc=t, n_sats=7, hdop=1.3, geoid_sep=45.4) == g["gga"]
    assert NMEAWriter("GN").gga(-22.9068, -43.1729, 9.876, time_utc=t, fix_quality=4, n_sats=15) == g["gga_rtk"]
    assert w.rmc(51.4778, -0.0014, time_utc=t, date_val=date(2024, 1, 15), speed_knots=12.34,
                 course_deg=359.96) == g["rmc"]
    assert w.gsa(list(range(1, 15)), pdop=2.1, hdop=1.1, vdop=1.8) == g["gsa"]
    assert w.gsv(sats) == g["gsv"] and w.gsv([]) == g["gsv_empty"]
    assert w.vtg(course_deg=10.0, speed_knots=5.0, speed_kmh=9.26) == g["vtg"]
    assert w.write_epoch(35.0, 139.0, 10.0, time_utc=t, n_sats=8, prn_list=[3, 7, 9], pdop=1.4, vdop=1.1) == g["epoch"]
    pg = g["positions_to_nmea"]
    text = positions_to_nmea(np.array(pg["lat"]), np.array(pg["lon"]), np.array(pg["alt"]),
                             times=[datetime.fromisoformat(x) for x in pg["times"]])
    assert text == pg["text"]


def test_nmea_round_trip(tmp_path):
    """Writer output parses back to the written values (to the printed precision)."""
    from gnss_gpu_b200.nmea import NMEAWriter, parse_nmea

    w = NMEAWriter()
    t = datetime(2024, 3, 1, 12, 30, 15, 500000)
    p = tmp_path / "rt.nmea"
    p.write_text("\n".join(w.write_epoch(-12.345678, 45.678901, 123.456, time_utc=t, n_sats=11)) + "\n")
    gga, rmc = parse_nmea(p)
    assert math.isclose(gga.latitude, -12.345678, abs_tol=1e-6) and math.isclose(gga.longitude, 45.678901, abs_tol=1e-6)
    assert gga.altitude == 123.456 and gga.n_satellites == 11
    assert rmc.time == datetime(2024, 3, 1, 12, 30, 15, 500000) and rmc.status == "A"
