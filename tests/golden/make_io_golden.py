"""Generate tests/golden/io_golden.json from the reference's own I/O code:
RINEX 2/3 observation parsing (io/rinex.py), NMEA parsing (io/nmea.py) and
the NMEA writer (io/nmea_writer.py, ecef_to_nmea through its pure-Python
ECEF -> geodetic conversion).

Run in a container that has the reference checkout:

    python tests/golden/make_io_golden.py /path/to/reference

The RINEX and NMEA files are written here, in the RINEX 2.11 / 3.04 and NMEA
0183 layouts, with the cases the parsers handle: multi-line observation-type
headers, wrapped satellite lists and observation records, blank fields,
event records, bad checksums, empty NMEA fields and both hemispheres.
"""
from __future__ import annotations

import json
import os
import sys
import tempfile
from datetime import date, datetime
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent / "io_golden.json"


def _hdr(text: str, label: str) -> str:
    return text.ljust(60)[:60] + label


def _obs(v) -> str:
    """One 16-column observation field (14-column value, LLI, strength)."""
    return " " * 16 if v is None else f"{v:14.3f}  "


def rinex3_text() -> str:
    g_codes = ["C1C", "L1C", "D1C", "S1C", "C2W", "L2W", "D2W", "S2W", "C5Q", "L5Q", "D5Q", "S5Q", "C1W", "L1W"]
    e_codes = ["C1C", "L1C", "C5Q", "S5Q"]
    lines = [_hdr("     3.04           OBSERVATION DATA    M: MIXED", "RINEX VERSION / TYPE"),
             _hdr("GOLDEN", "MARKER NAME"),
             _hdr("  -3957199.5000  3310205.2500  3737911.7500", "APPROX POSITION XYZ"),
             _hdr(f"G  {len(g_codes):3d}" + "".join(f" {c}" for c in g_codes[:13]), "SYS / # / OBS TYPES"),
             _hdr("      " + "".join(f" {c}" for c in g_codes[13:]), "SYS / # / OBS TYPES"),
             _hdr(f"E  {len(e_codes):3d}" + "".join(f" {c}" for c in e_codes), "SYS / # / OBS TYPES"),
             _hdr("     1.000", "INTERVAL"),
             _hdr("", "END OF HEADER")]
    rng = np.random.default_rng(4)

    def row(sat, codes, blanks=()):
        vals = [None if k in blanks else float(np.round(rng.uniform(2.0e7, 2.6e7), 3)) for k in range(len(codes))]
        return sat + "".join(_obs(v) for v in vals)

    lines.append("> 2024 01 15 00 00  0.0000000  0  4")
    lines.append(row("G01", g_codes))
    lines.append(row("G05", g_codes, blanks=(0, 5)))
    lines.append(row("E11", e_codes))
    full = row("G12", g_codes)
    lines.append(full[:3 + 16 * 5])          # wrapped record: continuation lines hold the rest
    lines.append("   " + full[3 + 16 * 5:3 + 16 * 10])
    lines.append("   " + full[3 + 16 * 10:])
    lines.append("> 2024 01 15 00 00  1.5000000  4  2")  # event record: two special lines skipped
    lines.append("  COMMENT LINE ONE")
    lines.append("  COMMENT LINE TWO")
    lines.append("> 2024 01 15 00 00  2.2500000  0  2")
    lines.append(row("G01", g_codes, blanks=(0,)))
    lines.append(row("E11", e_codes, blanks=(2,)))
    lines.append("> 2024 01 15 00 00  3.0000000  0  1")
    lines.append(row("G07", g_codes)[:3 + 16 * 3])  # short record, no continuation follows
    return "\n".join(lines) + "\n"


def rinex2_text() -> str:
    codes = ["C1", "L1", "D1", "S1", "P2", "L2", "S2"]
    lines = [_hdr("     2.11           OBSERVATION DATA    G (GPS)", "RINEX VERSION / TYPE"),
             _hdr("CORS", "MARKER NAME"),
             _hdr("  -2430697.6990 -4704189.5110  3544329.3860", "APPROX POSITION XYZ"),
             _hdr(f"{len(codes):6d}" + "".join(f"{c:>6s}" for c in codes), "# / TYPES OF OBSERV"),
             _hdr("    30.000", "INTERVAL"),
             _hdr("", "END OF HEADER")]
    rng = np.random.default_rng(5)

    def sat_rows(blank=()):
        vals = [None if k in blank else float(np.round(rng.uniform(2.0e7, 2.6e7), 3)) for k in range(len(codes))]
        cells = [_obs(v) for v in vals]
        return ["".join(cells[:5]).rstrip(), "".join(cells[5:]).rstrip()]

    sats = ["G01", "G02", " 3", "G04", "G05", "G06", "G07", "G08", "G09", "G10", "G11", "G12", "G13", "G14"]
    head = " 24  1 15  0  0  0.0000000  0 14" + "".join(f"{s:>3s}" for s in sats[:12])
    lines.append(head)
    lines.append(" " * 32 + "".join(f"{s:>3s}" for s in sats[12:]))
    for k in range(14):
        lines += sat_rows(blank=(1,) if k == 3 else ())
    lines.append(" 24  1 15  0  1  0.5000000  0  2G01G02")
    lines += sat_rows()
    lines += sat_rows(blank=(0, 4))
    # event record last: the reader takes its special line for satellite ids
    # and skips n_sat * lines-per-satellite lines after it
    lines.append(" 24  1 15  0  1 30.0000000  4  1")
    lines.append("                              COMMENT")
    return "\n".join(lines) + "\n"


def nmea_text(writer) -> str:
    t = datetime(2024, 1, 15, 3, 4, 5, 250000)
    good = [writer.gga(35.6812, 139.7671, 40.123, time_utc=t, n_sats=9, hdop=0.8),
            writer.rmc(35.6812, 139.7671, time_utc=t, speed_knots=3.2, course_deg=87.5),
            writer.gga(-33.8688, -151.2093, 12.5, time_utc=t, fix_quality=4, n_sats=12, hdop=0.6, geoid_sep=22.1),
            writer.rmc(-33.8688, -151.2093, time_utc=t, status="V"),
            writer.gsa([1, 5, 12], pdop=1.5, hdop=0.9, vdop=1.2)]
    bad = good[0][:-2] + ("00" if good[0][-2:] != "00" else "11")
    no_chk = "$GPGGA,030405.00,3540.8720,N,13946.0260,E,1,07,1.2,35.000,M,,M,,"
    empty = "$GPGGA,030406.00,,,,,0,,,,M,,M,,"
    junk = "not a sentence"
    return "\n".join(good[:2] + [bad, no_chk] + good[2:] + [empty, junk, "$GPRMC,123"]) + "\n"


def _val(v):
    if isinstance(v, datetime):
        return v.isoformat()
    if isinstance(v, (np.floating, float)):
        return float(v)
    if isinstance(v, np.ndarray):
        return v.tolist()
    return v


def main(ref_root: str) -> None:
    sys.path.insert(0, str(Path(ref_root) / "python"))
    from gnss_gpu.io.nmea import parse_nmea
    from gnss_gpu.io.nmea_writer import NMEAWriter, _ecef_to_lla_py, ecef_to_nmea, positions_to_nmea
    from gnss_gpu.io.rinex import read_rinex_obs

    out = {"rinex_obs": {}, "nmea": {}, "writer": {}}
    w = NMEAWriter()
    with tempfile.TemporaryDirectory() as d:
        for name, text in (("v3", rinex3_text()), ("v2", rinex2_text())):
            p = Path(d) / f"{name}.obs"
            p.write_text(text)
            obs = read_rinex_obs(p)
            h = obs.header
            times, pr, sats = obs.pseudoranges("C1C" if name == "v3" else "C1")
            out["rinex_obs"][name] = {
                "text": text,
                "header": {"version": h.version, "sat_system": h.sat_system, "marker_name": h.marker_name,
                           "approx_position": h.approx_position.tolist(), "obs_types": h.obs_types,
                           "interval": h.interval},
                "epochs": [{"time": e.time.isoformat(), "satellites": e.satellites,
                            "observations": e.observations} for e in obs.epochs],
                "pseudoranges": {"times": [t.isoformat() for t in times],
                                 "pr": np.where(np.isnan(pr), None, pr).tolist() if pr.size else [],
                                 "sats": sats},
            }
        text = nmea_text(w)
        p = Path(d) / "log.nmea"
        p.write_text(text)
        msgs = parse_nmea(p)
        out["nmea"] = {"text": text, "messages": [{"type": type(m).__name__, **{k: _val(v) for k, v in vars(m).items()}}
                                                 for m in msgs]}
    t = datetime(2024, 1, 15, 23, 59, 59, 990000)
    sats = [(1, 45, 120, 42), (5, 12, 300, 35), (12, 78, 15, 48), (17, 5, 200, 28), (24, 33, 95, 40), (30, 60, 250, 44)]
    out["writer"] = {
        "gga": w.gga(51.4778, -0.0014, 46.5, time_utc=t, n_sats=7, hdop=1.3, geoid_sep=45.4),
        "gga_rtk": NMEAWriter("GN").gga(-22.9068, -43.1729, 9.876, time_utc=t, fix_quality=4, n_sats=15),
        "rmc": w.rmc(51.4778, -0.0014, time_utc=t, date_val=date(2024, 1, 15), speed_knots=12.34, course_deg=359.96),
        "gsa": w.gsa(list(range(1, 15)), pdop=2.1, hdop=1.1, vdop=1.8),
        "gsv": w.gsv(sats),
        "gsv_empty": w.gsv([]),
        "vtg": w.vtg(course_deg=10.0, speed_knots=5.0, speed_kmh=9.26),
        "epoch": w.write_epoch(35.0, 139.0, 10.0, time_utc=t, n_sats=8, prn_list=[3, 7, 9], pdop=1.4, vdop=1.1),
    }
    lat = np.array([35.6812, -33.8688, 0.0])
    lon = np.array([139.7671, -151.2093, 179.99999])
    alt = np.array([40.0, -12.25, 1000.5])
    ts = [datetime(2024, 1, 15, 0, 0, k) for k in range(3)]
    out["writer"]["positions_to_nmea"] = {"lat": lat.tolist(), "lon": lon.tolist(), "alt": alt.tolist(),
                                          "times": [x.isoformat() for x in ts],
                                          "text": positions_to_nmea(lat, lon, alt, times=ts)}
    ecef = np.array([[-3957199.0, 3310205.0, 3737911.0], [-4646123.4, 2553452.1, -3534373.9],
                     [6378137.0, 0.0, 0.0], [0.5, -0.25, 6356752.3]])
    out["writer"]["ecef_to_nmea"] = {"ecef": ecef.tolist(), "times": [datetime(2024, 1, 15, 1, 2, k).isoformat()
                                                                        for k in range(len(ecef))],
                                     "lla": [list(_ecef_to_lla_py(*p)) for p in ecef],
                                     "text": ecef_to_nmea(ecef, times=[datetime(2024, 1, 15, 1, 2, k)
                                                                       for k in range(len(ecef))])}
    OUT.write_text(json.dumps(out, indent=1))
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["GNSS_GPU_REFERENCE"])
