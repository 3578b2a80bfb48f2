"""Generate tests/golden/orbit_golden.json from the reference's own CPU code:
broadcast-ephemeris positions/clocks (Ephemeris._compute_single_cpu, the
reference's multi-system path), GLONASS propagation (orbit_glonass), the
Sagnac range model (range_model), Ephemeris.compute / compute_batch record
selection, and RINEX 2/3 navigation parsing (io/nav_rinex).

Run in a container that has the reference checkout:

    python tests/golden/make_orbit_golden.py /path/to/reference

The GPS record is the reference test-suite's PRN 01 record
(tests/test_ephemeris.py:32-57, loaded from that file); the Galileo, QZSS
and BeiDou records reuse its orbit under their systems' constants; the RINEX
files are written here from these records in the RINEX 2.11 / 3.04 column
layout.
"""
from __future__ import annotations

import dataclasses
import importlib.util
import json
import math
import os
import sys
import tempfile
from datetime import datetime
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent / "orbit_golden.json"

KEPLER_FIELDS = ("sqrt_a", "e", "i0", "omega0", "omega", "M0", "delta_n", "omega_dot", "idot", "cuc", "cus",
                 "crc", "crs", "cic", "cis", "toe", "af0", "af1", "af2", "toc_seconds", "tgd", "week",
                 "data_sources", "bgd_e5a_e1", "bgd_e5b_e1", "prn", "system")
GLO_FIELDS = ("toe", "glo_px_m", "glo_py_m", "glo_pz_m", "glo_vx_m_s", "glo_vy_m_s", "glo_vz_m_s",
              "glo_ax_m_s2", "glo_ay_m_s2", "glo_az_m_s2", "glo_tau_n", "glo_gamma_n", "prn", "system")
NAV_FIELDS = ("prn", "system", "af0", "af1", "af2", "sqrt_a", "e", "i0", "omega0", "omega", "M0", "delta_n",
              "omega_dot", "idot", "cuc", "cus", "crc", "crs", "cic", "cis", "toe", "week", "tgd",
              "data_sources", "bgd_e5a_e1", "bgd_e5b_e1", "iode", "iodc", "codes_on_l2", "l2_p_flag",
              "sv_accuracy", "sv_health", "fit_interval", "toc_seconds", "glo_px_m", "glo_py_m", "glo_pz_m",
              "glo_vx_m_s", "glo_vy_m_s", "glo_vz_m_s", "glo_ax_m_s2", "glo_ay_m_s2", "glo_az_m_s2",
              "glo_tau_n", "glo_gamma_n", "glo_frequency_channel")


def _fmt(v: float, exp_char: str = "E") -> str:
    """One 19-column RINEX number, e.g. -3.930553793907E-05."""
    s = f"{v: .12E}"
    mant, ex = s.split("E")
    return f"{mant}{exp_char}{int(ex):+03d}".rjust(19)


def _v3_kepler(nav) -> list[str]:
    t = nav.toc
    head = f"{nav.system}{nav.prn:02d} {t.year:04d} {t.month:02d} {t.day:02d} {t.hour:02d} {t.minute:02d} {t.second:02d}"
    orbit = [nav.iode, nav.crs, nav.delta_n, nav.M0, nav.cuc, nav.e, nav.cus, nav.sqrt_a,
             nav.toe, nav.cic, nav.omega0, nav.cis, nav.i0, nav.crc, nav.omega, nav.omega_dot,
             nav.idot, nav.data_sources if nav.system == "E" else nav.codes_on_l2, float(nav.week), 0.0,
             nav.sv_accuracy, nav.sv_health, nav.bgd_e5a_e1 if nav.system == "E" else nav.tgd,
             nav.bgd_e5b_e1 if nav.system == "E" else nav.iodc, nav.toe, 4.0, 0.0, 0.0]
    lines = [head + "".join(_fmt(v) for v in (nav.af0, nav.af1, nav.af2))]
    for r in range(7):
        lines.append("    " + "".join(_fmt(v) for v in orbit[4 * r:4 * r + 4]))
    return lines


def _v3_glonass(nav) -> list[str]:
    t = nav.toc
    head = f"R{nav.prn:02d} {t.year:04d} {t.month:02d} {t.day:02d} {t.hour:02d} {t.minute:02d} {t.second:02d}"
    k = 1.0e-3
    rows = [(nav.glo_px_m * k, nav.glo_vx_m_s * k, nav.glo_ax_m_s2 * k, 0.0),
            (nav.glo_py_m * k, nav.glo_vy_m_s * k, nav.glo_ay_m_s2 * k, float(nav.glo_frequency_channel)),
            (nav.glo_pz_m * k, nav.glo_vz_m_s * k, nav.glo_az_m_s2 * k, 0.0)]
    lines = [head + "".join(_fmt(v, "e") for v in (-nav.glo_tau_n, nav.glo_gamma_n, 0.0))]
    for row in rows:
        lines.append("    " + "".join(_fmt(v, "e") for v in row))
    return lines


def _v2_kepler(nav) -> list[str]:
    t = nav.toc
    head = (f"{nav.prn:2d} {t.year % 100:02d} {t.month:2d} {t.day:2d} {t.hour:2d} {t.minute:2d}"
            f"{t.second:5.1f}")
    orbit = [nav.iode, nav.crs, nav.delta_n, nav.M0, nav.cuc, nav.e, nav.cus, nav.sqrt_a,
             nav.toe, nav.cic, nav.omega0, nav.cis, nav.i0, nav.crc, nav.omega, nav.omega_dot,
             nav.idot, nav.codes_on_l2, float(nav.week), 0.0, nav.sv_accuracy, nav.sv_health, nav.tgd,
             nav.iodc, nav.toe, 4.0, 0.0, 0.0]
    lines = [head + "".join(_fmt(v, "D") for v in (nav.af0, nav.af1, nav.af2))]
    for r in range(7):
        lines.append("   " + "".join(_fmt(v, "D") for v in orbit[4 * r:4 * r + 4]))
    return lines


def _dump(nav, fields):
    out = {}
    for f in fields:
        v = getattr(nav, f)
        out[f] = v if isinstance(v, (str, int)) and not isinstance(v, bool) else float(v)
    out["toc"] = nav.toc.isoformat()
    return out


def main(ref_root: str) -> None:
    ref = Path(ref_root)
    sys.path.insert(0, str(ref / "python"))
    from gnss_gpu import range_model
    from gnss_gpu.ephemeris import Ephemeris
    from gnss_gpu.io.nav_rinex import read_nav_rinex
    from gnss_gpu.orbit_glonass import GlonassBroadcastState, glonass_position_clock
    from gnss_gpu.io.nav_rinex import NavMessage

    spec = importlib.util.spec_from_file_location("ref_test_ephemeris", ref / "tests" / "test_ephemeris.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    gps = mod._make_reference_nav()

    gal = dataclasses.replace(gps, system="E", prn=11, data_sources=517.0, bgd_e5a_e1=-2.3283064365e-09,
                              bgd_e5b_e1=-2.7939677238e-09, tgd=-2.3283064365e-09)
    qzs = dataclasses.replace(gps, system="J", prn=2)
    bds = dataclasses.replace(gps, system="C", prn=23, toe=518400.0 - 14.0, toc_seconds=518400.0 - 14.0)
    # a record at the week start, evaluated across the week crossover
    wk = dataclasses.replace(gps, prn=7, toe=0.0, toc_seconds=0.0, M0=-2.1, omega0=1.3)

    kepler_cases = []
    t0 = gps.toe
    times = [t0, t0 + 300.0, t0 - 7200.0, t0 + 3600.5, t0 + 14400.0]
    for nav, codes in ((gps, [None]), (gal, [None, "C1C", "C5Q", "C7Q"]), (qzs, [None]), (bds, [None])):
        for code in codes:
            for gd in (True, False):
                pos, clk = zip(*[Ephemeris._compute_single_cpu(nav, t, code, apply_group_delay=gd) for t in times])
                kepler_cases.append({"nav": _dump(nav, KEPLER_FIELDS), "obs_code": code, "apply_group_delay": gd,
                                     "times": times, "pos": [list(map(float, p)) for p in pos],
                                     "clk": [float(c) for c in clk]})
    wt = [604500.0, 604799.5, 100.0, 3600.0]
    for nav in (wk, dataclasses.replace(wk, system="C", prn=24)):
        pos, clk = zip(*[Ephemeris._compute_single_cpu(nav, t) for t in wt])
        kepler_cases.append({"nav": _dump(nav, KEPLER_FIELDS), "obs_code": None, "apply_group_delay": True,
                             "times": wt, "pos": [list(map(float, p)) for p in pos],
                             "clk": [float(c) for c in clk]})

    glo_navs = [
        NavMessage(prn=1, toc=datetime(2026, 5, 20, 0, 15, 0), system="R", toe=259200.0 + 900.0,
                   glo_px_m=2.55e7, glo_vy_m_s=math.sqrt(3.9860044e14 / 2.55e7), glo_tau_n=1.0e-6),
        NavMessage(prn=9, toc=datetime(2026, 5, 20, 0, 45, 0), system="R", toe=259200.0 + 2700.0,
                   glo_px_m=-1.4612e7, glo_py_m=1.1384e7, glo_pz_m=1.7962e7,
                   glo_vx_m_s=-1185.3, glo_vy_m_s=-2696.7, glo_vz_m_s=748.1,
                   glo_ax_m_s2=1.86e-6, glo_ay_m_s2=-2.79e-6, glo_az_m_s2=-9.31e-7,
                   glo_tau_n=-3.41e-5, glo_gamma_n=9.1e-13, glo_frequency_channel=-2),
    ]
    glo_cases = []
    for nav in glo_navs:
        t_gps = nav.toe + 18.0
        ts = [t_gps, t_gps + 60.0, t_gps + 900.5, t_gps - 450.0, t_gps - 1800.0, t_gps + 1.0e-10]
        st = GlonassBroadcastState(toe=nav.toe, px_m=nav.glo_px_m, py_m=nav.glo_py_m, pz_m=nav.glo_pz_m,
                                   vx_m_s=nav.glo_vx_m_s, vy_m_s=nav.glo_vy_m_s, vz_m_s=nav.glo_vz_m_s,
                                   ax_m_s2=nav.glo_ax_m_s2, ay_m_s2=nav.glo_ay_m_s2, az_m_s2=nav.glo_az_m_s2,
                                   tau_n=nav.glo_tau_n, gamma_n=nav.glo_gamma_n)
        pos, clk = zip(*[glonass_position_clock(st, t) for t in ts])
        pos2, clk2 = zip(*[Ephemeris._compute_single_cpu(nav, t) for t in ts])
        assert np.array_equal(np.array(pos), np.array(pos2))
        glo_cases.append({"nav": _dump(nav, GLO_FIELDS), "times": ts, "pos": [list(map(float, p)) for p in pos],
                          "clk": [float(c) for c in clk]})

    rx = [-3957199.0, 3310205.0, 3737911.0]
    sats = [c["pos"][1] for c in kepler_cases[:1]] + [glo_cases[1]["pos"][2], [15600e3, 7540e3, 20140e3],
                                                    [-2.1e7, 1.2e7, 9.0e6]]
    sag = {"rx": rx, "sat": sats, "rot": range_model.rotate_satellites_sagnac(np.array(rx), np.array(sats)).tolist(),
           "range": range_model.geometric_ranges_sagnac(np.array(rx), np.array(sats)).tolist()}

    # Ephemeris.compute / compute_batch: several records per satellite, re-selection over time
    msgs = {}
    for k, nav in enumerate((gps, dataclasses.replace(gps, prn=5, M0=2.2, omega0=0.9))):
        msgs[nav.prn] = [dataclasses.replace(nav, toe=nav.toe + 7200.0 * j, toc_seconds=nav.toe + 7200.0 * j,
                                             M0=nav.M0 + 0.01 * j, af0=nav.af0 + 1e-7 * j) for j in range(3)]
    msgs["E11"] = [gal, dataclasses.replace(gal, data_sources=258.0, M0=gal.M0 + 0.02)]
    msgs["C23"] = [bds]
    msgs["C03"] = [dataclasses.replace(bds, prn=3)]   # BeiDou GEO: not usable
    msgs["R09"] = [glo_navs[1]]
    eph = Ephemeris(msgs)
    prns = [1, 5, "E11", "C23", "C03", "R09", 17]
    tq = t0 + 4000.0
    cpos, cclk, cused = eph.compute(tq, prns, obs_codes=["C1C", "C1C", "C1C", "C2I", "C2I", "C1C", "C1C"])
    bt = [t0 + 100.0, t0 + 5000.0, t0 + 11000.0]
    bprns = [1, 5, "E11", "C23", "C03", "R09", 17]
    bpos, bclk, bused = eph.compute_batch(np.array(bt), bprns)
    sel_b = [[eph.select_ephemeris(p, t) for p in bused] for t in bt]
    selection = {
        "records": {str(k): [(_dump(n, GLO_FIELDS) if n.system == "R" else _dump(n, KEPLER_FIELDS)) for n in v]
                    for k, v in msgs.items()},
        "compute": {"time": tq, "prns": prns, "obs_codes": ["C1C", "C1C", "C1C", "C2I", "C2I", "C1C", "C1C"],
                    "pos": np.asarray(cpos).tolist(), "clk": np.asarray(cclk).tolist(), "used": cused},
        "batch": {"times": bt, "prns": bprns, "pos": np.asarray(bpos).tolist(), "clk": np.asarray(bclk).tolist(),
                  "used": bused,
                  "selected_toe": [[float(n.toe) for n in row] for row in sel_b]},
    }

    # RINEX 3 mixed and RINEX 2 GPS navigation files
    v3 = ["     3.04           N: GNSS NAV DATA    M: MIXED            RINEX VERSION / TYPE",
          "golden              golden              20240115 000000 UTC PGM / RUN BY / DATE",
          "                                                            END OF HEADER"]
    gps_v = dataclasses.replace(gps, iode=78.0, iodc=78.0, codes_on_l2=1.0, sv_accuracy=2.0)
    for nav in (gps_v, dataclasses.replace(gps_v, prn=5, toc=datetime(2024, 1, 15, 2, 0, 0), toe=525600.0),
                dataclasses.replace(gal, toc=datetime(2024, 1, 15, 0, 0, 0)),
                dataclasses.replace(bds, toc=datetime(2024, 1, 14, 23, 59, 46))):
        v3 += _v3_kepler(nav)
    v3 += _v3_glonass(dataclasses.replace(glo_navs[1], glo_frequency_channel=-2))
    v3 += ["S20 2024 01 15 00 00 00 0.000000000000E+00 0.000000000000E+00 5.184000000000E+05"] + [
        "     4.000000000000E+04 0.000000000000E+00 0.000000000000E+00 6.300000000000E+01"] * 3
    v2 = ["     2.11           N: GPS NAV DATA                         RINEX VERSION / TYPE",
          "                                                            END OF HEADER"]
    v2 += _v2_kepler(gps_v) + _v2_kepler(dataclasses.replace(gps_v, prn=12, toc=datetime(2024, 1, 15, 2, 0, 0),
                                                             toe=525600.0, M0=-1.0))
    rinex = {}
    with tempfile.TemporaryDirectory() as d:
        for name, text, kw in (("v3_mixed", v3, {"systems": ("G", "E", "C", "R"), "key_by_sat_id": True}),
                               ("v3_gps_only", v3, {}),
                               ("v2", v2, {})):
            p = Path(d) / f"{name}.rnx"
            p.write_text("\n".join(text) + "\n")
            parsed = read_nav_rinex(p, **kw)
            rinex[name] = {"text": "\n".join(text) + "\n", "kwargs": {k: list(v) if isinstance(v, tuple) else v
                                                                        for k, v in kw.items()},
                           "parsed": {str(k): [_dump(n, NAV_FIELDS) for n in v] for k, v in parsed.items()}}

    OUT.write_text(json.dumps({"kepler": kepler_cases, "glonass": glo_cases, "sagnac": sag,
                               "selection": selection, "rinex": rinex}, indent=1))
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["GNSS_GPU_REFERENCE"])
