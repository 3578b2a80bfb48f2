"""CPU tests of the input-formation layer: the FP64 orbit oracle against the
reference's own outputs (tests/golden/orbit_golden.json, made by
make_orbit_golden.py from the reference's CPU path), the RINEX reader and
the record-selection host logic against the same fixture, and the C layout
of the broadcast records.  No device call."""
from __future__ import annotations

import json
import subprocess
from datetime import datetime
from pathlib import Path

import numpy as np
import pytest

from oracle import orbit as O

ROOT = Path(__file__).resolve().parents[1]
GOLD = json.loads((ROOT / "tests" / "golden" / "orbit_golden.json").read_text())


def kepler_rec(nav: dict, obs_code, apply_gd: bool) -> dict:
    """Record fields the oracle reads, with the group delay the reference's
    _group_delay picks for obs_code."""
    from gnss_gpu_b200.ephemeris import _group_delay
    from gnss_gpu_b200.nav_rinex import NavMessage

    m = NavMessage(prn=nav["prn"], toc=datetime.fromisoformat(nav["toc"]), system=nav["system"],
                   **{k: nav[k] for k in nav if k not in ("prn", "toc", "system")})
    rec = {k: nav[k] for k in ("sqrt_a", "e", "i0", "omega0", "omega", "M0", "delta_n", "omega_dot", "idot",
                                "cuc", "cus", "crc", "crs", "cic", "cis", "toe", "af0", "af1", "af2")}
    rec["toc"] = nav["toc_seconds"]
    rec["tgd"] = _group_delay(m, obs_code) if apply_gd else 0.0
    return rec


@pytest.mark.parametrize("case", range(len(GOLD["kepler"])))
def test_oracle_kepler_matches_reference(case):
    c = GOLD["kepler"][case]
    pos, clk = O.kepler(kepler_rec(c["nav"], c["obs_code"], c["apply_group_delay"]), c["nav"]["system"],
                        c["times"])
    np.testing.assert_allclose(pos, c["pos"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(clk, c["clk"], rtol=0, atol=1e-15)


@pytest.mark.parametrize("case", range(len(GOLD["glonass"])))
def test_oracle_glonass_matches_reference(case):
    c = GOLD["glonass"][case]
    n = c["nav"]
    st = {"toe": n["toe"], "pos": (n["glo_px_m"], n["glo_py_m"], n["glo_pz_m"]),
          "vel": (n["glo_vx_m_s"], n["glo_vy_m_s"], n["glo_vz_m_s"]),
          "acc": (n["glo_ax_m_s2"], n["glo_ay_m_s2"], n["glo_az_m_s2"]),
          "tau_n": n["glo_tau_n"], "gamma_n": n["glo_gamma_n"]}
    for t, p_ref, c_ref in zip(c["times"], c["pos"], c["clk"]):
        p, ck = O.glonass(st, t)
        np.testing.assert_allclose(p, p_ref, rtol=0, atol=1e-6)
        assert abs(ck - c_ref) <= 1e-18


def test_oracle_sagnac_matches_reference():
    s = GOLD["sagnac"]
    rot, rng = O.sagnac(s["rx"], s["sat"])
    np.testing.assert_allclose(rot, s["rot"], rtol=0, atol=1e-7)
    np.testing.assert_allclose(rng, s["range"], rtol=0, atol=1e-7)


def test_oracle_known_answers():
    """Orbit radius and clock at toc (reference tests/test_ephemeris.py:113-243)."""
    c = GOLD["kepler"][0]
    rec = kepler_rec(c["nav"], None, True)
    pos, clk = O.kepler(rec, "G", [rec["toe"], rec["toe"] + 300.0])
    r = np.linalg.norm(pos, axis=1)
    a = rec["sqrt_a"] ** 2
    assert np.all(np.abs(r - a) < rec["e"] * a * 1.5)
    assert abs(clk[0] - (rec["af0"] - rec["tgd"])) < 1e-6
    assert 100e3 < np.linalg.norm(pos[1] - pos[0]) < 5000e3


@pytest.mark.parametrize("name", ["v3_mixed", "v3_gps_only", "v2"])
def test_rinex_reader_matches_reference(tmp_path, name):
    from gnss_gpu_b200.nav_rinex import read_nav_rinex

    g = GOLD["rinex"][name]
    p = tmp_path / "nav.rnx"
    p.write_text(g["text"])
    kw = {k: tuple(v) if isinstance(v, list) else v for k, v in g["kwargs"].items()}
    out = read_nav_rinex(p, **kw)
    assert sorted(map(str, out)) == sorted(g["parsed"])
    for key, recs in out.items():
        ref = g["parsed"][str(key)]
        assert len(recs) == len(ref)
        for m, r in zip(recs, ref):
            assert m.toc.isoformat() == r["toc"]
            for f, v in r.items():
                if f == "toc":
                    continue
                assert getattr(m, f) == v, (key, f)


def test_rinex_reader_skips_truncated_and_blank(tmp_path):
    from gnss_gpu_b200.nav_rinex import read_nav_rinex

    text = GOLD["rinex"]["v3_gps_only"]["text"].splitlines()
    head = text[:3]
    rec = text[3:11]
    p = tmp_path / "t.rnx"
    p.write_text("\n".join(head + [""] + rec + rec[:5]) + "\n")
    out = read_nav_rinex(p)
    assert list(out) == [1] and len(out[1]) == 1
    p.write_text("\n".join(head) + "\n")
    assert read_nav_rinex(p) == {}


def _gold_messages():
    from gnss_gpu_b200.nav_rinex import NavMessage

    msgs = {}
    for k, recs in GOLD["selection"]["records"].items():
        key = int(k) if k.isdigit() else k
        msgs[key] = [NavMessage(prn=r["prn"], toc=datetime.fromisoformat(r["toc"]), system=r["system"],
                                **{f: v for f, v in r.items() if f not in ("prn", "toc", "system", "toe")},
                                toe=r["toe"]) for r in recs]
    return msgs


def test_select_ephemeris_matches_reference():
    from gnss_gpu_b200 import Ephemeris

    eph = Ephemeris(_gold_messages())
    b = GOLD["selection"]["batch"]
    for t, toes in zip(b["times"], b["selected_toe"]):
        assert [eph.select_ephemeris(p, t).toe for p in b["used"]] == toes
    assert eph.select_ephemeris(17, b["times"][0]) is None
    # ids are normalised ("e 11" -> "E11"); an int falls back to "Gnn", never the reverse
    assert eph.select_ephemeris("e 11", b["times"][0]) is eph.select_ephemeris("E11", b["times"][0])
    assert eph.select_ephemeris("g 1", b["times"][0]) is None
    # Galileo E1: the I/NAV message (data sources bit 0) wins a tie on toe
    e1 = eph.select_ephemeris("E11", b["times"][0], "C1C")
    assert int(e1.data_sources) & 0x001
    e5a = eph.select_ephemeris("E11", b["times"][0], "C5Q")
    assert int(e5a.data_sources) & 0x002 or int(e5a.data_sources) & 0x100


def test_validity_predicates():
    from gnss_gpu_b200.ephemeris import is_beidou_geo, is_broadcast_usable, is_kepler_broadcast_valid
    from gnss_gpu_b200.nav_rinex import NavMessage

    t = datetime(2024, 1, 15)
    assert not is_broadcast_usable(None)
    assert is_broadcast_usable(NavMessage(prn=1, toc=t, sqrt_a=5153.6, e=0.01))
    assert not is_kepler_broadcast_valid(NavMessage(prn=1, toc=t, sqrt_a=0.0, e=0.01))
    assert not is_kepler_broadcast_valid(NavMessage(prn=1, toc=t, sqrt_a=5153.6, e=1.0))
    assert not is_kepler_broadcast_valid(NavMessage(prn=1, toc=t, sqrt_a=float("nan"), e=0.0))
    assert is_beidou_geo(NavMessage(prn=3, toc=t, system="C", sqrt_a=6493.0, e=0.0))
    assert not is_broadcast_usable(NavMessage(prn=3, toc=t, system="C", sqrt_a=6493.0, e=0.0))
    assert is_broadcast_usable(NavMessage(prn=9, toc=t, system="R", glo_px_m=2.55e7))
    assert not is_broadcast_usable(NavMessage(prn=9, toc=t, system="R", glo_px_m=1.0e6))


def test_broadcast_record_layout_matches_header(tmp_path):
    """sizeof / offsetof of the C records equal the numpy dtypes the Python
    side packs."""
    from gnss_gpu_b200 import _native as N

    src = tmp_path / "l.c"
    src.write_text(f'#include <stdio.h>\n#include <stddef.h>\n#include "{ROOT}/include/gnss_pf_b200.h"\n'
                   "int main(void){printf(\"%zu %zu %zu %zu %zu %zu\\n\", sizeof(pf_ephemeris_t),"
                   " sizeof(pf_glonass_state_t), sizeof(pf_broadcast_t), offsetof(pf_broadcast_t, u),"
                   " offsetof(pf_ephemeris_t, tgd), offsetof(pf_ephemeris_t, week));return 0;}\n")
    exe = tmp_path / "l"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    vals = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()))
    E, B = N.EPHEMERIS_DTYPE, N.BROADCAST_DTYPE
    assert vals == [E.itemsize, N.GLONASS_DTYPE.itemsize, B.itemsize, B.fields["kepler"][1],
                    E.fields["tgd"][1], E.fields["week"][1]]
    assert vals[:3] == [176, 96, 184]


def test_params_too_small_raises_like_the_binding():
    from gnss_gpu_b200 import _gnss_gpu_ephemeris as E

    assert E.EPHEMERIS_PARAMS_SIZE == 176 and E.EPHEMERIS_PARAMS_N_DOUBLES == 21
    with pytest.raises(RuntimeError, match="too small"):
        E.compute_satellite_position(np.zeros(21), 0.0, 1)
    p = E.EphemerisParams()
    p.sqrt_a = 5153.6
    p.week = 2295
    raw = np.frombuffer(p.tobytes(), np.float64)
    assert raw.size == 22 and raw[0] == 5153.6
