"""Broadcast navigation records and the RINEX 2/3 navigation reader
(python/gnss_gpu/io/nav_rinex.py of the reference): ``NavMessage`` with the
same fields and ``read_nav_rinex`` / ``read_nav_rinex_multi`` with the same
keys, units, sorting and column rules, feeding ``gnss_gpu_b200.Ephemeris``.

The reader is host-side text parsing; the orbit arithmetic it feeds runs on
the device (``pf_broadcast_orbits``).
"""
from __future__ import annotations

from dataclasses import dataclass
from datetime import datetime
from pathlib import Path

GPS_EPOCH = datetime(1980, 1, 6)
WEEK_SEC = 604800.0


@dataclass
class NavMessage:
    """One broadcast record (nav_rinex.py:11-74).  Kepler systems fill the
    orbit and clock fields, GLONASS ("R") the ``glo_*`` state vector."""

    prn: int
    toc: datetime
    system: str = "G"
    af0: float = 0.0
    af1: float = 0.0
    af2: float = 0.0
    sqrt_a: float = 0.0
    e: float = 0.0
    i0: float = 0.0
    omega0: float = 0.0
    omega: float = 0.0
    M0: float = 0.0
    delta_n: float = 0.0
    omega_dot: float = 0.0
    idot: float = 0.0
    cuc: float = 0.0
    cus: float = 0.0
    crc: float = 0.0
    crs: float = 0.0
    cic: float = 0.0
    cis: float = 0.0
    toe: float = 0.0
    week: int = 0
    tgd: float = 0.0
    data_sources: float = 0.0
    bgd_e5a_e1: float = 0.0
    bgd_e5b_e1: float = 0.0
    iode: float = 0.0
    iodc: float = 0.0
    codes_on_l2: float = 0.0
    l2_p_flag: float = 0.0
    sv_accuracy: float = 0.0
    sv_health: float = 0.0
    fit_interval: float = 0.0
    toc_seconds: float = 0.0
    glo_px_m: float = 0.0
    glo_py_m: float = 0.0
    glo_pz_m: float = 0.0
    glo_vx_m_s: float = 0.0
    glo_vy_m_s: float = 0.0
    glo_vz_m_s: float = 0.0
    glo_ax_m_s2: float = 0.0
    glo_ay_m_s2: float = 0.0
    glo_az_m_s2: float = 0.0
    glo_tau_n: float = 0.0
    glo_gamma_n: float = 0.0
    glo_frequency_channel: int = 0

    @property
    def sat_id(self) -> str:
        return f"{self.system}{self.prn:02d}"


def _parse_nav_float(s: str) -> float:
    """A RINEX number with a D or E exponent; blank or malformed -> 0.0."""
    t = s.strip().replace("D", "E").replace("d", "e")
    if not t:
        return 0.0
    try:
        return float(t)
    except ValueError:
        return 0.0


def _gps_seconds_of_week(dt: datetime) -> float:
    return (dt - GPS_EPOCH).total_seconds() % WEEK_SEC


def _gps_week(dt: datetime) -> int:
    return int((dt - GPS_EPOCH).total_seconds() // WEEK_SEC)


def _fields(line: str, first: int) -> list[float]:
    """Four 19-column numbers starting at column ``first``; a field counts
    only when the line (newline included) reaches its last column."""
    out = []
    for j in range(4):
        a = first + 19 * j
        out.append(_parse_nav_float(line[a:a + 19]) if a + 19 <= len(line) else 0.0)
    return out


# Broadcast-orbit slots 0..27 (7 lines x 4) of a Kepler record -> field.
_KEPLER_SLOTS = {
    0: "iode", 1: "crs", 2: "delta_n", 3: "M0",
    4: "cuc", 5: "e", 6: "cus", 7: "sqrt_a",
    8: "toe", 9: "cic", 10: "omega0", 11: "cis",
    12: "i0", 13: "crc", 14: "omega", 15: "omega_dot",
    16: "idot", 17: "codes_on_l2", 19: "l2_p_flag",
    20: "sv_accuracy", 21: "sv_health", 22: "tgd", 23: "iodc",
    25: "fit_interval",
}


def _kepler(prn: int, toc: datetime, system: str, clock: list[float], orbit: list[float]) -> NavMessage:
    kw = {name: orbit[k] for k, name in _KEPLER_SLOTS.items()}
    kw["week"] = int(orbit[18])
    if system == "E":
        # Galileo: slot 17 is the data-source mask, 22/23 the BGDs; tgd keeps
        # BGD(E5a/E1) for callers that read only tgd (nav_rinex.py:263-270).
        kw["data_sources"] = orbit[17]
        kw["bgd_e5a_e1"] = orbit[22]
        kw["bgd_e5b_e1"] = orbit[23]
        kw["tgd"] = orbit[22]
    return NavMessage(prn=prn, toc=toc, system=system, af0=clock[0], af1=clock[1], af2=clock[2],
                      toc_seconds=_gps_seconds_of_week(toc), **kw)


def _glonass(prn: int, toc: datetime, head: list[float], rows: list[list[float]]) -> NavMessage:
    """RINEX 3 GLONASS record: -TauN, GammaN on the first line; per axis
    position, velocity, acceleration in km units (nav_rinex.py:354-424)."""
    (px, vx, ax, health), (py, vy, ay, chan), (pz, vz, az, _age) = rows
    sow = _gps_seconds_of_week(toc)
    k = 1000.0
    return NavMessage(prn=prn, toc=toc, system="R", sv_health=health, toe=sow, week=_gps_week(toc),
                      toc_seconds=sow, glo_px_m=px * k, glo_py_m=py * k, glo_pz_m=pz * k,
                      glo_vx_m_s=vx * k, glo_vy_m_s=vy * k, glo_vz_m_s=vz * k,
                      glo_ax_m_s2=ax * k, glo_ay_m_s2=ay * k, glo_az_m_s2=az * k,
                      glo_tau_n=-head[0], glo_gamma_n=head[1], glo_frequency_channel=int(chan))


def _record_v3(lines: list[str], i: int, keep: set[str]):
    line = lines[i]
    system = line[0] if line and line[0] != " " else "G"
    length = 4 if system in ("R", "S") else 8
    if i + length - 1 >= len(lines):
        return None, 1
    if system not in keep:
        return None, length
    prn_s = line[1:3].strip()
    if not prn_s:
        return None, length
    if system == "R":
        try:
            prn = int(prn_s)
        except ValueError:
            return None, 4
    else:
        prn = int(prn_s)
    toc = datetime(int(line[4:8]), int(line[9:11]), int(line[12:14]), int(line[15:17]), int(line[18:20]),
                   int(float(line[21:23])))
    head = [_parse_nav_float(line[23:42]), _parse_nav_float(line[42:61]), _parse_nav_float(line[61:80])]
    if system == "R":
        return _glonass(prn, toc, head, [_fields(lines[i + r], 4) for r in (1, 2, 3)]), 4
    orbit = []
    for r in range(1, 8):
        orbit += _fields(lines[i + r] if i + r < len(lines) else "", 4)
    return _kepler(prn, toc, system, head, orbit), length


def _record_v2(lines: list[str], i: int):
    if i + 7 >= len(lines):
        return None, 1
    line = lines[i]
    prn_s = line[0:2].strip()
    if not prn_s:
        return None, 8
    try:
        prn = int(prn_s)
    except ValueError:
        return None, 8
    yy = int(line[3:5])
    toc = datetime(yy + (2000 if yy < 80 else 1900), int(line[6:8]), int(line[9:11]), int(line[12:14]),
                   int(line[15:17]), int(float(line[17:22])))
    clock = [_parse_nav_float(line[22:41]), _parse_nav_float(line[41:60]), _parse_nav_float(line[60:79])]
    orbit = []
    for r in range(1, 8):
        orbit += _fields(lines[i + r], 3)
    return _kepler(prn, toc, "G", clock, orbit), 8


def read_nav_rinex(filepath, systems: tuple[str, ...] = ("G",), key_by_sat_id: bool = False):
    """Parse a RINEX 2 or 3 navigation file (nav_rinex.py:137-209): dict of
    PRN (or "G05"-style id) -> records sorted by toc.  RINEX 3 keeps only
    ``systems``; a record that fails to parse is skipped line by line."""
    with open(Path(filepath)) as f:
        lines = f.readlines()
    i, version = 0, 0.0
    while i < len(lines):
        line = lines[i]
        if "RINEX VERSION / TYPE" in line.rstrip():
            head = line[:20].strip()
            if head:
                try:
                    version = float(head.split()[0])
                except ValueError:
                    pass
        elif "END OF HEADER" in line.rstrip():
            i += 1
            break
        i += 1
    keep = {s.upper() for s in systems}
    out: dict = {}
    while i < len(lines):
        if not lines[i].strip():
            i += 1
            continue
        try:
            nav, used = _record_v3(lines, i, keep) if version >= 3.0 else _record_v2(lines, i)
        except (ValueError, IndexError):
            i += 1
            continue
        if nav is not None:
            out.setdefault(nav.sat_id if key_by_sat_id else nav.prn, []).append(nav)
        i += used
    for recs in out.values():
        recs.sort(key=lambda m: m.toc)
    return out


def read_nav_rinex_multi(filepath, systems: tuple[str, ...] = ("G", "E", "J")):
    """Mixed RINEX 3 file keyed by sat id (nav_rinex.py:212-217)."""
    return read_nav_rinex(filepath, systems=systems, key_by_sat_id=True)


__all__ = ["NavMessage", "read_nav_rinex", "read_nav_rinex_multi"]
