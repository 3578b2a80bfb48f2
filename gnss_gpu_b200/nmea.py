"""NMEA 0183 reading and writing (python/gnss_gpu/io/nmea.py and
nmea_writer.py of the reference): GGA / RMC parsing with checksum checks,
GGA / RMC / GSA / GSV / VTG sentences from positioning results, and
``ecef_to_nmea`` whose ECEF -> geodetic conversion runs on the device
(``pf_ecef_to_lla``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from datetime import date, datetime, timezone
from pathlib import Path

import numpy as np

from . import _native as N


# ----------------------------------------------------------------- reading
@dataclass
class GGAMessage:
    time: datetime
    latitude: float
    longitude: float
    fix_quality: int
    n_satellites: int
    hdop: float
    altitude: float
    geoid_sep: float


@dataclass
class RMCMessage:
    time: datetime
    status: str
    latitude: float
    longitude: float
    speed_knots: float
    course: float


def _angle(val: str, hemi: str, deg_digits: int, negative: str) -> float:
    """ddmm.mmmm / dddmm.mmmm -> signed degrees; blank -> 0."""
    if not val:
        return 0.0
    v = float(val[:deg_digits]) + float(val[deg_digits:]) / 60.0
    return -v if hemi == negative else v


def _time(hms: str, dmy: str = "") -> datetime:
    s = float(hms[4:])
    fields = (int(hms[0:2]), int(hms[2:4]), int(s), int((s - int(s)) * 1e6))
    if dmy:
        return datetime(int(dmy[4:6]) + 2000, int(dmy[2:4]), int(dmy[0:2]), *fields)
    return datetime(2000, 1, 1, *fields)


def _checksum_ok(sentence: str) -> bool:
    if "*" not in sentence:
        return True
    body, chk = sentence.split("*", 1)
    x = 0
    for ch in body.lstrip("$"):
        x ^= ord(ch)
    try:
        return x == int(chk[:2], 16)
    except ValueError:
        return False


def parse_nmea(filepath) -> list:
    """GGA and RMC messages of an NMEA file, in file order; lines that fail
    the checksum or do not parse are skipped (nmea.py:78-119)."""
    out = []
    with open(Path(filepath)) as f:
        for raw in f:
            line = raw.strip()
            if not line.startswith("$") or not _checksum_ok(line):
                continue
            fl = line.split("*")[0].lstrip("$").split(",")
            kind = fl[0][-3:]
            try:
                if kind == "GGA" and len(fl) >= 15:
                    out.append(GGAMessage(
                        time=_time(fl[1]), latitude=_angle(fl[2], fl[3], 2, "S"),
                        longitude=_angle(fl[4], fl[5], 3, "W"),
                        fix_quality=int(fl[6]) if fl[6] else 0, n_satellites=int(fl[7]) if fl[7] else 0,
                        hdop=float(fl[8]) if fl[8] else 0.0, altitude=float(fl[9]) if fl[9] else 0.0,
                        geoid_sep=float(fl[11]) if fl[11] else 0.0))
                elif kind == "RMC" and len(fl) >= 12:
                    out.append(RMCMessage(
                        time=_time(fl[1], fl[9]), status=fl[2], latitude=_angle(fl[3], fl[4], 2, "S"),
                        longitude=_angle(fl[5], fl[6], 3, "W"),
                        speed_knots=float(fl[7]) if fl[7] else 0.0, course=float(fl[8]) if fl[8] else 0.0))
            except (ValueError, IndexError):
                continue
    return out


# ----------------------------------------------------------------- writing
class NMEAWriter:
    """NMEA sentences from positioning results (nmea_writer.py:12-230)."""

    def __init__(self, talker_id: str = "GP"):
        self.talker_id = talker_id

    @staticmethod
    def _checksum(body: str) -> str:
        x = 0
        for ch in body:
            x ^= ord(ch)
        return f"{x:02X}"

    @staticmethod
    def _deg_to_nmea(deg: float, is_lat: bool = True) -> tuple[str, str]:
        hemi = ("N" if deg >= 0 else "S") if is_lat else ("E" if deg >= 0 else "W")
        a = abs(deg)
        d = int(a)
        m = (a - d) * 60.0
        return (f"{d:02d}{m:07.4f}" if is_lat else f"{d:03d}{m:07.4f}"), hemi

    def _wrap(self, body: str) -> str:
        return f"${body}*{self._checksum(body)}"

    def gga(self, lat_deg, lon_deg, alt_m, time_utc=None, fix_quality=1, n_sats=0, hdop=1.0,
            geoid_sep=0.0) -> str:
        t = time_utc if time_utc is not None else datetime.now(timezone.utc)
        la, ns = self._deg_to_nmea(lat_deg, True)
        lo, ew = self._deg_to_nmea(lon_deg, False)
        return self._wrap(f"{self.talker_id}GGA,{t.strftime('%H%M%S.%f')[:10]},{la},{ns},{lo},{ew},"
                          f"{fix_quality},{n_sats:02d},{hdop:.1f},{alt_m:.3f},M,{geoid_sep:.3f},M,,")

    def rmc(self, lat_deg, lon_deg, time_utc=None, date_val=None, speed_knots=0.0, course_deg=0.0,
            status="A") -> str:
        t = time_utc if time_utc is not None else datetime.now(timezone.utc)
        if date_val is None:
            date_val = t.date() if isinstance(t, datetime) else date.today()
        la, ns = self._deg_to_nmea(lat_deg, True)
        lo, ew = self._deg_to_nmea(lon_deg, False)
        d = f"{date_val.day:02d}{date_val.month:02d}{date_val.year % 100:02d}"
        return self._wrap(f"{self.talker_id}RMC,{t.strftime('%H%M%S.%f')[:10]},{status},{la},{ns},{lo},{ew},"
                          f"{speed_knots:.1f},{course_deg:.1f},{d},,,")

    def gsa(self, prn_list, pdop=0.0, hdop=0.0, vdop=0.0, fix_type=3, mode="A") -> str:
        prns = [f"{p:02d}" for p in list(prn_list)[:12]]
        prns += [""] * (12 - len(prns))
        return self._wrap(f"{self.talker_id}GSA,{mode},{fix_type},{','.join(prns)},{pdop:.1f},{hdop:.1f},{vdop:.1f}")

    def gsv(self, satellites) -> list:
        n = len(satellites)
        n_msg = math.ceil(n / 4) if n > 0 else 1
        out = []
        for m in range(n_msg):
            cells = [f"{p:02d},{el:02d},{az:03d},{snr:02d}" for p, el, az, snr in satellites[4 * m:4 * m + 4]]
            cells += [",,,"] * (4 - len(cells))
            out.append(self._wrap(f"{self.talker_id}GSV,{n_msg},{m + 1},{n:02d}," + ",".join(cells)))
        return out

    def vtg(self, course_deg=0.0, speed_knots=0.0, speed_kmh=0.0) -> str:
        return self._wrap(f"{self.talker_id}VTG,{course_deg:.1f},T,,M,{speed_knots:.1f},N,{speed_kmh:.1f},K")

    def write_epoch(self, lat_deg, lon_deg, alt_m, time_utc=None, n_sats=0, hdop=1.0, speed_knots=0.0,
                    course_deg=0.0, prn_list=None, pdop=0.0, vdop=0.0, fix_quality=1) -> list:
        """GGA, RMC, GSA (when prn_list is given) and VTG of one epoch."""
        out = [self.gga(lat_deg, lon_deg, alt_m, time_utc=time_utc, fix_quality=fix_quality, n_sats=n_sats,
                        hdop=hdop),
               self.rmc(lat_deg, lon_deg, time_utc=time_utc, speed_knots=speed_knots, course_deg=course_deg)]
        if prn_list is not None:
            out.append(self.gsa(prn_list, pdop=pdop, hdop=hdop, vdop=vdop))
        out.append(self.vtg(course_deg=course_deg, speed_knots=speed_knots, speed_kmh=speed_knots * 1.852))
        return out


def positions_to_nmea(lat_deg_array, lon_deg_array, alt_m_array, times=None, filepath=None):
    """NMEA text of per-epoch positions; written to ``filepath`` (returning
    None) when given (nmea_writer.py:258-286)."""
    w = NMEAWriter()
    lines = []
    for i in range(len(lat_deg_array)):
        lines += w.write_epoch(lat_deg_array[i], lon_deg_array[i], alt_m_array[i],
                               time_utc=times[i] if times is not None else None)
    text = "\n".join(lines) + "\n"
    if filepath is not None:
        Path(filepath).write_text(text)
        return None
    return text


def ecef_to_lla(ecef_positions) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """WGS84 latitude, longitude (rad) and height (m) of ECEF points [n, 3]
    on the device (pf_ecef_to_lla)."""
    p = np.asarray(ecef_positions, dtype=np.float64).reshape(-1, 3)
    n = p.shape[0]
    x, y, z = (np.ascontiguousarray(p[:, k]) for k in range(3))
    lat, lon, alt = np.empty(n), np.empty(n), np.empty(n)
    N.check(N.load().pf_ecef_to_lla(N.dptr(x), N.dptr(y), N.dptr(z), N.dptr(lat), N.dptr(lon), N.dptr(alt), n))
    return lat, lon, alt


def ecef_to_nmea(ecef_positions, times=None, filepath=None):
    """NMEA text of ECEF positions [n, 3] (nmea_writer.py:289-325)."""
    lat, lon, alt = ecef_to_lla(ecef_positions)
    return positions_to_nmea(np.degrees(lat), np.degrees(lon), alt, times=times, filepath=filepath)


__all__ = ["GGAMessage", "RMCMessage", "parse_nmea", "NMEAWriter", "positions_to_nmea", "ecef_to_nmea",
           "ecef_to_lla"]
