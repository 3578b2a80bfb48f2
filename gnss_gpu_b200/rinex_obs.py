"""RINEX 2.x / 3.x observation reader (python/gnss_gpu/io/rinex.py of the
reference): header metadata, observation codes per system, epochs with their
satellites and 16-column observation fields, and ``pseudoranges()`` giving
the [n_epoch, max_sat] array the filter's update takes.

Host-side text parsing with the reference's column rules and quirks; the
arrays it returns go to the device through the filter's own calls.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from datetime import datetime
from pathlib import Path

import numpy as np


@dataclass
class RinexHeader:
    version: float = 0.0
    sat_system: str = ""
    marker_name: str = ""
    approx_position: np.ndarray = field(default_factory=lambda: np.zeros(3))
    obs_types: dict = field(default_factory=dict)
    interval: float = 0.0


@dataclass
class RinexEpoch:
    time: datetime
    satellites: list
    observations: dict  # {sat_id: {obs_code: value}}


@dataclass
class RinexObs:
    header: RinexHeader
    epochs: list

    def pseudoranges(self, obs_code: str = "C1C"):
        """(times, pr [n_epoch, max_sat] NaN-padded, sat ids per epoch) of the
        epochs with at least one non-zero ``obs_code`` value (rinex.py:41-70)."""
        times, rows, sats = [], [], []
        for ep in self.epochs:
            vals = {s: o[obs_code] for s, o in ep.observations.items() if obs_code in o and o[obs_code] != 0.0}
            if vals:
                times.append(ep.time)
                sats.append(list(vals))
                rows.append(list(vals.values()))
        if not times:
            return [], np.array([]), []
        pr = np.full((len(rows), max(len(r) for r in rows)), np.nan)
        for i, r in enumerate(rows):
            pr[i, :len(r)] = r
        return times, pr, sats


def _values(record: str, codes: list, first: int) -> dict:
    """Fields of 16 columns (14-column value, LLI, strength) from ``first``;
    blank, short or malformed fields read 0.0."""
    out = {}
    for k, code in enumerate(codes):
        a = first + 16 * k
        txt = record[a:a + 14].strip() if a + 14 <= len(record) else ""
        try:
            out[code] = float(txt) if txt else 0.0
        except ValueError:
            out[code] = 0.0
    return out


def _sat_like(text: str) -> bool:
    t = text.strip().upper()
    return len(t) >= 2 and t[0].isalpha() and t[1:].strip().isdigit()


def _v2_sat(sat: str) -> str:
    s = sat.strip().upper()
    if not s:
        return s
    if s[0].isalpha():
        return f"{s[0]}{int(s[1:]):02d}" if s[1:].strip().isdigit() else s
    return f"G{int(s):02d}" if s.isdigit() else s


def _header(lines: list) -> tuple[RinexHeader, int]:
    h = RinexHeader()
    i = 0
    while i < len(lines):
        line = lines[i]
        label = line[60:].strip() if len(line) > 60 else ""
        if label == "RINEX VERSION / TYPE":
            h.version = float(line[:9])
            h.sat_system = line[40:41].strip()
        elif label == "MARKER NAME":
            h.marker_name = line[:60].strip()
        elif label == "APPROX POSITION XYZ":
            h.approx_position = np.array([float(v) for v in line[:60].split()[:3]])
        elif label.startswith("SYS / # / OBS TYPES"):
            system = line[0].strip()
            if system:
                n = int(line[3:6])
                codes = line[7:60].split()
                while len(codes) < n:
                    i += 1
                    codes += lines[i][7:60].split()
                h.obs_types[system] = codes[:n]
        elif label == "# / TYPES OF OBSERV":
            n = int(line[:6])
            codes = line[6:60].split()
            while len(codes) < n:
                i += 1
                codes += lines[i][6:60].split()
            h.obs_types[h.sat_system or "G"] = codes[:n]
            h.obs_types[""] = codes[:n]
        elif label == "INTERVAL":
            h.interval = float(line[:10])
        elif label == "END OF HEADER":
            return h, i + 1
        i += 1
    return h, i


def _epochs_v3(lines: list, i: int, h: RinexHeader) -> list:
    out = []
    while i < len(lines):
        line = lines[i]
        if not line.startswith(">"):
            i += 1
            continue
        parts = line[2:].split()
        if len(parts) < 7:
            i += 1
            continue
        try:
            sec = float(parts[5])
            t = datetime(int(parts[0]), int(parts[1]), int(parts[2]), int(parts[3]), int(parts[4]), int(sec),
                         int((sec - int(sec)) * 1e6))
            flag = int(parts[6])
            n_sat = int(parts[7]) if len(parts) > 7 else 0
        except (ValueError, IndexError):
            i += 1
            continue
        if flag > 1:  # event records: skip the special lines
            i += 1 + n_sat
            continue
        sats, obs = [], {}
        for _ in range(n_sat):
            i += 1
            if i >= len(lines):
                break
            rec = lines[i].rstrip("\n")
            sat = rec[:3].strip()
            sats.append(sat)
            codes = h.obs_types.get(sat[0] if sat else "", [])
            need = 3 + 16 * len(codes)
            while len(rec) < need and i + 1 < len(lines):
                nxt = lines[i + 1]
                if nxt.startswith(">") or _sat_like(nxt[:3].strip()):
                    break
                i += 1
                rec += lines[i][3:].rstrip("\n")
            obs[sat] = _values(rec, codes, 3)
        out.append(RinexEpoch(time=t, satellites=sats, observations=obs))
        i += 1
    return out


def _epochs_v2(lines: list, i: int, h: RinexHeader) -> list:
    out = []
    codes = h.obs_types.get("", [])
    per_sat = max(1, (len(codes) + 4) // 5)
    while i < len(lines):
        line = lines[i]
        if not line.strip():
            i += 1
            continue
        try:
            yy = int(line[1:3])
            sec = float(line[15:26])
            t_fields = (yy + (2000 if yy < 80 else 1900), int(line[4:6]), int(line[7:9]), int(line[10:12]),
                        int(line[13:15]), int(sec), int(round((sec - int(sec)) * 1e6)))
            flag = int(line[28:29])
            n_sat = int(line[29:32])
        except (ValueError, IndexError):
            i += 1
            continue
        blob = line[32:].rstrip("\n")
        while len(blob) < 3 * n_sat and i + 1 < len(lines):
            i += 1
            blob += lines[i][32:].rstrip("\n")
        sats = [_v2_sat(s) for s in (blob[k:k + 3].strip() for k in range(0, 3 * n_sat, 3)) if s.strip()]
        i += 1
        if flag > 1:
            i += n_sat * per_sat
            continue
        obs = {}
        for sat in sats:
            rec = ""
            for _ in range(per_sat):
                if i >= len(lines):
                    break
                rec += lines[i].rstrip("\n").ljust(80)
                i += 1
            obs[sat] = _values(rec, codes, 0)
        out.append(RinexEpoch(time=datetime(*t_fields), satellites=sats, observations=obs))
    return out


def read_rinex_obs(filepath) -> RinexObs:
    """Parse a RINEX 2.x / 3.x observation file (rinex.py:156-263)."""
    with open(Path(filepath)) as f:
        lines = f.readlines()
    h, i = _header(lines)
    epochs = _epochs_v2(lines, i, h) if h.version < 3.0 else _epochs_v3(lines, i, h)
    return RinexObs(header=h, epochs=epochs)


__all__ = ["RinexHeader", "RinexEpoch", "RinexObs", "read_rinex_obs"]
