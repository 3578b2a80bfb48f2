"""Broadcast ephemeris on the device: drop-in for the reference's
``gnss_gpu.ephemeris.Ephemeris`` (python/gnss_gpu/ephemeris.py:174-587).

Record selection (closest toe, Galileo message priority), validity checks,
time-scale alignment and the group-delay choice are host logic with the
reference's rules.  Every position and clock is computed on the device by
``pf_broadcast_orbits``: GPS, Galileo, QZSS and BeiDou Kepler records with
their own constants and GLONASS state vectors through the RK4 integrator, all
epochs and satellites of one call in one launch.  The reference runs only GPS
on its GPU kernel and every other system through its CPU code; here nothing
falls back to the host.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _native as N

GPS_MU = 3.986005e14
GPS_OMEGA_E = 7.2921151467e-5
GPS_F = -4.442807633e-10
GAL_MU = 3.986004418e14
GAL_OMEGA_E = 7.2921151467e-5
GAL_F = -4.442807309e-10
QZS_MU, QZS_OMEGA_E, QZS_F = GPS_MU, GPS_OMEGA_E, GPS_F
BDS_MU = GAL_MU
BDS_OMEGA_E = 7.292115e-5
BDS_F = GAL_F

GPS_WEEK_SEC = 604800.0
GPST_MINUS_BDT_S = 14.0
GPST_MINUS_UTC_S = 18.0
GLO_EPHEMERIS_TSTEP = 60.0

# BeiDou GEO PRNs left out of the usable set (nav_validity.py:22).
BEIDOU_GEO_PRNS = frozenset({1, 2, 3, 4, 5, 59, 60, 61, 62, 63})


# ------------------------------------------------------------ time scales
def unwrap_week_seconds(value: float) -> float:
    """Fold a second of week into [0, week) (gnss_time_scales.py:34-47)."""
    v = float(value)
    if not math.isfinite(v):
        return v
    while v < 0.0:
        v += GPS_WEEK_SEC
    while v >= GPS_WEEK_SEC:
        v -= GPS_WEEK_SEC
    return v


def broadcast_rx_seconds_of_week(system: str, recv_gpst_sow: float) -> float:
    """GPST receive time in the record's time scale: BDT for "C", the
    UTC-aligned GLONASS scale for "R" (gnss_time_scales.py:50-63)."""
    if system == "C":
        return unwrap_week_seconds(float(recv_gpst_sow) - GPST_MINUS_BDT_S)
    if system == "R":
        return unwrap_week_seconds(float(recv_gpst_sow) - GPST_MINUS_UTC_S)
    return float(recv_gpst_sow)


# ---------------------------------------------------------------- validity
def is_kepler_broadcast_valid(nav) -> bool:
    """Finite sqrt_a > 0 and 0 <= e < 1, not GLONASS or SBAS (nav_validity.py:25-45)."""
    if nav is None or getattr(nav, "system", None) in ("R", "S"):
        return False
    sa = float(getattr(nav, "sqrt_a", 0.0))
    ec = float(getattr(nav, "e", 0.0))
    return math.isfinite(sa) and sa > 0.0 and math.isfinite(ec) and 0.0 <= ec < 1.0


def is_glonass_broadcast_valid(nav) -> bool:
    """GLONASS state vector with radius in [1.5e7, 5e7] m (nav_validity.py:48-62)."""
    if nav is None or getattr(nav, "system", None) != "R":
        return False
    r = math.sqrt(sum(float(getattr(nav, k, 0.0)) ** 2 for k in ("glo_px_m", "glo_py_m", "glo_pz_m")))
    return math.isfinite(r) and 1.5e7 <= r <= 5.0e7


def is_beidou_geo(nav) -> bool:
    if nav is None or getattr(nav, "system", None) != "C":
        return False
    try:
        return int(getattr(nav, "prn")) in BEIDOU_GEO_PRNS
    except (TypeError, ValueError):
        return False


def is_broadcast_usable(nav) -> bool:
    """A GLONASS state or a Kepler broadcast, not a BeiDou GEO (nav_validity.py:78-86)."""
    if is_beidou_geo(nav):
        return False
    return is_glonass_broadcast_valid(nav) or is_kepler_broadcast_valid(nav)


# ------------------------------------------------------ record selection
def _normalize_sat_id(sat):
    """"g 5" -> "G05"; integers stay integers (ephemeris.py:85-95)."""
    if isinstance(sat, str):
        s = sat.strip().upper()
        if not s:
            return s
        system, prn = s[0], s[1:].strip().replace(" ", "")
        if system.isalpha() and prn.isdigit():
            return f"{system}{int(prn):02d}"
        return s.replace(" ", "")
    return int(sat)


def _obs_band(obs_code) -> str:
    return obs_code[1] if obs_code and len(obs_code) >= 2 else ""


def _data_sources(nav) -> int:
    return int(round(nav.data_sources or nav.codes_on_l2))


def _galileo_priority(nav, obs_code) -> int:
    """Preference of a Galileo message for a signal band: I/NAV over F/NAV
    for E1 and E5b, F/NAV for E5a (ephemeris.py:104-117)."""
    band, ds = _obs_band(obs_code), _data_sources(nav)
    bit = lambda m: int(bool(ds & m))  # noqa: E731
    if band == "1":
        return 4 * bit(0x001) + 2 * bit(0x200) + bit(0x004)
    if band == "5":
        return 4 * bit(0x002) + 2 * bit(0x100)
    if band == "7":
        return 4 * bit(0x004) + 2 * bit(0x200)
    return 0


def _group_delay(nav, obs_code) -> float:
    """tgd, or for Galileo E1 the BGD of the message's signal pair
    (ephemeris.py:120-132)."""
    if nav.system != "E":
        return nav.tgd
    if _obs_band(obs_code) == "1":
        ds = _data_sources(nav)
        if ds & 0x200:
            return nav.bgd_e5b_e1
        if ds & 0x100:
            return nav.bgd_e5a_e1
        return nav.bgd_e5b_e1 if nav.bgd_e5b_e1 != 0.0 else nav.bgd_e5a_e1
    return nav.tgd


def _pack(navs, obs_codes=None, apply_group_delay: bool = True) -> np.ndarray:
    """pf_broadcast_t records of the messages (GLONASS state vectors or Kepler
    elements; the chosen group delay goes into tgd)."""
    rec = np.zeros(len(navs), N.BROADCAST_DTYPE)
    for j, nav in enumerate(navs):
        rec["system"][j] = ord(nav.system[0]) if nav.system else ord("G")
        if nav.system == "R":
            g = rec["glonass"]
            g["toe"][j] = nav.toe
            g["pos"][j] = (nav.glo_px_m, nav.glo_py_m, nav.glo_pz_m)
            g["vel"][j] = (nav.glo_vx_m_s, nav.glo_vy_m_s, nav.glo_vz_m_s)
            g["acc"][j] = (nav.glo_ax_m_s2, nav.glo_ay_m_s2, nav.glo_az_m_s2)
            g["tau_n"][j] = nav.glo_tau_n
            g["gamma_n"][j] = nav.glo_gamma_n
            continue
        k = rec["kepler"]
        for f in N.EPHEMERIS_FIELDS:
            if f not in ("toc", "tgd"):
                k[f][j] = float(getattr(nav, f))
        k["toc"][j] = nav.toc_seconds
        code = None if obs_codes is None else obs_codes[j]
        k["tgd"][j] = _group_delay(nav, code) if apply_group_delay else 0.0
        k["week"][j] = int(nav.week)
    return rec


def broadcast_orbits(records: np.ndarray, times, rec_index=None, glo_step: float = GLO_EPHEMERIS_TSTEP):
    """Positions [E, S, 3] and clocks [E, S] of pf_broadcast_t ``records`` at
    GPST seconds of week ``times`` [E], one device launch: rec_index [E, S]
    picks the record of each output (default: record s for column s; -1
    gives NaN).  Raises if no CUDA device is present."""
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("gnss_gpu_b200 ephemeris needs a CUDA device (no host fallback)")
    rec = np.ascontiguousarray(records, dtype=N.BROADCAST_DTYPE)
    t = np.ascontiguousarray(np.asarray(times, dtype=np.float64).reshape(-1))
    n_epoch = t.size
    if rec_index is None:
        n_sat, idx = len(rec), None
    else:
        idx = np.ascontiguousarray(np.asarray(rec_index, dtype=np.int32))
        if idx.ndim != 2 or idx.shape[0] != n_epoch:
            raise ValueError("rec_index must have shape [n_epoch, n_sat]")
        n_sat = idx.shape[1]
    pos = np.empty((n_epoch, n_sat, 3), np.float64)
    clk = np.empty((n_epoch, n_sat), np.float64)
    if n_epoch == 0 or n_sat == 0:
        return pos, clk
    dev = torch.device("cuda", torch.cuda.current_device())
    d_rec = torch.from_numpy(rec.view(np.uint8).copy()).to(dev) if len(rec) else None
    d_t = torch.from_numpy(t).to(dev)
    d_idx = torch.from_numpy(idx).to(dev) if idx is not None else None
    d_pos = torch.empty((n_epoch, n_sat, 3), dtype=torch.float64, device=dev)
    d_clk = torch.empty((n_epoch, n_sat), dtype=torch.float64, device=dev)
    st = torch.cuda.current_stream(dev)
    ptr = lambda x: C.c_void_p(x.data_ptr() if x is not None else 0)  # noqa: E731
    N.check(N.load().pf_broadcast_orbits(ptr(d_rec), len(rec), ptr(d_idx), ptr(d_t), n_epoch, n_sat,
                                         float(glo_step), ptr(d_pos), ptr(d_clk), C.c_void_p(st.cuda_stream)))
    pos[...] = d_pos.cpu().numpy()
    clk[...] = d_clk.cpu().numpy()
    return pos, clk


class Ephemeris:
    """Satellite positions and clocks from parsed navigation messages
    (ephemeris.py:174-412), any of G/E/J/C/R, computed on the device."""

    def __init__(self, nav_messages: dict) -> None:
        self._nav_messages = nav_messages
        self._prn_list = sorted(nav_messages.keys(), key=str)

    @property
    def available_prns(self) -> list:
        return list(self._prn_list)

    def select_ephemeris(self, prn, gps_time: float, obs_code: str | None = None):
        """The message whose toe is closest to ``gps_time`` in its own time
        scale (week crossover folded), ties broken by the Galileo priority
        for ``obs_code`` (ephemeris.py:196-236); None if the PRN is unknown."""
        prn = _normalize_sat_id(prn)
        if prn not in self._nav_messages and isinstance(prn, int):
            prn = f"G{prn:02d}"
        msgs = self._nav_messages.get(prn)
        if not msgs:
            return None
        best, best_key = None, None
        for m in msgs:
            dt = abs(broadcast_rx_seconds_of_week(m.system, gps_time) - m.toe)
            if dt > GPS_WEEK_SEC / 2.0:
                dt = GPS_WEEK_SEC - dt
            pri = _galileo_priority(m, obs_code) if (obs_code is not None and m.system == "E") else 0
            key = (dt, -pri)
            if best_key is None or key < best_key:
                best, best_key = m, key
        return best

    def compute_single(self, nav, gps_time: float, obs_code: str | None = None, *,
                       apply_group_delay: bool = True):
        """Position (3,) and clock of one message at ``gps_time``
        (ephemeris.py:428-512, on the device)."""
        if not (is_glonass_broadcast_valid(nav) or is_kepler_broadcast_valid(nav)):
            raise ValueError(f"invalid or unsupported broadcast ephemeris (system={nav.system!r}, "
                             f"sqrt_a={nav.sqrt_a!r}, e={nav.e!r})")
        pos, clk = broadcast_orbits(_pack([nav], None if obs_code is None else [obs_code], apply_group_delay),
                                    [gps_time])
        return pos[0, 0], float(clk[0, 0])

    def compute(self, gps_time: float, prn_list=None, obs_codes=None):
        """Positions [n, 3], clocks [n] and the PRNs of the rows at GPS
        second of week ``gps_time`` (ephemeris.py:277-318): unusable or
        non-finite results are dropped."""
        if prn_list is None:
            prn_list = self._prn_list
        if obs_codes is not None and len(obs_codes) != len(prn_list):
            raise ValueError("obs_codes must match prn_list length")
        navs, codes, used = [], [], []
        for i, prn in enumerate(prn_list):
            code = None if obs_codes is None else obs_codes[i]
            nav = self.select_ephemeris(prn, gps_time, code)
            if is_broadcast_usable(nav):
                navs.append(nav)
                codes.append(code)
                used.append(prn)
        if not used:
            return np.array([]).reshape(0, 3), np.array([]), []
        pos, clk = broadcast_orbits(_pack(navs, codes), [gps_time])
        pos, clk = pos[0], clk[0]
        ok = np.isfinite(pos).all(axis=1) & np.isfinite(clk)
        if not ok.all():
            used = [p for p, k in zip(used, ok) if k]
            pos, clk = pos[ok], clk[ok]
            if not used:
                return np.array([]).reshape(0, 3), np.array([]), []
        return pos, clk, used

    def compute_batch(self, gps_times, prn_list=None):
        """Positions [E, n, 3] and clocks [E, n] with records re-selected per
        epoch; the PRNs kept are those usable at every epoch
        (ephemeris.py:320-412).  One launch for all epochs."""
        t = np.asarray(gps_times, dtype=np.float64).reshape(-1)
        if prn_list is None:
            prn_list = self._prn_list
        if t.size == 0:
            return np.array([]).reshape(0, 0, 3), np.array([]).reshape(0, 0), []
        sel = [[self.select_ephemeris(p, float(x)) for p in prn_list] for x in t]
        keep = [j for j in range(len(prn_list)) if all(is_broadcast_usable(row[j]) for row in sel)]
        used = [prn_list[j] for j in keep]
        if not used:
            return np.array([]).reshape(t.size, 0, 3), np.array([]).reshape(t.size, 0), []
        slot: dict[int, int] = {}
        navs = []
        idx = np.empty((t.size, len(keep)), np.int32)
        for e, row in enumerate(sel):
            for c, j in enumerate(keep):
                nav = row[j]
                k = slot.get(id(nav))
                if k is None:
                    k = slot[id(nav)] = len(navs)
                    navs.append(nav)
                idx[e, c] = k
        pos, clk = broadcast_orbits(_pack(navs), t, idx)
        return pos, clk, used


__all__ = [
    "Ephemeris", "broadcast_orbits", "broadcast_rx_seconds_of_week", "unwrap_week_seconds",
    "is_kepler_broadcast_valid", "is_glonass_broadcast_valid", "is_beidou_geo", "is_broadcast_usable",
    "GPS_MU", "GPS_OMEGA_E", "GPS_F", "GAL_MU", "GAL_OMEGA_E", "GAL_F", "BDS_MU", "BDS_OMEGA_E", "BDS_F",
    "GPS_WEEK_SEC",
]
