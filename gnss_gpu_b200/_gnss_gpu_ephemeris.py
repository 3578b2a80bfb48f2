"""Drop-in for the reference's ``_gnss_gpu_ephemeris`` extension module
(python/gnss_gpu/_ephemeris_bindings.cpp:1-90): broadcast-ephemeris
satellite positions of packed ``EphemerisParams`` records, computed by this
library's FP64 kernel (``pf_sat_positions`` / ``pf_sat_positions_batch``).

``params_flat`` is the float64 view of the packed records, 176 bytes each
(21 doubles, the int week and padding; ephemeris.py:135-171 packs them), and
the functions keep the binding's argument order, shapes and error text.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N

EPHEMERIS_PARAMS_SIZE = N.EPHEMERIS_DTYPE.itemsize          # 176
EPHEMERIS_PARAMS_N_DOUBLES = (EPHEMERIS_PARAMS_SIZE - 4) // 8  # 21


class EphemerisParams:
    """Field-by-field record (the binding's ``EphemerisParams`` class,
    _ephemeris_bindings.cpp:11-34).  ``tobytes()`` packs it in the C layout."""

    __slots__ = N.EPHEMERIS_FIELDS + ("week",)

    def __init__(self):
        for k in N.EPHEMERIS_FIELDS:
            setattr(self, k, 0.0)
        self.week = 0

    def tobytes(self) -> bytes:
        rec = np.zeros(1, N.EPHEMERIS_DTYPE)
        for k in N.EPHEMERIS_FIELDS:
            rec[k] = float(getattr(self, k))
        rec["week"] = int(self.week)
        return rec.tobytes()


def _records(params_flat, n_sat: int) -> np.ndarray:
    buf = np.ascontiguousarray(np.asarray(params_flat, dtype=np.float64)).reshape(-1)
    if buf.size * 8 < n_sat * EPHEMERIS_PARAMS_SIZE:
        raise RuntimeError("params_flat is too small for n_sat EphemerisParams structs")
    return buf


def compute_satellite_position(params_flat, gps_time: float, n_sat: int):
    """ECEF positions [n_sat, 3] and clock corrections [n_sat] at GPS second
    of week ``gps_time`` (GPS constants; _ephemeris_bindings.cpp:37-58)."""
    n_sat = int(n_sat)
    buf = _records(params_flat, n_sat)
    pos = np.empty((n_sat, 3), np.float64)
    clk = np.empty(n_sat, np.float64)
    N.check(N.load().pf_sat_positions(C.c_void_p(buf.ctypes.data), float(gps_time), N.dptr(pos), N.dptr(clk), n_sat))
    return pos, clk


def compute_satellite_position_batch(params_flat, gps_times, n_sat: int):
    """Positions [n_epoch, n_sat, 3] and clocks [n_epoch, n_sat] of the same
    records at every time of ``gps_times`` (_ephemeris_bindings.cpp:61-84)."""
    n_sat = int(n_sat)
    buf = _records(params_flat, n_sat)
    t = np.ascontiguousarray(np.asarray(gps_times, dtype=np.float64)).reshape(-1)
    pos = np.empty((t.size, n_sat, 3), np.float64)
    clk = np.empty((t.size, n_sat), np.float64)
    N.check(N.load().pf_sat_positions_batch(C.c_void_p(buf.ctypes.data), N.dptr(t), N.dptr(pos), N.dptr(clk),
                                            int(t.size), n_sat))
    return pos, clk
