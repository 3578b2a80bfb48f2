"""Sagnac-corrected geometric range on the device: drop-in for the
reference's python/gnss_gpu/range_model.py:1-40 (``pf_sagnac``).

The satellite is rotated about the earth axis by omega_e * |rx - sat| / c,
the earth's rotation during the signal's transit, and the range is taken to
the rotated position.  The batch forms take one receiver per epoch and
every satellite of that epoch in one launch.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N

C_LIGHT = 299792458.0
OMEGA_E = 7.2921151467e-5


def _sagnac(rx: np.ndarray, sat: np.ndarray, want_rot: bool, want_range: bool):
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("gnss_gpu_b200.range_model needs a CUDA device (no host fallback)")
    n_epoch, n_sat = sat.shape[0], sat.shape[1]
    rot = np.empty((n_epoch, n_sat, 3), np.float64)
    rng = np.empty((n_epoch, n_sat), np.float64)
    if n_epoch == 0 or n_sat == 0:
        return rot, rng
    dev = torch.device("cuda", torch.cuda.current_device())
    d_rx = torch.from_numpy(np.ascontiguousarray(rx)).to(dev)
    d_sat = torch.from_numpy(np.ascontiguousarray(sat)).to(dev)
    d_rot = torch.empty((n_epoch, n_sat, 3), dtype=torch.float64, device=dev) if want_rot else None
    d_rng = torch.empty((n_epoch, n_sat), dtype=torch.float64, device=dev) if want_range else None
    ptr = lambda x: C.c_void_p(x.data_ptr() if x is not None else 0)  # noqa: E731
    st = torch.cuda.current_stream(dev)
    N.check(N.load().pf_sagnac(ptr(d_rx), ptr(d_sat), n_epoch, n_sat, ptr(d_rot), ptr(d_rng),
                               C.c_void_p(st.cuda_stream)))
    if want_rot:
        rot[...] = d_rot.cpu().numpy()
    if want_range:
        rng[...] = d_rng.cpu().numpy()
    return rot, rng


def rotate_satellites_sagnac(receiver_ecef, sat_ecef) -> np.ndarray:
    """Satellite positions [n, 3] rotated for the earth's rotation during
    signal transit (range_model.py:12-30)."""
    rx = np.asarray(receiver_ecef, dtype=np.float64).reshape(1, 3)
    sat = np.asarray(sat_ecef, dtype=np.float64).reshape(1, -1, 3)
    return _sagnac(rx, sat, True, False)[0][0]


def geometric_ranges_sagnac(receiver_ecef, sat_ecef) -> np.ndarray:
    """Receiver-to-satellite ranges [n] to the rotated positions
    (range_model.py:33-40)."""
    rx = np.asarray(receiver_ecef, dtype=np.float64).reshape(1, 3)
    sat = np.asarray(sat_ecef, dtype=np.float64).reshape(1, -1, 3)
    return _sagnac(rx, sat, False, True)[1][0]


def sagnac_batch(receivers_ecef, sat_ecef):
    """Rotated satellites [E, S, 3] and ranges [E, S] for receivers [E, 3]
    and satellites [E, S, 3], one launch."""
    rx = np.asarray(receivers_ecef, dtype=np.float64).reshape(-1, 3)
    sat = np.asarray(sat_ecef, dtype=np.float64)
    if sat.ndim != 3 or sat.shape[0] != rx.shape[0] or sat.shape[2] != 3:
        raise ValueError("sat_ecef must have shape [n_epoch, n_sat, 3] matching receivers_ecef [n_epoch, 3]")
    return _sagnac(rx, sat, True, True)


__all__ = ["C_LIGHT", "OMEGA_E", "rotate_satellites_sagnac", "geometric_ranges_sagnac", "sagnac_batch"]
