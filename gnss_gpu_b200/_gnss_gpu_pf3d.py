"""Drop-in for the reference's pybind11 module gnss_gpu._gnss_gpu_pf3d:
pf_weight_3d on FP64 NumPy arrays, log_weights written in place."""
from __future__ import annotations

import numpy as np

from . import _native as N
from ._gnss_gpu_pf import _in, _out

__all__ = ["pf_weight_3d"]


def pf_weight_3d(px, py, pz, pcb, sat_ecef, pseudoranges, weights_sat, triangles, log_weights, n_particles, n_sat,
                 sigma_los, sigma_nlos, nlos_bias, blocked_nlos_prob=1.0, clear_nlos_prob=0.0):
    n, s = int(n_particles), int(n_sat)
    L = N.load()
    p = [_in(a, n, nm) for a, nm in ((px, "px"), (py, "py"), (pz, "pz"), (pcb, "pcb"))]
    sat = _in(sat_ecef, 3 * s, "sat_ecef")
    pr = _in(pseudoranges, s, "pseudoranges")
    w = _in(weights_sat, s, "weights_sat")
    tri = np.ascontiguousarray(triangles, dtype=np.float64).reshape(-1)
    if tri.size % 9:
        raise ValueError("triangles must have shape [N, 3, 3]")
    lw = _out(log_weights, n, "log_weights")
    N.check(L.pf_weight_3d(*(N.dptr(a) for a in p), N.dptr(sat), N.dptr(pr), N.dptr(w), N.dptr(tri),
                           tri.size // 9, N.dptr(lw), n, s, float(sigma_los), float(sigma_nlos), float(nlos_bias),
                           float(blocked_nlos_prob), float(clear_nlos_prob)))
