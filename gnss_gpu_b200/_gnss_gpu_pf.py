"""Drop-in for the reference's pybind11 module gnss_gpu._gnss_gpu_pf
(python/gnss_gpu/_particle_filter_bindings.cpp:7-145): the same eight
functions, argument names and in-place semantics on FP64 NumPy arrays.

Differences kept on purpose:
* an output array that is not a C-contiguous float64 array of at least
  n_particles elements raises ValueError (the reference silently writes into
  a converted temporary and the result is lost);
* n_sat above 1024 raises ValueError (the reference overruns a 64-entry
  shared-memory table, weight.cu:11,21-28);
* random draws come from Philox4x32-10 keyed by (seed, particle, step), so
  they equal the reference's cuRAND draws in distribution only.
"""
from __future__ import annotations

import numpy as np

from . import _native as N

__all__ = ["pf_initialize", "pf_predict", "pf_weight", "pf_compute_ess",
           "pf_resample_systematic", "pf_resample_megopolis", "pf_estimate",
           "pf_get_particles"]


def _out(a, n, name):
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not a.flags.c_contiguous:
        raise ValueError(f"{name} must be a C-contiguous float64 numpy array")
    if a.size < n:
        raise ValueError(f"{name} has {a.size} elements, need {n}")
    return a


def _in(a, n, name):
    arr = np.ascontiguousarray(a, dtype=np.float64).ravel()
    if arr.size < n:
        raise ValueError(f"{name} has {arr.size} elements, need {n}")
    return arr


def pf_initialize(px, py, pz, pcb, init_x, init_y, init_z, init_cb, spread_pos, spread_cb,
                  n_particles, seed):
    n = int(n_particles)
    L = N.load()
    arrs = [_out(a, n, nm) for a, nm in ((px, "px"), (py, "py"), (pz, "pz"), (pcb, "pcb"))]
    N.check(L.pf_initialize(*(N.dptr(a) for a in arrs), float(init_x), float(init_y), float(init_z),
                            float(init_cb), float(spread_pos), float(spread_cb), n, int(seed)))


def pf_predict(px, py, pz, pcb, vx, vy, vz, dt, sigma_pos, sigma_cb, n_particles, seed, step):
    n = int(n_particles)
    L = N.load()
    arrs = [_out(a, n, nm) for a, nm in ((px, "px"), (py, "py"), (pz, "pz"), (pcb, "pcb"))]
    v = [_in(a, 1, nm) for a, nm in ((vx, "vx"), (vy, "vy"), (vz, "vz"))]
    N.check(L.pf_predict(*(N.dptr(a) for a in arrs), *(N.dptr(a) for a in v), float(dt), float(sigma_pos),
                         float(sigma_cb), n, int(seed), int(step)))


def pf_weight(px, py, pz, pcb, sat_ecef, pseudoranges, weights_sat, log_weights, n_particles, n_sat,
              sigma_pr):
    n, s = int(n_particles), int(n_sat)
    L = N.load()
    ins = [_in(a, n, nm) for a, nm in ((px, "px"), (py, "py"), (pz, "pz"), (pcb, "pcb"))]
    sat = _in(sat_ecef, 3 * s, "sat_ecef")
    pr = _in(pseudoranges, s, "pseudoranges")
    ws = _in(weights_sat, s, "weights_sat")
    lw = _out(log_weights, n, "log_weights")
    N.check(L.pf_weight(*(N.dptr(a) for a in ins), N.dptr(sat), N.dptr(pr), N.dptr(ws), N.dptr(lw), n, s,
                        float(sigma_pr)))


def pf_compute_ess(log_weights, n_particles):
    n = int(n_particles)
    L = N.load()
    lw = _in(log_weights, n, "log_weights")
    out = np.zeros(1)
    N.check(L.pf_compute_ess(N.dptr(lw), n, N.dptr(out)))
    return float(out[0])


def pf_resample_systematic(px, py, pz, pcb, log_weights, n_particles, seed):
    n = int(n_particles)
    L = N.load()
    arrs = [_out(a, n, nm) for a, nm in ((px, "px"), (py, "py"), (pz, "pz"), (pcb, "pcb"))]
    lw = _in(log_weights, n, "log_weights")
    N.check(L.pf_resample_systematic(*(N.dptr(a) for a in arrs), N.dptr(lw), n, int(seed)))


def pf_resample_megopolis(px, py, pz, pcb, log_weights, n_particles, n_iterations, seed):
    n = int(n_particles)
    L = N.load()
    arrs = [_out(a, n, nm) for a, nm in ((px, "px"), (py, "py"), (pz, "pz"), (pcb, "pcb"))]
    lw = _in(log_weights, n, "log_weights")
    N.check(L.pf_resample_megopolis(*(N.dptr(a) for a in arrs), N.dptr(lw), n, int(n_iterations), int(seed)))


def pf_estimate(px, py, pz, pcb, log_weights, result, n_particles):
    n = int(n_particles)
    L = N.load()
    ins = [_in(a, n, nm) for a, nm in ((px, "px"), (py, "py"), (pz, "pz"), (pcb, "pcb"))]
    lw = _in(log_weights, n, "log_weights")
    res = _out(result, 4, "result")
    N.check(L.pf_estimate(*(N.dptr(a) for a in ins), N.dptr(lw), N.dptr(res), n))


def pf_get_particles(px, py, pz, pcb, output, n_particles):
    n = int(n_particles)
    L = N.load()
    ins = [_in(a, n, nm) for a, nm in ((px, "px"), (py, "py"), (pz, "pz"), (pcb, "pcb"))]
    out = _out(output, 4 * n, "output")
    N.check(L.pf_get_particles(*(N.dptr(a) for a in ins), N.dptr(out), n))
