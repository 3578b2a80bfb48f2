"""Run the reference's own device-resident particle-filter module
(_gnss_gpu_pf_device, built from src/particle_filter/pf_device.cu and
python/gnss_gpu/_pf_device_bindings.cpp, installed unmodified into
baseline/_ref) on seeded particle sets and record the log-weights (and, for
Doppler, the velocity states) each likelihood produces, so the CPU oracle's
restatements of those likelihoods can be pinned to the reference itself.

Needs a GPU and the reference install:  python tests/golden/make_ref_device_fixtures.py
Writes tests/golden/ref_device_fixtures.npz.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "baseline" / "_ref"))

N_PART = 512
WL_L1 = 0.190293673
SEED = 20261204


def main():
    import gnss_gpu._gnss_gpu_pf_device as R  # the reference's module
    fx = json.loads((HERE / "tokyo_fixture.json").read_text())
    sat = np.array(fx["sat_ecef"], np.float64).reshape(-1, 3)
    S = len(sat)
    tp = np.array(fx["true_pos"], np.float64)
    tcb = float(fx["true_cb"])
    rng = np.random.default_rng(SEED)

    pos = tp[None, :] + rng.normal(0.0, 20.0, (N_PART, 3))
    cb = tcb + rng.normal(0.0, 30.0, N_PART)
    vel = rng.normal(0.0, 2.0, (N_PART, 3))
    vcov = np.tile(np.diag([1.5, 1.0, 0.5]).ravel(), (N_PART, 1))
    states = np.concatenate([pos, cb[:, None], vel, vcov], axis=1)  # (N, 16)

    rng_true = np.linalg.norm(sat - tp[None, :], axis=1)
    pr = rng_true + tcb + rng.normal(0.0, 3.0, S)
    pr[[2, 5]] += [40.0, 65.0]  # two NLOS-like outliers for the gate and the robust costs
    w = rng.uniform(0.5, 2.0, S)

    def run(fn):
        st = R.pf_device_create(N_PART)
        R.pf_device_set_particle_states(st, states)
        fn(st)
        lw = np.empty(N_PART)
        R.pf_device_get_log_weights(st, lw)
        out = R.pf_device_get_particle_states(st).copy()
        R.pf_device_destroy(st)
        return lw, out

    rec = {"states": states, "sat": sat, "pr": pr, "w": w}
    flat = sat.ravel().copy()
    cases = {
        "gauss": dict(nu=0.0, thr=0.0, hub=False, k=1.5),
        "student_t": dict(nu=4.0, thr=0.0, hub=False, k=1.5),
        "huber": dict(nu=0.0, thr=0.0, hub=True, k=1.5),
        "gate": dict(nu=0.0, thr=15.0, hub=False, k=1.5),
    }
    for name, c in cases.items():
        rec[f"lw_{name}"], _ = run(lambda st, c=c: R.pf_device_weight(st, flat, pr, w, S, 5.0, c["nu"], c["thr"],
                                                                      c["hub"], c["k"]))
    rec["lw_gmm"], _ = run(lambda st: R.pf_device_weight_gmm(st, flat, pr, w, S, 5.0, 0.7, 15.0, 30.0))

    # carrier phase (cycles): range + clock over the wavelength, noise, integer ambiguities
    cp = (rng_true + tcb) / WL_L1 + rng.normal(0.0, 0.03, S) + rng.integers(-1000, 1000, S)
    rec["cp"] = cp
    rec["lw_carrier_afv"], _ = run(lambda st: R.pf_device_weight_carrier_afv(st, flat, cp, w, S, WL_L1, 0.05))

    # double differences against satellite 0 with a base station 800 m away
    base = tp + np.array([500.0, -400.0, 480.0])
    b = np.linalg.norm(sat - base[None, :], axis=1)
    k_idx = np.arange(1, S)
    sat_k = sat[k_idx].ravel().copy()
    ref = np.repeat(sat[[0]], len(k_idx), axis=0).ravel().copy()
    base_k, base_ref = b[k_idx].copy(), np.repeat(b[0], len(k_idx))
    dd = (rng_true[k_idx] - rng_true[0]) - (base_k - base_ref) + rng.normal(0.0, 1.0, len(k_idx))
    dd[2] += 30.0
    wdd = rng.uniform(0.5, 2.0, len(k_idx))
    rec.update(dd_sat_k=sat_k, dd_ref=ref, dd_base_k=base_k, dd_base_ref=base_ref, dd=dd, w_dd=wdd)
    nd = len(k_idx)
    rec["lw_dd_pr"], _ = run(lambda st: R.pf_device_weight_dd_pseudorange(st, sat_k, ref, dd, base_k, base_ref, wdd,
                                                                          nd, 2.0, 0.0, False, 1.5))
    rec["lw_dd_pr_gate_huber"], _ = run(lambda st: R.pf_device_weight_dd_pseudorange(
        st, sat_k, ref, dd, base_k, base_ref, wdd, nd, 2.0, 10.0, True, 1.5))
    wl = np.full(nd, WL_L1)
    ddc = dd / WL_L1 + rng.integers(-50, 50, nd)
    rec.update(ddc=ddc, dd_wl=wl)
    rec["lw_dd_carrier"], _ = run(lambda st: R.pf_device_weight_dd_carrier_afv(
        st, sat_k, ref, ddc, base_k, base_ref, wdd, wl, nd, 0.05, 0.0, False, 1.5))
    rec["lw_dd_carrier_gate_huber"], _ = run(lambda st: R.pf_device_weight_dd_carrier_afv(
        st, sat_k, ref, ddc, base_k, base_ref, wdd, wl, nd, 0.05, 0.3, True, 1.5))

    # Doppler: satellite velocities, range rates from the true receiver velocity
    sat_vel = rng.normal(0.0, 2500.0, (S, 3))
    v_true = np.array([3.0, -1.0, 0.2])
    los = (sat - tp[None, :]) / rng_true[:, None]
    rr = np.sum((sat_vel - v_true[None, :]) * los, axis=1) + 0.7  # + clock drift (m/s)
    dop = -(rr + rng.normal(0.0, 0.2, S)) / WL_L1
    rec.update(sat_vel=sat_vel, doppler_hz=dop)
    rec["lw_doppler"], rec["states_doppler"] = run(lambda st: R.pf_device_weight_doppler(
        st, flat, sat_vel.ravel().copy(), dop, w, S, WL_L1, 0.5, 0.25, 10.0))
    rec["lw_doppler_kf"], rec["states_doppler_kf"] = run(lambda st: R.pf_device_doppler_kf_update(
        st, flat, sat_vel.ravel().copy(), dop, w, S, WL_L1, 0.5))

    np.savez_compressed(HERE / "ref_device_fixtures.npz", **rec)
    print("wrote", HERE / "ref_device_fixtures.npz", {k: np.asarray(v).shape for k, v in rec.items()})


if __name__ == "__main__":
    main()
