"""Shared helpers of the GPU parity tests: run one engine step and compare
every output with the FP64 oracle on the same inputs."""
from __future__ import annotations

import numpy as np

from gnss_gpu_b200 import _native as N
from gnss_gpu_b200.engine import Engine, EngineOptions, FilterSpec
from oracle import oracle as O

# Tolerances against the FP64 oracle (north-star precision gates):
#   state after predict: |dx| <= 1e-6 * max(1, |x|)  (FP32 storage of the offsets)
#   log-weights:         |dlw| <= 1e-5 * max(1, |lw|) (1e-5 relative; below one
#                        nat an absolute 1e-5, i.e. 1e-5 relative in the weight)
#   estimate:            <= 1 mm (0.001 m) in ECEF and in the clocks
#   ESS:                 1e-5 relative
STATE_RTOL = 1e-6
LW_RTOL = 1e-5
EST_TOL_M = 1e-3
ESS_RTOL = 1e-5


def lw_close(got, want, rtol=LW_RTOL):
    err = np.abs(np.asarray(got, np.float64) - np.asarray(want, np.float64))
    lim = rtol * np.maximum(1.0, np.abs(want))
    return err <= lim, err / np.maximum(1.0, np.abs(want))


def make_engine(ns, n_clk=1, resampler="systematic", iters=32, seeds=None, sigma_pos=(1.0, 1.0, 0.5),
                sigma_clk=0.5, sigma_pr=3.0, ess=0.5, sys_offset="random", weight_mode="gaussian",
                lw_mode="overwrite", recenter=True, max_sats=64, obs_slots=1, chain=False):
    seeds = seeds if seeds is not None else [1000 + k for k in range(len(ns))]
    specs = [FilterSpec(n_particles=int(n), seed=int(seeds[k]), sigma_pos=sigma_pos, sigma_clk=sigma_clk,
                        sigma_pr=sigma_pr) for k, n in enumerate(ns)]
    opts = EngineOptions(n_clk=n_clk, resampler=resampler, megopolis_iters=iters, ess_threshold=ess,
                         sys_offset=sys_offset, weight_mode=weight_mode, lw_mode=lw_mode, recenter=recenter,
                         max_sats=max_sats, obs_slots=obs_slots, kernel_chain=chain)
    return Engine(specs, opts)


def sat_rows(sats, pr, w=None):
    w = np.ones(len(pr)) if w is None else np.asarray(w, np.float64)
    return np.column_stack([np.asarray(sats, np.float64), np.asarray(pr, np.float64), w])


def check_step(eng: Engine, k: int, before_state, before_shift, rec, weight_mode=0, huber_k=1.5,
               accumulate_base=None, check_resample=True):
    """Compare filter k's last step with the oracle.  before_state: the
    gathered state read before the step; before_shift: pending shift then."""
    spec = eng.filters[k]
    D = eng.D
    rot, _ = eng.frame(k)
    anchor_new, clk_new, _ = eng.anchor(k)
    x_raw, lw_raw = eng.state_f32(k, raw=True)
    res = eng.results()[k]
    epoch = res["epoch"] - 1
    fl = int(rec.get("flags", N.PF_EP_PREDICT | N.PF_EP_WEIGHT))
    sigma = np.zeros(D, np.float32)
    sigma[:3] = np.asarray(spec.sigma_pos, np.float32)
    sigma[3:] = np.float32(spec.sigma_clk)
    x_pred = O.predict(before_state.astype(np.float64), None, np.asarray(rec.get("disp", (0, 0, 0))),
                       before_shift.astype(np.float64), sigma, fl & N.PF_EP_PREDICT, spec.seed, epoch, k)
    dx = np.abs(x_raw.astype(np.float64) - x_pred)
    # FP32 storage of the offsets plus FP32 Box-Muller noise (~1e-6 of sigma
    # per normal, scaled with the draw's magnitude)
    noise = 2e-6 * sigma.astype(np.float64)[:, None] * 6.0 if fl & N.PF_EP_PREDICT else 0.0
    state_ok = np.all(dx <= STATE_RTOL * np.maximum(1.0, np.abs(x_pred)) + 2e-6 + noise)
    out = {"state_err": float(dx.max()) if dx.size else 0.0, "state_ok": bool(state_ok)}
    if fl & N.PF_EP_WEIGHT:
        rows = sat_rows(rec["sats"], rec["pr"], rec.get("w"))
        clk = np.asarray(rec.get("clk", np.zeros(len(rows))), np.int32)
        lw_o = O.weight(x_raw, anchor_new, clk_new, rot, rows, clk, spec.sigma_pr, mode=weight_mode,
                        huber_k=huber_k, lw_base=accumulate_base)
        ok, rel = lw_close(lw_raw, lw_o)
        out["lw_ok"] = bool(ok.all())
        out["lw_rel_err"] = float(rel.max())
        st = O.stats(x_raw, lw_raw.astype(np.float64), anchor_new, clk_new, rot)
        out["est_err_m"] = float(np.max(np.abs(st["est_ecef"] - res["est_ecef"])))
        out["clk_err_m"] = float(np.max(np.abs(st["est_clk"] - res["est_clk"]))) if D > 3 else 0.0
        out["ess_rel_err"] = abs(st["ess"] - res["ess"]) / st["ess"]
        out["max_lw_equal"] = bool(np.float32(lw_raw.max()) == np.float32(res["max_lw"]))
        out["resampled"] = res["resampled"]
        if check_resample and res["resampled"] and eng.cfg.resampler == N.PF_RESAMPLE_SYSTEMATIC:
            u, W, M = eng.resample_info(k)
            anc_o, W_o = O.systematic_tiled(lw_raw, u)
            anc_g = eng.ancestors(k)
            out["anc_equal"] = bool(np.array_equal(anc_o, anc_g))
            out["wq_equal"] = W == W_o
    return out
