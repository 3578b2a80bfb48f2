"""Learned NLOS likelihood: training set, training and evaluation.

The network (pf_mlp.cuh) maps 12 per-satellite features to the NLOS
probability and NLOS bias mean that parameterise the mixture likelihood of
the epoch kernel (weight mode "mixture").  Everything numerical runs in the
library's kernels: the plain particle filter that provides the prior means
of the training set, the BF16 tensor-core forward/backward/Adam kernels of
the training, and the filters being compared.  This module only drives them
and computes the features on the host exactly as the kernel does
(pf_learned.cuh):

    f0 = sin el, f1 = cos el, f2 = sin az, f3 = cos az, f4 = (C/N0 - 40)/10,
    f5 = clamp(rc/20, -8, 8), f6 = min(|rc|/20, 8), f7 = blocked,
    f8 = n_sat/40, f9 = min(median|rc|/20, 8), f10 = blocked fraction,
    f11 = (C/N0 - mean C/N0)/10,

with r = pr - |s - prior| - prior clock, rc = r - median r (per clock
group) and the ray-traced `blocked` flag taken at the prior mean.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from . import citysim as CS
from .engine import Engine, EngineOptions, FilterSpec

FEAT = 12
SIGMA_PR = 3.0
HUBER_K = 1.5


def lower_median(v: np.ndarray, axis=-1):
    """Element of rank (m - 1) // 2 in ascending order (the kernel's median)."""
    s = np.sort(v, axis=axis)
    m = v.shape[axis]
    return np.take(s, (m - 1) // 2, axis=axis)


def features(e_enu: np.ndarray, res: np.ndarray, cn0: np.ndarray, blocked: np.ndarray):
    """Features of one filter-epoch (one clock group): e_enu (S, 3) unit
    lines of sight at the prior, res (S,) residuals against the prior.
    Returns (X (S, 12) float32, fallback (S,) bool)."""
    S = len(res)
    rc = res - lower_median(res) if S else res
    arc = np.abs(rc)
    med_arc = lower_median(arc) if S else 0.0
    ch = np.sqrt(e_enu[:, 0] ** 2 + e_enu[:, 1] ** 2)
    inv = np.where(ch > 0, 1.0 / np.maximum(ch, 1e-300), 0.0)
    X = np.zeros((S, FEAT), np.float64)
    X[:, 0] = e_enu[:, 2]
    X[:, 1] = ch
    X[:, 2] = e_enu[:, 0] * inv
    X[:, 3] = e_enu[:, 1] * inv
    X[:, 4] = (cn0 - 40.0) * 0.1
    X[:, 5] = np.clip(rc / 20.0, -8.0, 8.0)
    X[:, 6] = np.minimum(arc / 20.0, 8.0)
    X[:, 7] = blocked
    X[:, 8] = S / 40.0
    X[:, 9] = min(med_arc / 20.0, 8.0)
    X[:, 10] = np.mean(blocked) if S else 0.0
    X[:, 11] = (cn0 - (np.mean(cn0) if S else 0.0)) * 0.1
    fallback = ~((cn0 >= 10.0) & (cn0 <= 70.0)) | ~(arc <= 150.0) | (S < 4)
    return X.astype(np.float32), fallback


def prior_geometry(tr: CS.CityTrajectory, t: int, prior_ecef: np.ndarray, prior_clk: float):
    """Lines of sight (ENU), residuals, azimuth/elevation and the ray-traced
    blocked flag of epoch t's satellites at a prior mean."""
    sats = tr.sats[t]
    v = sats - prior_ecef
    rng = np.linalg.norm(v, axis=1)
    u = v / rng[:, None]
    e = u @ tr.rot.T
    res = tr.pr[t] - rng - prior_clk
    az = np.mod(np.arctan2(e[:, 0], e[:, 1]), 2 * np.pi)
    el = np.arcsin(np.clip(e[:, 2], -1.0, 1.0))
    p_enu = (prior_ecef - tr.anchor) @ tr.rot.T
    p_enu = np.array([p_enu[0], p_enu[1], CS.RX_HEIGHT])
    blk = CS.los_blocked_device(tr.city, np.repeat(p_enu[None], len(sats), 0), az, el).astype(np.float32)
    return e, res, blk


def epoch_record(tr: CS.CityTrajectory, t: int, blocked: np.ndarray):
    return {"disp": tr.disp_enu[t], "sats": tr.sats[t], "pr": tr.pr[t], "cn0": tr.cn0[t], "blocked": blocked,
            "flags": N.PF_EP_PREDICT | N.PF_EP_WEIGHT}


@dataclass
class RunResult:
    err2d: np.ndarray          # (F, E) horizontal error of the fused estimate, m
    priors: list               # per filter, per epoch (prior ECEF, prior clock)
    steps_per_s: float         # particle-steps/s of the device steps (event-timed)
    h2d_bytes: float = 0.0     # mean host-to-device bytes per epoch (rays, records, satellites)
    d2h_bytes: float = 0.0     # mean device-to-host bytes per epoch (blocked flags, results)


def prior_geometry_many(trajs, t: int, priors):
    """prior_geometry for many filters at once: per city, the satellites of
    all its filters in one set of array operations and one device ray
    trace."""
    out = [None] * len(trajs)
    by_city = {}
    for k, tr in enumerate(trajs):
        by_city.setdefault(id(tr.city), []).append(k)
    for ks in by_city.values():
        city = trajs[ks[0]].city
        counts = [len(trajs[k].sats[t]) for k in ks]
        sats = np.concatenate([trajs[k].sats[t] for k in ks])
        pe = np.repeat(np.stack([priors[k][0] for k in ks]), counts, axis=0)
        pc = np.repeat(np.array([priors[k][1] for k in ks], np.float64), counts)
        rot = np.repeat(np.stack([trajs[k].rot for k in ks]), counts, axis=0)
        anchor = np.repeat(np.stack([trajs[k].anchor for k in ks]), counts, axis=0)
        pr = np.concatenate([trajs[k].pr[t] for k in ks])
        v = sats - pe
        rng = np.linalg.norm(v, axis=1)
        e = np.einsum("nij,nj->ni", rot, v / rng[:, None])
        res = pr - rng - pc
        p_enu = np.einsum("nij,nj->ni", rot, pe - anchor)
        p_enu[:, 2] = CS.RX_HEIGHT
        az = np.mod(np.arctan2(e[:, 0], e[:, 1]), 2 * np.pi)
        el = np.arcsin(np.clip(e[:, 2], -1.0, 1.0))
        blk = CS.los_blocked_device(city, p_enu, az, el).astype(np.float32)
        o = 0
        for k, m in zip(ks, counts):
            out[k] = (e[o:o + m], res[o:o + m], blk[o:o + m])
            o += m
    return out


def run_filters(trajs, n_particles, mode: str, params=None, seed: int = 0, keep_priors: bool = False,
                init_spread=(5.0, 10.0), max_sats=None) -> RunResult:
    """Run one filter per trajectory through all epochs on the GPU engine
    (batched, one launch per epoch); the prior of epoch t is the estimate of
    epoch t-1 moved by the known displacement.  n_particles: one count or
    one per trajectory."""
    F, E = len(trajs), len(trajs[0].pr)
    counts = [int(n_particles)] * F if np.isscalar(n_particles) else [int(n) for n in n_particles]
    specs = [FilterSpec(n_particles=counts[k], seed=seed * 1000 + k, sigma_pos=(1.0, 1.0, 0.5), sigma_clk=1.0,
                        sigma_pr=SIGMA_PR) for k in range(F)]
    ms = max_sats or max(len(s) for tr in trajs for s in tr.sats)
    opts = EngineOptions(n_clk=1, resampler="systematic", weight_mode=mode, huber_k=HUBER_K,
                         max_sats=ms, obs_slots=1)
    eng = Engine(specs, opts)
    if mode == "mixture":
        eng.set_mlp(params)
    rng = np.random.default_rng(seed)
    prior = []
    for k, tr in enumerate(trajs):
        start = tr.truth_ecef[0] - tr.disp_enu[0] @ tr.rot + rng.normal(0, 2.0, 3)
        eng.initialize(k, start, tr.truth_clk[0] + rng.normal(0, 5.0, 1), *init_spread)
        prior.append((start + tr.disp_enu[0] @ tr.rot, float(tr.truth_clk[0][0])))
    err = np.zeros((F, E))
    priors = [[] for _ in range(F)]
    h2d = d2h = 0
    rots = np.stack([tr.rot for tr in trajs])
    eng.enable_timing(E + 1)
    for t in range(E):
        geo = prior_geometry_many(trajs, t, prior)
        recs = []
        for k, tr in enumerate(trajs):
            recs.append(epoch_record(tr, t, geo[k][2]))
            if keep_priors:
                priors[k].append((prior[k][0].copy(), prior[k][1]))
        fe, sv = eng.pack_epoch(recs)
        eng.upload(0, fe, sv)
        eng.step()
        res = eng.results_array()
        # one ray per satellite (origin + direction, FP64) up and a flag back
        h2d += fe.nbytes + sv.nbytes + 48 * len(sv)
        d2h += eng.result_bytes() + len(sv)
        est = res["est_ecef"]
        d = np.einsum("kij,kj->ki", rots, est - np.stack([tr.truth_ecef[t] for tr in trajs]))
        err[:, t] = np.hypot(d[:, 0], d[:, 1])
        nxt = min(t + 1, E - 1)
        moved = est + np.einsum("kj,kji->ki", np.stack([tr.disp_enu[nxt] for tr in trajs]), rots)
        prior = [(moved[k], float(res["est_clk"][k, 0])) for k in range(F)]
    _, whole = eng.read_timing()
    eng.close()
    sps = float(np.sum(counts)) * len(whole) / max(float(np.sum(whole)) / 1e3, 1e-12)
    return RunResult(err, priors, sps, h2d / E, d2h / E)


def training_set(trajs, priors):
    """Features and labels (nlos, bias) of every in-range satellite-epoch."""
    Xs, Ys = [], []
    for tr, pk in zip(trajs, priors):
        for t, (pe, pc) in enumerate(pk):
            e, res, blk = prior_geometry(tr, t, pe, pc)
            X, fb = features(e, res, tr.cn0[t], blk)
            keep = ~fb
            Xs.append(X[keep])
            Ys.append(np.column_stack([tr.nlos[t][keep], tr.bias[t][keep]]).astype(np.float32))
    return np.concatenate(Xs), np.concatenate(Ys)


def make_trajectories(n: int, n_epochs: int, seed: int, cities: int = 8, n_sat: int = 24, sat_range=None):
    """n drives spread over `cities` box cities (seeded)."""
    out = []
    for c in range(cities):
        m = len(range(c, n, cities))
        if m:
            out.extend(CS.drive_many(CS.make_city(seed * 1000 + c), m, n_epochs, seed=seed * 100_003 + c,
                                     n_sat=n_sat, sat_range=sat_range))
    return out


def train(X: np.ndarray, Y: np.ndarray, steps: int = 3000, batch: int = 8192, lr: float = 2e-3, seed: int = 0,
          params=None):
    """Adam on the GPU (pf_mlp_adam_step over mini-batches of a host-shuffled
    copy of the set, reshuffled every pass); returns (params, losses every
    100 steps)."""
    import torch
    L = N.load()
    rng = np.random.default_rng(seed)
    n = len(X)
    batch = min(batch, n)
    prm = torch.as_tensor(init_params(seed) if params is None else np.asarray(params, np.float32), device="cuda")
    m = torch.zeros_like(prm)
    v = torch.zeros_like(prm)
    loss = torch.zeros(1, device="cuda")
    scratch = torch.zeros(L.pf_mlp_scratch_bytes(), dtype=torch.uint8, device="cuda")
    dX = torch.empty((n, FEAT), dtype=torch.float32, device="cuda")
    dY = torch.empty((n, 2), dtype=torch.float32, device="cuda")
    per_pass = max(1, n // batch)
    losses = []
    for step in range(1, steps + 1):
        j = (step - 1) % per_pass
        if j == 0:
            perm = rng.permutation(n)
            dX.copy_(torch.as_tensor(np.ascontiguousarray(X[perm], np.float32)))
            dY.copy_(torch.as_tensor(np.ascontiguousarray(Y[perm], np.float32)))
        off = j * batch
        N.check(L.pf_mlp_adam_step(dX.data_ptr() + off * FEAT * 4, dY.data_ptr() + off * 2 * 4, batch,
                                   prm.data_ptr(), m.data_ptr(), v.data_ptr(), step, C.c_float(lr),
                                   loss.data_ptr(), scratch.data_ptr(), scratch.numel(), None))
        if step % 100 == 0 or step == 1:
            torch.cuda.synchronize()
            losses.append(float(loss.item()))
    torch.cuda.synchronize()
    return prm.cpu().numpy(), losses


def predict(params, X: np.ndarray):
    """(p_nlos, mu) per row from the tensor-core forward kernel."""
    import torch
    L = N.load()
    dX = torch.as_tensor(np.ascontiguousarray(X, np.float32), device="cuda")
    dp = torch.as_tensor(np.ascontiguousarray(params, np.float32), device="cuda")
    out = torch.empty(2 * len(X), dtype=torch.float32, device="cuda")
    N.check(L.pf_mlp_forward(dX.data_ptr(), len(X), dp.data_ptr(), out.data_ptr(), None))
    torch.cuda.synchronize()
    o = out.cpu().numpy().reshape(-1, 2)
    return o[:, 0], o[:, 1]


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initial parameters in the library's layout (FP32)."""
    H, IN = 64, 16
    rng = np.random.default_rng(seed)
    p = np.zeros(N.load().pf_mlp_param_count(), np.float32)
    o_b1 = H * IN
    o_w2 = o_b1 + H
    o_b2 = o_w2 + H * H
    o_w3 = o_b2 + H
    o_b3 = o_w3 + 2 * H
    p[:o_b1] = (rng.normal(0, np.sqrt(2.0 / FEAT), (H, IN)) * (np.arange(IN) < FEAT)).ravel()
    p[o_w2:o_b2] = rng.normal(0, np.sqrt(2.0 / H), H * H)
    p[o_w3:o_b3] = rng.normal(0, np.sqrt(1.0 / H), 2 * H)
    p[o_b3:o_b3 + 2] = [-1.0, 0.0]
    return p
