"""The learned mixture likelihood (weight mode "mixture") on the GPU:
features and network outputs computed inside the epoch kernel against the
host features and the FP64 network oracle, log-weights against the FP64
mixture oracle, and what the trained network gains over the plain robust
filter on simulated box cities."""
import numpy as np
import pytest

from gnss_gpu_b200 import _native as N
from gnss_gpu_b200 import citysim as CS
from gnss_gpu_b200 import learned as LR
from gnss_gpu_b200.engine import Engine, EngineOptions, FilterSpec
from oracle import mlp_oracle as M
from oracle import oracle as O

import pfhelp as H

pytestmark = pytest.mark.gpu


def _run_mixture(n=4096, epochs=4, seed=3, params=None):
    city = CS.make_city(11)
    tr = CS.drive(city, epochs + 1, seed=seed)
    eng = Engine([FilterSpec(n_particles=n, seed=9, sigma_pos=(1.0, 1.0, 0.5), sigma_clk=1.0, sigma_pr=3.0)],
                 EngineOptions(n_clk=1, weight_mode="mixture", huber_k=1.5, max_sats=24, obs_slots=1))
    prm = M.init_params(5) if params is None else params
    eng.set_mlp(prm)
    start = tr.truth_ecef[0] - tr.disp_enu[0] @ tr.rot
    eng.initialize(0, start, tr.truth_clk[0], 5.0, 10.0)
    prior = (start + tr.disp_enu[0] @ tr.rot, float(tr.truth_clk[0][0]))
    out = []
    for t in range(epochs):
        e, res, blk = LR.prior_geometry(tr, t, *prior)
        before, _ = eng.state_f32(0)
        _, _, shift = eng.anchor(0)
        rec = LR.epoch_record(tr, t, blk)
        fe, sv = eng.pack_epoch([rec])
        eng.upload(0, fe, sv)
        eng.step()
        out.append(dict(t=t, prior=prior, e=e, res=res, blk=blk, rec=rec, before=before, shift=shift,
                        dbg=eng.sat_debug(0), x=eng.state_f32(0, raw=True), anchor=eng.anchor(0),
                        result=eng.results()[0]))
        r = eng.results()[0]
        prior = (r["est_ecef"] + tr.disp_enu[t + 1] @ tr.rot, float(r["est_clk"][0]))
    return eng, tr, prm, out


def test_kernel_features_and_outputs_match_host_and_oracle():
    eng, tr, prm, out = _run_mixture()
    for o in out:
        Xh, fb = LR.features(o["e"], o["res"], tr.cn0[o["t"]], o["blk"])
        d = o["dbg"]
        assert d.shape == (len(Xh), 16)
        assert np.max(np.abs(d[:, :12] - Xh)) < 2e-3, np.max(np.abs(d[:, :12] - Xh))
        assert np.max(np.abs(d[:, 15] - o["res"])) < 1e-2
        assert np.array_equal(d[:, 14] > 0.5, fb)
        p, mu = M.predict(prm, d[:, :12].astype(np.float64))
        assert np.max(np.abs(d[:, 12] - np.clip(p, 1e-4, 1 - 1e-4))) < 2e-3
        assert np.max(np.abs(d[:, 13] - mu) / np.maximum(1.0, mu)) < 2e-3
    eng.close()


def test_mixture_log_weights_match_oracle():
    eng, tr, prm, out = _run_mixture(n=5000, epochs=3)
    rot, _ = eng.frame(0)
    for o in out:
        x_raw, lw_raw = o["x"]
        anchor, clk, _ = o["anchor"]
        d = o["dbg"]
        rows = H.sat_rows(o["rec"]["sats"], o["rec"]["pr"])
        lw_o = O.weight_mixture(x_raw, anchor, clk, rot, rows, 3.0, d[:, 12].astype(np.float64),
                                d[:, 13].astype(np.float64), d[:, 14], huber_k=1.5)
        ok, rel = H.lw_close(lw_raw, lw_o)
        assert ok.all(), float(rel.max())
    eng.close()


def test_mixture_requires_network_and_epoch_path():
    with pytest.raises(ValueError):
        Engine([FilterSpec(n_particles=100, seed=1)],
               EngineOptions(n_clk=1, weight_mode="mixture", kernel_chain=True))
    eng = Engine([FilterSpec(n_particles=100, seed=1)], EngineOptions(n_clk=1, weight_mode="mixture"))
    tr = CS.drive(CS.make_city(1), 2, seed=1)
    eng.initialize(0, tr.truth_ecef[0], tr.truth_clk[0], 5.0, 10.0)
    fe, sv = eng.pack_epoch([LR.epoch_record(tr, 0, np.zeros(len(tr.pr[0]), np.float32))])
    eng.upload(0, fe, sv)
    with pytest.raises(N.PFError):
        eng.step()
    eng.close()


def test_trained_network_beats_plain_robust_filter():
    """Train on simulated cities (prior means from the plain filter), then
    compare horizontal errors on held-out trajectories in other cities."""
    tr_train = LR.make_trajectories(24, 200, seed=21)
    r = LR.run_filters(tr_train, 8000, "huber", seed=1, keep_priors=True)
    X, Y = LR.training_set(tr_train, r.priors)
    params, losses = LR.train(X, Y, steps=1200, batch=8192, lr=2e-3, seed=4)
    assert losses[-1] < 0.5 * losses[0]
    tr_eval = LR.make_trajectories(8, 200, seed=22)
    plain = LR.run_filters(tr_eval, 10_000, "huber", seed=5).err2d[:, 10:]
    learned = LR.run_filters(tr_eval, 10_000, "mixture", params=params, seed=5).err2d[:, 10:]
    p50_plain, p50_learned = np.median(plain), np.median(learned)
    assert p50_learned < 0.8 * p50_plain, (p50_plain, p50_learned)
    assert np.sqrt(np.mean(learned ** 2)) < np.sqrt(np.mean(plain ** 2))


def test_city_los_device_equals_host():
    """pf_city_los restates the simulator's box-city DDA with the same FP64
    rounding: flags equal to the host's, ray for ray, including rays along
    the grid axes, from inside buildings and from outside the grid."""
    from gnss_gpu_b200 import citysim as CS

    rng = np.random.default_rng(8)
    total = 0
    for seed in (1, 2, 3):
        city = CS.make_city(seed)
        m = 20_000
        p = np.column_stack([rng.uniform(-200.0, city.size + 200.0, m), rng.uniform(-200.0, city.size + 200.0, m),
                             rng.uniform(0.0, 40.0, m)])
        az = rng.uniform(0.0, 2 * np.pi, m)
        el = rng.uniform(np.radians(2.0), np.radians(89.0), m)
        az[:200] = rng.choice([0.0, np.pi / 2, np.pi, 3 * np.pi / 2], 200)  # along the grid axes
        host = CS.los_blocked(city, p, az, el)
        dev = CS.los_blocked_device(city, p, az, el)
        assert np.array_equal(host, dev), int(np.sum(host != dev))
        total += int(host.sum())
    assert total > 1000  # the cases exercise blocked rays


def test_mixture_batched_uneven_filters_match_oracle():
    """Several filters of uneven size (one tile shared by none of them, ragged
    tails, 3 to 70,001 particles) and different cities and satellite counts
    in one engine: every filter's in-kernel network outputs and log-weights
    match the FP64 oracles, as for a single filter."""
    ns = [3, 1500, 4096, 9000, 70_001]
    prm = M.init_params(6)
    specs = [FilterSpec(n_particles=n, seed=40 + k, sigma_pos=(1.0, 1.0, 0.5), sigma_clk=1.0, sigma_pr=3.0)
             for k, n in enumerate(ns)]
    eng = Engine(specs, EngineOptions(n_clk=1, weight_mode="mixture", huber_k=1.5, max_sats=40, obs_slots=1))
    eng.set_mlp(prm)
    trs, priors = [], []
    for k, n in enumerate(ns):
        tr = CS.drive(CS.make_city(30 + k), 4, seed=50 + k, n_sat=[6, 12, 24, 33, 40][k])
        start = tr.truth_ecef[0] - tr.disp_enu[0] @ tr.rot
        eng.initialize(k, start, tr.truth_clk[0], 5.0, 10.0)
        trs.append(tr)
        priors.append((start + tr.disp_enu[0] @ tr.rot, float(tr.truth_clk[0][0])))
    for t in range(2):
        recs = []
        for k, tr in enumerate(trs):
            _, _, blk = LR.prior_geometry(tr, t, *priors[k])
            recs.append(LR.epoch_record(tr, t, blk))
        fe, sv = eng.pack_epoch(recs)
        eng.upload(0, fe, sv)
        eng.step()
        for k, tr in enumerate(trs):
            rot, _ = eng.frame(k)
            x_raw, lw_raw = eng.state_f32(k, raw=True)
            anchor, clk, _ = eng.anchor(k)
            d = eng.sat_debug(k)
            p, mu = M.predict(prm, d[:, :12].astype(np.float64))
            assert np.max(np.abs(d[:, 12] - np.clip(p, 1e-4, 1 - 1e-4))) < 2e-3
            rows = H.sat_rows(recs[k]["sats"], recs[k]["pr"])
            lw_o = O.weight_mixture(x_raw, anchor, clk, rot, rows, 3.0, d[:, 12].astype(np.float64),
                                    d[:, 13].astype(np.float64), d[:, 14], huber_k=1.5)
            ok, rel = H.lw_close(lw_raw, lw_o)
            assert ok.all(), (k, float(rel.max()))
            r = eng.results()[k]
            priors[k] = (r["est_ecef"] + tr.disp_enu[t + 1] @ tr.rot, float(r["est_clk"][0]))
    eng.close()
