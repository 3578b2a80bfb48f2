"""GPU parity of the resident engine against the FP64 oracle (calls go
through the C ABI of libgnsspf_b200.so)."""
import numpy as np
import pytest

from gnss_gpu_b200 import _native as N
from gnss_gpu_b200 import scenario as S
from oracle import oracle as O

import pfhelp as H

pytestmark = pytest.mark.gpu


def _epoch_rec(tr, t, flags=N.PF_EP_PREDICT | N.PF_EP_WEIGHT, nclk=1):
    clk = tr.clk_idx[t] if nclk > 1 else np.zeros(len(tr.pr[t]), np.int32)
    return {"disp": tr.disp_enu[t], "sats": tr.sats[t], "pr": tr.pr[t], "clk": clk, "flags": flags}


def _run_and_check(eng, tr, epochs, nclk=1, flags=N.PF_EP_PREDICT | N.PF_EP_WEIGHT, k=0, wmode=0):
    outs = []
    for t in range(epochs):
        before, _ = eng.state_f32(k)
        _, _, shift = eng.anchor(k)
        rec = _epoch_rec(tr, t, flags, nclk)
        fe, sv = eng.pack_epoch([rec])
        eng.upload(0, fe, sv)
        eng.step()
        outs.append(H.check_step(eng, k, before, shift, rec, weight_mode=wmode))
    return outs


@pytest.mark.parametrize("nclk", [1, 4])
def test_init_matches_oracle(nclk):
    tr = S.config1(n_epochs=1) if nclk == 4 else S.config0()
    eng = H.make_engine([5000], n_clk=nclk)
    eng.initialize(0, tr.anchor, tr.truth_clk[0], 10.0, 30.0)
    x, lw = eng.state_f32(0)
    xo = O.init_state(5000, 3 + nclk, 10.0, 30.0, eng.filters[0].seed, 0)
    # FP32 storage (1e-6 relative) + FP32 Box-Muller (~1e-6 of the spread)
    spread = np.array([10.0] * 3 + [30.0] * nclk)[:, None]
    assert np.all(np.abs(x - xo) <= 1e-6 * np.abs(xo) + 2e-6 * spread * (1 + np.abs(xo) / spread) + 1e-6)
    assert np.all(lw == 0)
    assert eng.ess(0) == pytest.approx(5000)


@pytest.mark.parametrize("nclk,n", [(1, 10_000), (4, 20_000), (1, 1), (1, 5), (1, 1023), (1, 1025), (4, 3077)])
def test_step_parity_systematic(nclk, n):
    tr = S.config1(n_epochs=6) if nclk == 4 else S.config0()
    eng = H.make_engine([n], n_clk=nclk, sigma_clk=0.5)
    eng.initialize(0, tr.anchor, tr.truth_clk[0], 10.0, 30.0)
    outs = _run_and_check(eng, tr, 5, nclk)
    for o in outs:
        assert o["state_ok"], o
        assert o["lw_ok"], o
        assert o["est_err_m"] <= H.EST_TOL_M, o
        assert o["clk_err_m"] <= H.EST_TOL_M, o
        assert o["ess_rel_err"] <= H.ESS_RTOL, o
        assert o["max_lw_equal"], o
        if o["resampled"]:
            assert o["anc_equal"] and o["wq_equal"], o


def test_forced_resample_every_epoch_bit_exact_ancestors():
    tr = S.config1(n_epochs=8)
    eng = H.make_engine([50_000], n_clk=4)
    eng.initialize(0, tr.anchor, tr.truth_clk[0], 10.0, 30.0)
    outs = _run_and_check(eng, tr, 6, 4, flags=N.PF_EP_PREDICT | N.PF_EP_WEIGHT | N.PF_EP_FORCE_RESAMPLE)
    assert all(o["resampled"] for o in outs)
    assert all(o["anc_equal"] and o["wq_equal"] for o in outs), [(o["anc_equal"], o["wq_equal"]) for o in outs]
    assert all(o["lw_ok"] and o["state_ok"] and o["est_err_m"] <= H.EST_TOL_M for o in outs)


def test_reference_offset_mode_matches_reference_formula():
    tr = S.config0()
    eng = H.make_engine([4096], sys_offset="reference", seeds=[12345])
    eng.initialize(0, tr.anchor, tr.truth_clk[0], 10.0, 30.0)
    fe, sv = eng.pack_epoch([_epoch_rec(tr, 0, N.PF_EP_PREDICT | N.PF_EP_WEIGHT | N.PF_EP_FORCE_RESAMPLE)])
    eng.upload(0, fe, sv)
    eng.step()
    u, _, _ = eng.resample_info(0)
    assert u == int(np.floor((12345 % 1000000) / (1e6 * 4096) * 2 ** 32))


def test_huber_mode_parity():
    tr = S.config0()
    eng = H.make_engine([8192], weight_mode="huber")
    eng.initialize(0, tr.anchor, tr.truth_clk[0], 10.0, 30.0)
    outs = _run_and_check(eng, tr, 3, 1, wmode=1)
    assert all(o["lw_ok"] for o in outs), outs


def test_megopolis_matches_oracle_and_ks():
    """Megopolis with B = 32 on moderately peaked weights (ESS ~ N/5): the
    ancestors equal the oracle's chain with the same draws, the offspring
    counts match an independent oracle run in distribution (KS p > 0.01),
    and the offspring mass follows the weights.  (With ESS << N a
    32-iteration Metropolis chain cannot reach the few heavy particles --
    a property of the method, not of the kernel.)"""
    from scipy import stats
    tr = S.config0()
    n = 65_536
    eng = H.make_engine([n], resampler="megopolis", iters=32, sigma_pr=30.0)
    eng.initialize(0, tr.anchor, tr.truth_clk[0], 3.0, 3.0)
    fe, sv = eng.pack_epoch([_epoch_rec(tr, 0, N.PF_EP_PREDICT | N.PF_EP_WEIGHT | N.PF_EP_FORCE_RESAMPLE)])
    eng.upload(0, fe, sv)
    eng.step()
    _, lw = eng.state_f32(0, raw=True)
    w_all = np.exp(lw.astype(np.float64) - lw.max())
    assert w_all.sum() ** 2 / (w_all ** 2).sum() > n / 50  # moderately peaked
    anc = eng.ancestors(0)
    res = eng.results()[0]
    seed = eng.filters[0].seed
    same = O.megopolis(lw, 32, seed, res["epoch"] - 1, 0)
    assert np.mean(same == anc) > 0.999
    other = O.megopolis(lw, 32, seed + 77, res["epoch"] - 1, 0)
    c_gpu = np.bincount(anc, minlength=n)
    c_orc = np.bincount(other, minlength=n)
    p = stats.ks_2samp(c_gpu, c_orc).pvalue
    assert p > 0.01, p
    # and against the target distribution: offspring mass tracks the weights
    w = w_all / w_all.sum()
    heavy = w > 2.0 / n
    assert c_gpu[heavy].sum() / n == pytest.approx(w[heavy].sum(), abs=0.05)


def test_batched_equals_per_filter_and_graph():
    ns = [1000, 4097, 20_000, 777, 65_536, 3]
    trs = [S.single_filter(n_epochs=4, sats_per_const=8 + 5 * k, seed=k, nlos_frac=0.25) for k in range(len(ns))]

    def run(mode):
        eng = H.make_engine(ns, seeds=[7 + k for k in range(len(ns))])
        for k, tr in enumerate(trs):
            eng.initialize(k, tr.anchor, tr.truth_clk[0], 20.0, 30.0)
        if mode == "graph":
            eng.capture(False)
        for t in range(4):
            fe, sv = eng.pack_epoch([_epoch_rec(tr, t) for tr in trs])
            eng.upload(0, fe, sv)
            if mode == "batched":
                eng.step()
            elif mode == "per_filter":
                eng.step_per_filter()
            else:
                eng.replay(1)
        st = [eng.state_f32(k, raw=True) for k in range(len(ns))]
        return eng.results(), st

    rb, sb = run("batched")
    rp, sp = run("per_filter")
    rg, sg = run("graph")
    for k in range(len(ns)):
        assert np.array_equal(sb[k][0], sp[k][0]) and np.array_equal(sb[k][1], sp[k][1])
        assert np.array_equal(sb[k][0], sg[k][0]) and np.array_equal(sb[k][1], sg[k][1])
        assert np.array_equal(rb[k]["est_ecef"], rp[k]["est_ecef"])
        assert np.array_equal(rb[k]["est_ecef"], rg[k]["est_ecef"])


def test_batched_parity_each_filter():
    ns = [1500, 30_000, 9000]
    trs = [S.single_filter(n_epochs=3, sats_per_const=6 + 12 * k, seed=10 + k, nlos_frac=0.25) for k in range(3)]
    eng = H.make_engine(ns)
    for k, tr in enumerate(trs):
        eng.initialize(k, tr.anchor, tr.truth_clk[0], 15.0, 30.0)
    for t in range(3):
        befores = [eng.state_f32(k) for k in range(3)]
        shifts = [eng.anchor(k)[2] for k in range(3)]
        recs = [_epoch_rec(tr, t) for tr in trs]
        fe, sv = eng.pack_epoch(recs)
        eng.upload(0, fe, sv)
        eng.step()
        for k in range(3):
            o = H.check_step(eng, k, befores[k][0], shifts[k], recs[k])
            assert o["state_ok"] and o["lw_ok"] and o["est_err_m"] <= H.EST_TOL_M, (k, o)
            if o["resampled"]:
                assert o["anc_equal"], (k, o)


@pytest.mark.parametrize("resampler", ["systematic", "megopolis"])
def test_epoch_kernel_equals_kernel_chain(resampler):
    """The cooperative one-kernel epoch and the one-kernel-per-phase chain
    compute the same tile rows, merge them in the same order and resample
    with the same integer arithmetic: every output is bit-identical."""
    ns = [70_000, 1500, 4097]
    trs = [S.single_filter(n_epochs=4, sats_per_const=8 + 3 * k, seed=20 + k, nlos_frac=0.25) for k in range(3)]

    def run(chain):
        eng = H.make_engine(ns, resampler=resampler, chain=chain, seeds=[31, 32, 33])
        for k, tr in enumerate(trs):
            eng.initialize(k, tr.anchor, tr.truth_clk[0], 20.0, 30.0)
        outs = []
        for t in range(4):
            fl = N.PF_EP_PREDICT | N.PF_EP_WEIGHT | (N.PF_EP_FORCE_RESAMPLE if t % 2 else 0)
            fe, sv = eng.pack_epoch([_epoch_rec(tr, t, fl) for tr in trs])
            eng.upload(0, fe, sv)
            eng.step()
            outs.append([(eng.state_f32(k, raw=True), eng.ancestors(k), eng.results()[k]) for k in range(3)])
        return outs

    a, b = run(False), run(True)
    for sa, sb in zip(a, b):
        for (xa, anca, ra), (xb, ancb, rb) in zip(sa, sb):
            assert np.array_equal(xa[0], xb[0]) and np.array_equal(xa[1], xb[1])
            assert ra["resampled"] == rb["resampled"]
            if ra["resampled"]:
                assert np.array_equal(anca, ancb)
            assert np.array_equal(ra["est_ecef"], rb["est_ecef"]) and ra["ess"] == rb["ess"]


def test_determinism_same_seed_bit_identical():
    tr = S.config0()

    def run():
        eng = H.make_engine([30_000])
        eng.initialize(0, tr.anchor, tr.truth_clk[0], 10.0, 30.0)
        for t in range(5):
            fe, sv = eng.pack_epoch([_epoch_rec(tr, t)])
            eng.upload(0, fe, sv)
            eng.step()
        return eng.results()[0], eng.state_f32(0)

    (r1, s1), (r2, s2) = run(), run()
    assert np.array_equal(r1["est_ecef"], r2["est_ecef"])
    assert np.array_equal(s1[0], s2[0])


def test_step_io_equals_separate_calls():
    """pfe_step_io (upload, step, read in one call) gives the same results
    and state as the three calls."""
    tr = S.config0()

    def run(io):
        eng = H.make_engine([20_000, 3000], seeds=[5, 6])
        for k in range(2):
            eng.initialize(k, tr.anchor, tr.truth_clk[0], 10.0, 30.0)
        for t in range(4):
            fe, sv = eng.pack_epoch([_epoch_rec(tr, t)] * 2)
            if io:
                raw = eng.step_io(fe, sv)
                assert raw[1].epoch == t + 1
            else:
                eng.upload(0, fe, sv)
                eng.step()
        return eng.results(), eng.state_f32(0)

    (ra, sa), (rb, sb) = run(True), run(False)
    for k in range(2):
        assert np.array_equal(ra[k]["est_ecef"], rb[k]["est_ecef"]) and ra[k]["ess"] == rb[k]["ess"]
    assert np.array_equal(sa[0], sb[0]) and np.array_equal(sa[1], sb[1])
    eng = H.make_engine([1000], obs_slots=2)
    eng.initialize(0, tr.anchor, tr.truth_clk[0], 10.0, 30.0)
    fe, sv = eng.pack_epoch([_epoch_rec(tr, 0)])
    with pytest.raises(ValueError):
        eng.step_io(fe, sv)


def test_degenerate_weights_single_survivor():
    """One particle carries all the weight: the ESS is 1 and every slot
    descends from it (merge path with one particle owning all N slots)."""
    n = 70_000
    eng = H.make_engine([n], lw_mode="accumulate")
    tr = S.config0()
    eng.initialize(0, tr.anchor, tr.truth_clk[0], 10.0, 30.0)
    st, _ = eng.state_f32(0)
    lw = np.full(n, -1e5, np.float32)
    lw[54_321] = 0.0
    eng.set_state_f32(0, st, lw)
    fe, sv = eng.pack_epoch([_epoch_rec(tr, 0, N.PF_EP_WEIGHT | N.PF_EP_FORCE_RESAMPLE)])
    eng.upload(0, fe, sv)
    eng.step()
    res = eng.results()[0]
    assert res["ess"] == pytest.approx(1.0)
    anc = eng.ancestors(0)
    assert np.all(anc == 54_321)
    u, W, M = eng.resample_info(0)
    _, lw_raw = eng.state_f32(0, raw=True)
    assert np.array_equal(O.systematic_tiled(lw_raw, u)[0], anc)
    x, _ = eng.state_f32(0)
    assert np.all(x == st[:, 54_321][:, None])


@pytest.mark.parametrize("chain", [False, True])
def test_device_wait_timeout_sets_error_without_hang(chain):
    """A bounded device wait (grid barrier of the epoch kernel, look-back of
    the kernel chain) gives up, flags the error word, and the context stays
    usable (no trap, no hang)."""
    tr = S.config0()
    eng = H.make_engine([16 * 1024], chain=chain)
    eng.initialize(0, tr.anchor, tr.truth_clk[0], 10.0, 30.0)
    eng.set_spin_limit(2000)
    eng.poison_lookback(True)
    fe, sv = eng.pack_epoch([_epoch_rec(tr, 0, N.PF_EP_PREDICT | N.PF_EP_WEIGHT | N.PF_EP_FORCE_RESAMPLE)])
    eng.upload(0, fe, sv)
    eng.step()
    assert eng.error_word() & (1 | 8)
    with pytest.raises(N.PFError) as ei:
        eng.results()
    assert ei.value.status == N.PF_ETIMEOUT
    eng.poison_lookback(False)
    eng.set_spin_limit(0)
    eng.initialize(0, tr.anchor, tr.truth_clk[0], 10.0, 30.0)
    eng.upload(0, fe, sv)
    eng.step()
    assert eng.error_word() == 0
    assert eng.results()[0]["resampled"]


def test_recentering_keeps_offsets_small_over_a_trajectory():
    tr = S.config0()
    eng = H.make_engine([20_000])
    eng.initialize(0, tr.anchor, tr.truth_clk[0], 10.0, 30.0)
    errs = []
    for t in range(60):
        fe, sv = eng.pack_epoch([_epoch_rec(tr, t)])
        eng.upload(0, fe, sv)
        eng.step()
        r = eng.results()[0]
        errs.append(np.linalg.norm((r["est_ecef"] - tr.truth_ecef[t]) @ tr.rot[:2].T))
    x, _ = eng.state_f32(0)
    assert np.abs(x[:3]).max() < 200.0  # offsets stay near the anchor after 60 epochs (600 m travelled)
    assert np.median(errs[10:]) < 5.0


def test_step_io_graph_tracks_sizes_and_parameters():
    """pfe_step_io runs a captured graph per staging buffer: epochs with
    different satellite counts (the upload node is resized) and a likelihood
    change between calls (the graph is re-captured) give exactly the results
    of separate upload / step / read calls."""
    rng = np.random.RandomState(9)
    d = rng.randn(8, 3)
    sats = d / np.linalg.norm(d, axis=1, keepdims=True) * 20_000_000.0
    pr = np.linalg.norm(sats, axis=1) + 100.0 + rng.randn(8)
    from gnss_gpu_b200.engine import Engine, EngineOptions, FilterSpec

    counts = [8, 5, 8, 6, 4, 7, 8, 5]
    kinds = ["gaussian", "gaussian", "gaussian", "student_t", "student_t", "huber", "gaussian", "gmm"]

    def run(io):
        eng = Engine([FilterSpec(n_particles=30_000, seed=11, sigma_pos=(1.0, 1.0, 1.0), sigma_clk=3.0,
                                 sigma_pr=5.0)],
                     EngineOptions(n_clk=1, max_sats=8, obs_slots=1, weight_mode="generic"))
        eng.initialize(0, np.zeros(3), 100.0, 20.0, 50.0)
        out = []
        for t, (k, kind) in enumerate(zip(counts, kinds)):
            eng.set_likelihood(kind, nu=4.0)
            fe, sv = eng.pack_epoch([{"disp": np.zeros(3), "sats": sats[:k], "pr": pr[:k],
                                      "flags": N.PF_EP_PREDICT | N.PF_EP_WEIGHT | N.PF_EP_RESAMPLE_CHECK}])
            if io:
                r = eng.step_io(fe, sv)[0]
                out.append((tuple(r.est_ecef), r.ess, r.resampled, r.epoch))
            else:
                eng.upload(0, fe, sv)
                eng.step()
                r = eng.results()[0]
                out.append((tuple(r["est_ecef"]), r["ess"], int(r["resampled"]), r["epoch"]))
        st = eng.state_f32(0)
        eng.close()
        return out, st

    (oa, sa), (ob, sb) = run(True), run(False)
    for a, b in zip(oa, ob):
        assert np.array_equal(np.asarray(a[0]), np.asarray(b[0])) and a[1] == b[1] and a[2] == b[2] and a[3] == b[3]
    assert np.array_equal(sa[0], sb[0]) and np.array_equal(sa[1], sb[1])
