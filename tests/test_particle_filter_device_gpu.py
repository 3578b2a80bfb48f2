"""ParticleFilterDevice drop-in: the reference's wrapper tests
(tests/test_cuda_streams.py of the reference project, the parts this
filter models) and FP64 parity of every likelihood, position term, shift
and statistic with the oracle."""
from types import SimpleNamespace

import numpy as np
import pytest

from conftest import TOKYO_SATS, TOKYO_PR, TOKYO_TRUE_POS, TOKYO_TRUE_CB
from oracle import oracle as O
from pfhelp import lw_close, EST_TOL_M, ESS_RTOL

pytestmark = pytest.mark.gpu

SEED = 42
ORIGIN = np.array([0.0, 0.0, 0.0])
ORIGIN_CB = 100.0


def _origin_sats(n_sat=8):
    """Satellites of the reference's stream tests: receiver at the ECEF
    origin, 20,000 km away in seeded random directions."""
    rng = np.random.RandomState(123)
    d = rng.randn(n_sat, 3)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    sat = d * 20_000_000.0
    pr = np.linalg.norm(sat - ORIGIN, axis=1) + ORIGIN_CB
    return sat, pr, np.ones(n_sat)


@pytest.fixture(scope="module")
def PFD():
    from gnss_gpu_b200 import ParticleFilterDevice
    return ParticleFilterDevice


def _cloud(pf):
    """(offsets (4, n) FP64, anchor, clock anchor, rot) of the current
    particles -- the frame the device weighted them in."""
    eng = pf._engine
    x, _ = eng.state_f32(0)
    anchor, clk, _ = eng.anchor(0)
    rot, _ = eng.frame(0)
    return x.astype(np.float64), anchor, clk, rot


# ------------------------------------------------ reference tests, ported
class TestWrapper:
    def test_sync_method_exists(self, PFD):
        pf = PFD(n_particles=1000, seed=SEED)
        pf.initialize(position_ecef=ORIGIN, clock_bias=ORIGIN_CB, spread_pos=50.0, spread_cb=200.0)
        pf.sync()

    def test_full_pipeline_with_sync(self, PFD):
        sat, pr, w = _origin_sats()
        pf = PFD(n_particles=100_000, sigma_pos=1.0, sigma_cb=300.0, sigma_pr=5.0, resampling="systematic",
                 seed=SEED)
        pf.initialize(position_ecef=ORIGIN, clock_bias=ORIGIN_CB, spread_pos=50.0, spread_cb=200.0)
        for _ in range(3):
            pf.predict(dt=1.0)
            pf.update(sat, pr, w)
        pf.sync()
        res = pf.estimate()
        assert res.shape == (4,)
        assert np.all(np.isfinite(res))

    def test_get_log_weights_shape(self, PFD):
        sat, pr, w = _origin_sats()
        pf = PFD(n_particles=1024, sigma_pos=1.0, sigma_cb=300.0, sigma_pr=5.0, resampling="systematic", seed=SEED)
        pf.initialize(position_ecef=ORIGIN, clock_bias=ORIGIN_CB, spread_pos=50.0, spread_cb=200.0)
        pf.predict(dt=1.0)
        pf.update(sat, pr, w, resample=False)
        lw = pf.get_log_weights()
        assert lw.shape == (1024,)
        assert np.all(np.isfinite(lw))
        pf.resample_if_needed()

    def test_get_particle_states_shape(self, PFD):
        pf = PFD(n_particles=2048, seed=SEED)
        pf.initialize(position_ecef=ORIGIN, clock_bias=ORIGIN_CB, spread_pos=0.0, spread_cb=0.0)
        st = pf.get_particle_states()
        assert st.shape == (2048, 16)
        np.testing.assert_allclose(st[:, :3], 0.0, atol=1e-9)
        np.testing.assert_allclose(st[:, 3], ORIGIN_CB, atol=1e-9)
        assert pf.estimate().shape == (4,)

    def test_get_position_spread_shrinks_after_update(self, PFD):
        sat, pr, w = _origin_sats()
        pf = PFD(n_particles=50_000, sigma_pos=1.0, sigma_cb=300.0, sigma_pr=5.0, resampling="systematic", seed=SEED)
        pf.initialize(position_ecef=ORIGIN, clock_bias=ORIGIN_CB, spread_pos=80.0, spread_cb=200.0)
        s0 = pf.get_position_spread(center=ORIGIN)
        pf.update(sat, pr, w, resample=False)
        s1 = pf.get_position_spread()
        assert np.isfinite(s0) and np.isfinite(s1)
        assert s1 < s0

    def test_per_particle_nlos_gate_skips_outlier_residuals(self, PFD):
        sat, pr, w = _origin_sats(5)
        out = pr.copy()
        out[0] += 100.0
        kw = dict(n_particles=1024, sigma_pos=1.0, sigma_cb=300.0, sigma_pr=5.0, resampling="systematic", seed=SEED,
                  per_particle_nlos_gate=True, per_particle_nlos_undiff_pr_threshold_m=30.0)
        pf = PFD(**kw)
        pf.initialize(ORIGIN, clock_bias=ORIGIN_CB, spread_pos=0.0, spread_cb=0.0)
        pf.update(sat, out, w, resample=False)
        assert float(np.max(np.abs(pf.get_log_weights()))) < 1e-6
        pf2 = PFD(**kw)
        pf2.initialize(ORIGIN, clock_bias=ORIGIN_CB, spread_pos=0.0, spread_cb=0.0)
        pf2.update(sat, pr + 100.0, w, resample=False)
        assert float(np.max(pf2.get_log_weights())) < -900.0

    def test_per_particle_huber_softens_outlier_cost_without_rejecting(self, PFD):
        sat, pr, w = _origin_sats(5)
        out = pr.copy()
        out[0] += 100.0

        def lw0(huber):
            pf = PFD(n_particles=1024, sigma_pos=1.0, sigma_cb=300.0, sigma_pr=5.0, resampling="systematic",
                     seed=SEED, per_particle_huber=huber, per_particle_huber_undiff_pr_k=1.5)
            pf.initialize(ORIGIN, clock_bias=ORIGIN_CB, spread_pos=0.0, spread_cb=0.0)
            pf.update(sat, out, w, resample=False)
            return float(pf.get_log_weights()[0])

        g, h = lw0(False), lw0(True)
        assert g == pytest.approx(-200.0)
        assert h == pytest.approx(-28.875)
        assert g < h < 0.0

    def test_get_resample_ancestors_after_systematic(self, PFD):
        sat, pr, w = _origin_sats()
        pf = PFD(n_particles=512, sigma_pos=1.0, sigma_cb=300.0, sigma_pr=5.0, resampling="systematic", seed=SEED)
        pf.initialize(position_ecef=ORIGIN, clock_bias=ORIGIN_CB, spread_pos=50.0, spread_cb=200.0)
        pf.predict(dt=1.0)
        pf.update(sat, pr, w)
        pf._resample()
        anc = pf.get_resample_ancestors()
        assert anc.shape == (512,) and anc.dtype == np.int32
        assert np.all(anc >= 0) and np.all(anc < 512)

    @pytest.mark.parametrize("method", ["systematic", "megopolis"])
    def test_convergence_near_truth(self, PFD, method):
        sat, pr, w = _origin_sats()
        pf = PFD(n_particles=100_000, sigma_pos=1.0, sigma_cb=300.0, sigma_pr=5.0, resampling=method,
                 ess_threshold=0.5, seed=SEED)
        pf.initialize(position_ecef=ORIGIN, clock_bias=ORIGIN_CB, spread_pos=20.0, spread_cb=200.0)
        for _ in range(5):
            pf.predict(dt=0.0)
            pf.update(sat, pr, w)
        assert np.linalg.norm(pf.estimate()[:3] - ORIGIN) < 100.0

    @staticmethod
    def _dd(outlier, carrier=False, n_sat=5):
        sat, _, _ = _origin_sats(n_sat)
        base = np.array([120.0, -35.0, 18.0])
        rr = np.linalg.norm(sat - ORIGIN, axis=1)
        br = np.linalg.norm(sat - base, axis=1)
        dd = (rr[1:] - rr[0]) - (br[1:] - br[0])
        wl = np.full(n_sat - 1, 0.190293673)
        if carrier:
            dd = dd / wl
        dd[0] += outlier
        return SimpleNamespace(dd_pseudorange_m=dd, dd_carrier_cycles=dd, sat_ecef_k=sat[1:],
                               sat_ecef_ref=np.repeat(sat[[0]], n_sat - 1, axis=0), base_range_k=br[1:],
                               base_range_ref=np.repeat(br[0], n_sat - 1), dd_weights=np.ones(n_sat - 1),
                               wavelengths_m=wl, n_dd=n_sat - 1)

    @pytest.mark.parametrize("huber,want", [(False, -5000.0), (True, -148.875)])
    def test_dd_pseudorange_huber_known_answers(self, PFD, huber, want):
        pf = PFD(n_particles=1024, sigma_pos=1.0, sigma_cb=300.0, sigma_pr=5.0, resampling="systematic", seed=SEED,
                 per_particle_huber=huber, per_particle_huber_dd_pr_k=1.5)
        pf.initialize(ORIGIN, clock_bias=0.0, spread_pos=0.0, spread_cb=0.0)
        pf.update_dd_pseudorange(self._dd(50.0), sigma_pr=0.5, resample=False)
        assert float(pf.get_log_weights()[0]) == pytest.approx(want)

    @pytest.mark.parametrize("huber,want", [(False, -40.5), (True, -12.375)])
    def test_dd_carrier_huber_known_answers(self, PFD, huber, want):
        pf = PFD(n_particles=1024, sigma_pos=1.0, sigma_cb=300.0, sigma_pr=5.0, resampling="systematic", seed=SEED,
                 per_particle_huber=huber, per_particle_huber_dd_carrier_k=1.5)
        pf.initialize(ORIGIN, clock_bias=0.0, spread_pos=0.0, spread_cb=0.0)
        pf.update_dd_carrier_afv(self._dd(0.45, carrier=True), sigma_cycles=0.05, resample=False)
        assert float(pf.get_log_weights()[0]) == pytest.approx(want, abs=1e-5)

    def test_dd_gates_skip_outlier_pairs(self, PFD):
        kw = dict(n_particles=1024, sigma_pos=1.0, sigma_cb=300.0, sigma_pr=5.0, resampling="systematic", seed=SEED,
                  per_particle_nlos_gate=True, per_particle_nlos_dd_pr_threshold_m=10.0,
                  per_particle_nlos_dd_carrier_threshold_cycles=0.3)
        pf = PFD(**kw)
        pf.initialize(ORIGIN, clock_bias=0.0, spread_pos=0.0, spread_cb=0.0)
        pf.update_dd_pseudorange(self._dd(50.0), sigma_pr=0.5, resample=False)
        assert float(np.max(np.abs(pf.get_log_weights()))) < 1e-6
        pf2 = PFD(**kw)
        pf2.initialize(ORIGIN, clock_bias=0.0, spread_pos=0.0, spread_cb=0.0)
        pf2.update_dd_carrier_afv(self._dd(0.45, carrier=True), sigma_cycles=0.05, resample=False)
        assert float(np.max(np.abs(pf2.get_log_weights()))) < 1e-6

    def test_update_dd_pseudorange_smoke(self, PFD):
        rng = np.random.RandomState(321)
        d = rng.randn(5, 3)
        sat = d / np.linalg.norm(d, axis=1, keepdims=True) * 20_000_000.0
        base = np.array([120.0, -35.0, 18.0])
        rr = np.linalg.norm(sat, axis=1)
        br = np.linalg.norm(sat - base, axis=1)
        res = SimpleNamespace(dd_pseudorange_m=(rr[1:] - rr[0]) - (br[1:] - br[0]), sat_ecef_k=sat[1:],
                              sat_ecef_ref=np.repeat(sat[[0]], 4, axis=0), base_range_k=br[1:],
                              base_range_ref=np.repeat(br[0], 4), dd_weights=np.ones(4), n_dd=4)
        pf = PFD(n_particles=50_000, sigma_pos=1.0, sigma_cb=300.0, sigma_pr=5.0, resampling="systematic", seed=SEED)
        pf.initialize(ORIGIN, clock_bias=250.0, spread_pos=30.0, spread_cb=200.0)
        pf.update_dd_pseudorange(res, sigma_pr=0.5)
        pf.sync()
        est = pf.estimate()
        assert np.all(np.isfinite(est)) and np.linalg.norm(est[:3]) < 10.0

    def test_update_dd_carrier_afv_smoke(self, PFD):
        sat = np.array([[20_200_000.0, 0.0, 0.0], [0.0, 21_000_000.0, 0.0], [0.0, 0.0, 20_600_000.0],
                        [-20_800_000.0, 2_000_000.0, 1_000_000.0]])
        rover = np.array([0.3, -0.2, 0.1])
        base = np.array([120.0, -35.0, 18.0])
        rr = np.linalg.norm(sat - rover, axis=1)
        br = np.linalg.norm(sat - base, axis=1)
        wl = np.array([0.190293673, 0.192039486, 0.190293673])
        refs, ks = np.array([0, 2, 2]), np.array([1, 3, 1])
        res = SimpleNamespace(dd_carrier_cycles=((rr[ks] - rr[refs]) - (br[ks] - br[refs])) / wl, sat_ecef_k=sat[ks],
                              sat_ecef_ref=sat[refs], base_range_k=br[ks], base_range_ref=br[refs],
                              dd_weights=np.ones(3), wavelengths_m=wl, n_dd=3)
        pf = PFD(n_particles=30_000, sigma_pos=0.1, sigma_cb=300.0, sigma_pr=5.0, resampling="systematic", seed=SEED)
        pf.initialize(position_ecef=rover, clock_bias=0.0, spread_pos=0.2, spread_cb=10.0)
        pf.update_dd_carrier_afv(res, sigma_cycles=0.05)
        pf.sync()
        est = pf.estimate()
        assert np.all(np.isfinite(est)) and np.linalg.norm(est[:3] - rover) < 2.0

    def test_not_built_paths_raise(self, PFD):
        pf = PFD(n_particles=1024)
        with pytest.raises(RuntimeError):
            pf.predict()
        pf.initialize(ORIGIN, clock_bias=ORIGIN_CB)
        with pytest.raises(RuntimeError):
            pf.smooth()  # no stored epochs
        with pytest.raises(RuntimeError):
            pf.get_resample_ancestors()  # megopolis


# ------------------------------------------------------ FP64 parity
LIKELIHOODS = [
    ("gaussian", dict(), dict(kind="gaussian")),
    ("student_t", dict(nu=4.0), dict(kind="student_t", nu=4.0)),
    ("huber", dict(per_particle_huber=True, per_particle_huber_undiff_pr_k=1.5), dict(kind="huber", huber_k=1.5)),
    ("gate", dict(per_particle_nlos_gate=True, per_particle_nlos_undiff_pr_threshold_m=20.0),
     dict(kind="gaussian", gate_m=20.0)),
    ("student_t_gate", dict(nu=3.0, per_particle_nlos_gate=True, per_particle_nlos_undiff_pr_threshold_m=25.0),
     dict(kind="student_t", nu=3.0, gate_m=25.0)),
]


def _nlos_pr(seed=9):
    rng = np.random.default_rng(seed)
    pr = TOKYO_PR.copy()
    pr[[1, 4]] += rng.uniform(20.0, 60.0, 2)  # two NLOS delays
    w = rng.uniform(0.5, 2.0, len(pr))
    return pr, w


@pytest.mark.parametrize("name,ctor,lik", LIKELIHOODS, ids=[l[0] for l in LIKELIHOODS])
@pytest.mark.parametrize("method", ["systematic", "megopolis"])
def test_update_log_weights_match_oracle(PFD, name, ctor, lik, method):
    pr, w = _nlos_pr()
    pf = PFD(n_particles=60_000, sigma_pos=2.0, sigma_cb=3.0, sigma_pr=5.0, resampling=method, seed=7, **ctor)
    pf.initialize(TOKYO_TRUE_POS + 15.0, clock_bias=TOKYO_TRUE_CB, spread_pos=40.0, spread_cb=30.0)
    for t in range(3):
        pf.predict(velocity=np.array([1.0, -0.5, 0.2]), dt=1.0)
        pf.update(TOKYO_SATS, pr, w, resample=(t < 2))
        if t == 2:
            x, anchor, clk, rot = _cloud(pf)
            rows = np.column_stack([TOKYO_SATS, pr, w])
            want, res = O.weight_generic(x, anchor, clk, rot, rows, 5.0, **lik)
            got = pf.get_log_weights()
            ok, rel = lw_close(got, want)
            if lik.get("gate_m", 0.0) > 0.0:
                # particles with a residual within 2 cm of the gate may fall
                # either side in FP32
                ok |= np.any(np.abs(np.abs(res) - lik["gate_m"]) < 0.02, axis=0)
                assert np.mean(ok) == 1.0
            assert ok.all(), f"{name}: worst {rel.max():.2e}"
            # estimate and ESS of the same weights
            pos = anchor[None, :] + x[:3].T @ rot
            wt = np.exp(want - want.max())
            est = np.concatenate([(wt[:, None] * pos).sum(0), [(wt * (clk[0] + x[3])).sum()]]) / wt.sum()
            assert np.max(np.abs(pf.estimate() - est)) <= EST_TOL_M
            ess = wt.sum() ** 2 / (wt * wt).sum()
            assert pf.get_ess() == pytest.approx(ess, rel=ESS_RTOL)


def test_update_gmm_log_weights_match_oracle(PFD):
    pr, w = _nlos_pr(3)
    pf = PFD(n_particles=50_000, sigma_pos=2.0, sigma_cb=3.0, sigma_pr=4.0, resampling="systematic", seed=11)
    pf.initialize(TOKYO_TRUE_POS, clock_bias=TOKYO_TRUE_CB, spread_pos=30.0, spread_cb=20.0)
    pf.predict(dt=1.0)
    pf.update_gmm(TOKYO_SATS, pr, w, w_los=0.8, mu_nlos=20.0, sigma_nlos=25.0, resample=False)
    x, anchor, clk, rot = _cloud(pf)
    want, _ = O.weight_generic(x, anchor, clk, rot, np.column_stack([TOKYO_SATS, pr, w]), 4.0, kind="gmm",
                               w_los=0.8, mu_nlos=20.0, sigma_nlos=25.0)
    ok, rel = lw_close(pf.get_log_weights(), want)
    assert ok.all(), f"worst {rel.max():.2e}"


def test_sigma_pr_override_and_zero_weight_satellite(PFD):
    pr, w = _nlos_pr(4)
    w[2] = 0.0
    pf = PFD(n_particles=20_000, sigma_pr=5.0, nu=5.0, seed=3)
    pf.initialize(TOKYO_TRUE_POS, clock_bias=TOKYO_TRUE_CB, spread_pos=20.0, spread_cb=20.0)
    pf.update(TOKYO_SATS, pr, w, sigma_pr=2.5, resample=False)
    x, anchor, clk, rot = _cloud(pf)
    want, _ = O.weight_generic(x, anchor, clk, rot, np.column_stack([TOKYO_SATS, pr, w]), 2.5, kind="student_t",
                               nu=5.0)
    ok, rel = lw_close(pf.get_log_weights(), want)
    assert ok.all(), f"worst {rel.max():.2e}"


# ------------------------------------------------ position terms, shifts
def _weighted(pf, n=40_000, seed=5):
    pf.initialize(TOKYO_TRUE_POS, clock_bias=TOKYO_TRUE_CB, spread_pos=25.0, spread_cb=15.0)
    pf.predict(dt=1.0)
    pf.update(TOKYO_SATS, TOKYO_PR, None, resample=False)
    return pf


def test_position_update_matches_oracle(PFD):
    pf = _weighted(PFD(n_particles=40_000, resampling="systematic", seed=2))
    before = pf.get_log_weights()
    p = pf.get_particles()
    ref = TOKYO_TRUE_POS + np.array([3.0, -4.0, 2.0])
    pf.position_update(ref, sigma_pos=30.0)
    want = before - 0.5 * np.sum((p[:, :3] - ref) ** 2, axis=1) / 900.0
    ok, rel = lw_close(pf.get_log_weights(), want)
    assert ok.all(), f"worst {rel.max():.2e}"
    wt = np.exp(want - want.max())
    assert pf.get_ess() == pytest.approx(wt.sum() ** 2 / (wt * wt).sum(), rel=ESS_RTOL)
    est = (wt[:, None] * p).sum(0) / wt.sum()
    assert np.max(np.abs(pf.estimate() - est)) <= EST_TOL_M


@pytest.mark.parametrize("K", [1, 3, 8, 40])
def test_position_mixture_update_matches_oracle(PFD, K):
    pf = _weighted(PFD(n_particles=40_000, resampling="systematic", seed=4))
    before = pf.get_log_weights()
    p = pf.get_particles()
    rng = np.random.default_rng(K)
    refs = TOKYO_TRUE_POS + rng.normal(0, 10.0, (K, 3))
    mix = rng.uniform(0.0, 1.0, K)
    if K > 1:
        mix[0] = 0.0  # a zero-weight component
    pf.position_mixture_update(refs, sigma_pos=6.0, mixture_weights=mix)
    m = mix / mix.sum()
    with np.errstate(divide="ignore"):
        comp = np.log(m)[None, :] - 0.5 * np.sum((p[:, None, :3] - refs[None]) ** 2, axis=2) / 36.0
    mx = comp.max(1)
    want = before + mx + np.log(np.exp(comp - mx[:, None]).sum(1))
    ok, rel = lw_close(pf.get_log_weights(), want)
    assert ok.all(), f"worst {rel.max():.2e}"


def test_position_update_after_resample_and_resample_if_needed(PFD):
    pf = PFD(n_particles=30_000, resampling="systematic", seed=8, ess_threshold=0.5)
    pf.initialize(TOKYO_TRUE_POS, clock_bias=TOKYO_TRUE_CB, spread_pos=60.0, spread_cb=30.0)
    pf.update(TOKYO_SATS, TOKYO_PR, None)            # resamples: weights reset
    assert pf.get_ess() == pytest.approx(30_000.0)
    assert np.all(pf.get_log_weights() == 0.0)
    p = pf.get_particles()
    ref = TOKYO_TRUE_POS + np.array([20.0, 0.0, 0.0])
    pf.position_update(ref, sigma_pos=2.0)            # sharp: ESS falls
    want = -0.5 * np.sum((p[:, :3] - ref) ** 2, axis=1) / 4.0
    ok, rel = lw_close(pf.get_log_weights(), want)
    assert ok.all(), f"worst {rel.max():.2e}"
    wt = np.exp(want - want.max())
    ess = wt.sum() ** 2 / (wt * wt).sum()
    assert ess < 15_000
    assert pf.get_ess() == pytest.approx(ess, rel=ESS_RTOL)
    assert pf.resample_if_needed() is True
    assert pf.get_ess() == pytest.approx(30_000.0)
    anc = pf.get_resample_ancestors()
    np.testing.assert_array_equal(np.sort(anc), anc)  # systematic: ancestors ascending
    np.testing.assert_allclose(pf.get_particles(), p[anc], atol=1e-4)  # FP32 offsets re-centred
    assert pf.resample_if_needed() is False


def test_shifts_move_every_particle(PFD):
    pf = _weighted(PFD(n_particles=20_000, resampling="megopolis", seed=6))
    p0 = pf.get_particles()
    lw0 = pf.get_log_weights()
    pf.shift_clock_bias(12.5)
    p1 = pf.get_particles()
    np.testing.assert_allclose(p1[:, 3] - p0[:, 3], 12.5, atol=1e-6)
    np.testing.assert_allclose(p1[:, :3], p0[:, :3], atol=1e-9)
    est = pf.estimate()
    target = est[:3] + np.array([5.0, -3.0, 1.0])
    norm, applied = pf.recenter_position(target, max_shift_m=100.0)
    assert applied and norm == pytest.approx(np.sqrt(35.0), rel=1e-9)
    np.testing.assert_allclose(pf.estimate()[:3], target, atol=EST_TOL_M)
    norm, applied = pf.recenter_position(target + 1e4, max_shift_m=100.0)
    assert not applied
    assert pf.recenter_position(np.array([np.nan, 0.0, 0.0])) == (float("inf"), False)
    np.testing.assert_array_equal(pf.get_log_weights(), lw0)
    # clock re-centring on the residual median at the estimate
    est = pf.estimate()
    res = TOKYO_PR - np.linalg.norm(TOKYO_SATS - est[:3], axis=1)
    pf.correct_clock_bias(TOKYO_SATS, TOKYO_PR, quantile=0.5)
    assert pf.estimate()[3] == pytest.approx(np.median(res), abs=EST_TOL_M)


def test_state_and_weight_roundtrip(PFD):
    pf = _weighted(PFD(n_particles=10_000, resampling="systematic", seed=12))
    rng = np.random.default_rng(1)
    st = np.zeros((10_000, 16))
    st[:, :3] = TOKYO_TRUE_POS + rng.normal(0, 30.0, (10_000, 3))
    st[:, 3] = TOKYO_TRUE_CB + rng.normal(0, 10.0, 10_000)
    pf.set_particle_states(st)
    assert np.all(pf.get_log_weights() == 0.0)
    assert pf.get_ess() == pytest.approx(10_000.0)
    np.testing.assert_allclose(pf.get_particles(), st[:, :4], atol=1e-4)
    np.testing.assert_allclose(pf.get_particle_states()[:, 4:], 0.0)
    lw = rng.normal(0, 2.0, 10_000)
    lw[:10] = -np.inf
    pf.set_log_weights(lw)
    got = pf.get_log_weights()
    np.testing.assert_array_equal(got[:10], -np.inf)
    np.testing.assert_allclose(got[10:], lw[10:].astype(np.float32), rtol=0, atol=0)
    wt = np.exp(lw - lw.max())
    assert pf.get_ess() == pytest.approx(wt.sum() ** 2 / (wt * wt).sum(), rel=ESS_RTOL)
    c = TOKYO_TRUE_POS + np.array([4.0, 4.0, -2.0])
    want = np.sqrt(np.sum(wt * np.sum((st[:, :3] - c) ** 2, axis=1)) / wt.sum())
    assert pf.get_position_spread(center=c) == pytest.approx(want, rel=1e-5)
    est = (wt[:, None] * st[:, :4]).sum(0) / wt.sum()
    np.testing.assert_allclose(pf.estimate(), est, atol=EST_TOL_M)
    want0 = np.sqrt(np.sum(wt * np.sum((st[:, :3] - est[:3]) ** 2, axis=1)) / wt.sum())
    assert pf.get_position_spread() == pytest.approx(want0, rel=1e-5)
    # the filter steps on from the restored state
    pf.predict(dt=1.0)
    pf.update(TOKYO_SATS, TOKYO_PR)
    assert np.all(np.isfinite(pf.estimate()))
    with pytest.raises(ValueError):
        pf.set_particle_states(st[:10])
    with pytest.raises(ValueError):
        pf.set_log_weights(lw[:10])


# --------------------------------- differenced / carrier terms, FP64 parity
def _dd_tokyo(rng, n_pairs, carrier=False, nlos=()):
    base = TOKYO_TRUE_POS + np.array([800.0, -450.0, 30.0])
    sats = TOKYO_SATS[: n_pairs + 1]
    rr = np.linalg.norm(sats - TOKYO_TRUE_POS, axis=1)
    br = np.linalg.norm(sats - base, axis=1)
    refs = np.zeros(n_pairs, int)
    ks = np.arange(1, n_pairs + 1)
    wl = rng.choice([0.190293673, 0.244210213, 0.254828049], n_pairs)
    dd = (rr[ks] - rr[refs]) - (br[ks] - br[refs])
    if carrier:
        dd = dd / wl + rng.normal(0, 0.02, n_pairs) + rng.integers(-50, 50, n_pairs)
    else:
        dd = dd + rng.normal(0, 0.5, n_pairs)
    for i in nlos:
        dd[i] += 25.0 if not carrier else 0.4
    return SimpleNamespace(dd_pseudorange_m=dd, dd_carrier_cycles=dd, sat_ecef_k=sats[ks], sat_ecef_ref=sats[refs],
                           base_range_k=br[ks], base_range_ref=br[refs], dd_weights=rng.uniform(0.5, 2.0, n_pairs),
                           wavelengths_m=wl, n_dd=n_pairs)


def _obs_want(pf, kind, res, obs, sigma, gate=0.0, huber_k=0.0, wl=None):
    x, anchor, clk, rot = _cloud(pf)
    return O.obs_term(x, anchor, clk, rot, kind, res.sat_ecef_k, obs, res.dd_weights, res.sat_ecef_ref,
                      res.base_range_k, res.base_range_ref, wl, sigma, gate, huber_k)


def _mask_edges(ok, r, gate, afv):
    if gate > 0:
        ok |= np.any(np.abs(np.abs(r) - gate) < 1e-6, axis=0)
    if afv:
        ok |= np.any(np.abs(np.abs(r) - 0.5) < 1e-6, axis=0)
    return ok


DD_CASES = [("gauss", dict(), 0.0, 0.0), ("huber", dict(per_particle_huber=True, per_particle_huber_dd_pr_k=1.2), 0.0, 1.2),
            ("gate", dict(per_particle_nlos_gate=True, per_particle_nlos_dd_pr_threshold_m=8.0), 8.0, 0.0)]


@pytest.mark.parametrize("name,ctor,gate,hk", DD_CASES, ids=[c[0] for c in DD_CASES])
def test_dd_pseudorange_matches_oracle(PFD, name, ctor, gate, hk):
    rng = np.random.default_rng(21)
    res = _dd_tokyo(rng, 7, nlos=(2,))
    pf = PFD(n_particles=40_000, resampling="systematic", seed=5, **ctor)
    pf.initialize(TOKYO_TRUE_POS, clock_bias=TOKYO_TRUE_CB, spread_pos=15.0, spread_cb=20.0)
    pf.predict(dt=1.0)
    pf.update(TOKYO_SATS, TOKYO_PR, None, resample=True)     # a gathered cloud underneath
    pf.update_dd_pseudorange(res, sigma_pr=0.8, resample=False)
    want, r = _obs_want(pf, O.OBS_DD_PSEUDORANGE, res, res.dd_pseudorange_m, 0.8, gate, hk)
    ok, rel = lw_close(pf.get_log_weights(), want, rtol=1e-6)
    ok = _mask_edges(ok, r, gate, False)
    assert ok.all(), f"worst {rel.max():.2e}"


@pytest.mark.parametrize("gate,hk", [(0.0, 0.0), (0.25, 0.0), (0.0, 1.5)])
def test_dd_carrier_accumulates_and_matches_oracle(PFD, gate, hk):
    rng = np.random.default_rng(22)
    res = _dd_tokyo(rng, 7, carrier=True, nlos=(4,))
    ctor = dict(per_particle_nlos_gate=gate > 0, per_particle_nlos_dd_carrier_threshold_cycles=gate or 0.5,
                per_particle_huber=hk > 0, per_particle_huber_dd_carrier_k=hk or 1.5)
    pf = PFD(n_particles=40_000, resampling="megopolis", seed=6, **ctor)
    pf.initialize(TOKYO_TRUE_POS, clock_bias=TOKYO_TRUE_CB, spread_pos=0.5, spread_cb=5.0)
    pf.update(TOKYO_SATS, TOKYO_PR, None, resample=False)
    before = pf.get_log_weights()
    pf.update_dd_carrier_afv(res, sigma_cycles=0.05, resample=False)
    term, r = _obs_want(pf, O.OBS_DD_CARRIER_AFV, res, res.dd_carrier_cycles, 0.05, gate, hk, res.wavelengths_m)
    ok, rel = lw_close(pf.get_log_weights(), before + term)
    ok = _mask_edges(ok, r, gate, True)
    assert ok.all(), f"worst {rel.max():.2e}"


def test_carrier_afv_matches_oracle_and_resamples(PFD):
    rng = np.random.default_rng(23)
    wl = 0.190293673
    rng_true = np.linalg.norm(TOKYO_SATS - TOKYO_TRUE_POS, axis=1)
    cyc = (rng_true + TOKYO_TRUE_CB) / wl + rng.normal(0, 0.02, len(rng_true)) + rng.integers(-1_000_000, 1_000_000, len(rng_true))
    w = rng.uniform(0.5, 1.5, len(cyc))
    pf = PFD(n_particles=50_000, resampling="systematic", seed=9, ess_threshold=0.5)
    pf.initialize(TOKYO_TRUE_POS, clock_bias=TOKYO_TRUE_CB, spread_pos=0.3, spread_cb=0.3)
    pf.update_carrier_afv(TOKYO_SATS, cyc, w, wavelength=wl, sigma_cycles=0.05, resample=False)
    x, anchor, clk, rot = _cloud(pf)
    want, r = O.obs_term(x, anchor, clk, rot, O.OBS_CARRIER_AFV, TOKYO_SATS, cyc, w, wavelength=np.full(len(cyc), wl),
                         sigma=0.05)
    ok, rel = lw_close(pf.get_log_weights(), want)
    ok = _mask_edges(ok, r, 0.0, True)
    assert ok.all(), f"worst {rel.max():.2e}"
    wt = np.exp(want - want.max())
    ess = wt.sum() ** 2 / (wt * wt).sum()
    assert pf.get_ess() == pytest.approx(ess, rel=ESS_RTOL)
    assert pf.resample_if_needed() == bool(ess < 25_000)


def test_obs_term_rejects_bad_rows(PFD):
    pf = PFD(n_particles=1024)
    pf.initialize(TOKYO_TRUE_POS, clock_bias=TOKYO_TRUE_CB)
    res = _dd_tokyo(np.random.default_rng(1), 4, carrier=True)
    res.wavelengths_m = np.array([0.19, 0.0, 0.19, 0.19])
    with pytest.raises(ValueError):
        pf.update_dd_carrier_afv(res)
    res.wavelengths_m = np.full(4, 0.19)
    res.dd_carrier_cycles = np.array([1.0, np.nan, 2.0, 3.0])
    with pytest.raises(ValueError):
        pf.update_dd_carrier_afv(res)
    with pytest.raises(ValueError):
        pf.update_dd_pseudorange(res, sigma_pr=0.0)


# ------------------------------------------------- velocity states, Doppler
from test_oracle import doppler_case, L1  # noqa: E402


class TestVelocityWrapper:
    """The reference's velocity-state tests (tests/test_cuda_streams.py:
    216-337, 406-505), through the drop-in."""

    def test_states_include_velocity_and_covariance(self, PFD):
        pf = PFD(n_particles=2048, seed=SEED)
        pf.initialize(np.array([10.0, 20.0, 30.0]), clock_bias=ORIGIN_CB, spread_pos=0.0, spread_cb=0.0,
                      velocity=np.array([1.5, -2.0, 0.25]), spread_vel=0.0, velocity_init_sigma=2.0)
        st = pf.get_particle_states()
        assert st.shape == (2048, 16)
        np.testing.assert_allclose(st[:, :3], np.tile([10.0, 20.0, 30.0], (2048, 1)), atol=1e-5)
        np.testing.assert_allclose(st[:, 4:7], np.tile([1.5, -2.0, 0.25], (2048, 1)))
        np.testing.assert_allclose(st[:, [7, 11, 15]], 4.0)
        np.testing.assert_allclose(st[:, [8, 9, 10, 12, 13, 14]], 0.0)

    def test_predict_moves_by_the_guide(self, PFD):
        pf = PFD(n_particles=2048, seed=SEED, velocity_guide_alpha=0.999999999)
        pf.initialize(ORIGIN, clock_bias=ORIGIN_CB, spread_pos=0.0, spread_cb=0.0)
        pf.predict(velocity=np.array([2.0, -1.0, 0.5]), dt=0.25, sigma_pos=0.0)
        st = pf.get_particle_states()
        np.testing.assert_allclose(st[:, :3], np.tile([0.5, -0.25, 0.125], (2048, 1)), atol=1e-5)
        np.testing.assert_allclose(st[:, 4:7], np.tile([2.0, -1.0, 0.5], (2048, 1)), atol=1e-8)

    def test_rbpf_predict_spreads_by_velocity_covariance(self, PFD):
        pf = PFD(n_particles=20_000, seed=SEED, rbpf_velocity_kf=True, velocity_process_noise=0.5)
        pf.initialize(ORIGIN, clock_bias=ORIGIN_CB, spread_pos=0.0, spread_cb=0.0, velocity=np.array([1.0, 0, 0]),
                      velocity_init_sigma=2.0)
        pf.predict(velocity=np.array([1.0, 0.0, 0.0]), dt=1.0, sigma_pos=1.0)
        st = pf.get_particle_states()
        np.testing.assert_allclose(st[:, 4:7], np.tile([1.0, 0.0, 0.0], (20_000, 1)))
        for i, c in enumerate((1.0, 0.0, 0.0)):
            assert 1.6 < float(np.std(st[:, i] - c)) < 2.4
        np.testing.assert_allclose(st[:, [7, 11, 15]], 4.5)

    def test_wrapper_rbpf_predict_controls(self, PFD):
        pf = PFD(n_particles=4096, seed=SEED, rbpf_velocity_kf=True, velocity_process_noise=0.25)
        pf.initialize(ORIGIN, clock_bias=ORIGIN_CB, spread_pos=0.0, spread_cb=0.0, velocity=np.array([0.5, -0.25, 0.0]),
                      velocity_init_sigma=1.0)
        pf.predict(velocity=np.array([0.5, -0.25, 0.0]), dt=2.0, sigma_pos=0.0)
        st = pf.get_particle_states()
        np.testing.assert_allclose(st[:, 4:7], np.tile([0.5, -0.25, 0.0], (4096, 1)))
        np.testing.assert_allclose(st[:, [7, 11, 15]], 1.5)

    def test_update_doppler_moves_velocity(self, PFD):
        rx, sat, sv, dop, tv = doppler_case()
        pf = PFD(n_particles=2048, seed=SEED, resampling="systematic")
        pf.initialize(rx, clock_bias=ORIGIN_CB, spread_pos=0.0, spread_cb=0.0, velocity=np.zeros(3))
        pf.update_doppler(sat, sv, dop, weights=np.ones(6), sigma_mps=0.5, velocity_update_gain=1.0,
                          max_velocity_update_mps=100.0, resample=False)
        np.testing.assert_allclose(pf.get_particle_states()[:, 4:7], np.tile(tv, (2048, 1)), atol=1e-3)

    def test_update_doppler_kf_moves_velocity(self, PFD):
        rx, sat, sv, dop, tv = doppler_case()
        pf = PFD(n_particles=2048, seed=SEED, resampling="systematic")
        pf.initialize(rx, clock_bias=ORIGIN_CB, spread_pos=0.0, spread_cb=0.0, velocity=np.zeros(3),
                      velocity_init_sigma=10.0)
        pf.update_doppler_kf(sat, sv, dop, weights=np.ones(6), sigma_mps=0.5, resample=False)
        st = pf.get_particle_states()
        np.testing.assert_allclose(st[:, 4:7], np.tile(tv, (2048, 1)), atol=2e-2)
        assert np.all(st[:, [7, 11, 15]] < 100.0) and np.all(st[:, [7, 11, 15]] > 0.0)


@pytest.mark.parametrize("kf", [False, True])
def test_velocity_predict_matches_oracle(PFD, kf):
    n = 3000
    pf = PFD(n_particles=n, seed=77, resampling="systematic", sigma_vel=0.0 if kf else 0.7,
             velocity_guide_alpha=0.6, rbpf_velocity_kf=kf, velocity_process_noise=0.3)
    pf.initialize(TOKYO_TRUE_POS, clock_bias=TOKYO_TRUE_CB, spread_pos=5.0, spread_cb=3.0,
                  velocity=np.array([3.0, -1.0, 0.5]), spread_vel=1.5, velocity_init_sigma=0.8)
    st0 = pf.get_particle_states()
    guide = np.array([2.0, 1.0, -0.5])
    pf.predict(velocity=guide, dt=0.5, sigma_pos=0.4)
    st1 = pf.get_particle_states()
    pos, v, P = O.vel_predict(st0[:, :3], st0[:, 4:7], st0[:, 7:], guide, 0.5, 0.4, 0.0 if kf else 0.7, 0.6, kf, 0.3,
                              pf._step, 77)
    np.testing.assert_allclose(st1[:, 4:7], v, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(st1[:, 7:], P, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(st1[:, :3], pos, rtol=0, atol=2e-5)  # FP32 offsets about the anchor


@pytest.mark.parametrize("kf", [False, True])
def test_doppler_matches_oracle(PFD, kf):
    rx, sat, sv, dop, tv = doppler_case()
    rng = np.random.default_rng(3)
    dop = dop + rng.normal(0, 2.0, len(dop))
    w = rng.uniform(0.5, 2.0, len(dop))
    n = 2000
    pf = PFD(n_particles=n, seed=5, resampling="systematic", rbpf_velocity_kf=kf)
    pf.initialize(rx, clock_bias=ORIGIN_CB, spread_pos=20.0, spread_cb=10.0, velocity=np.array([0.5, 0.0, -0.2]),
                  spread_vel=1.0, velocity_init_sigma=3.0)
    pf.update(sat, np.linalg.norm(sat - rx, axis=1) + ORIGIN_CB, None, resample=False)
    before = pf.get_log_weights()
    st0 = pf.get_particle_states()
    if kf:
        pf.update_doppler_kf(sat, sv, dop, weights=w, sigma_mps=0.4, resample=False)
    else:
        pf.update_doppler(sat, sv, dop, weights=w, sigma_mps=0.4, velocity_update_gain=0.5,
                          max_velocity_update_mps=2.0, resample=False)
    st1 = pf.get_particle_states()
    # positions the device used: the FP32 offsets about the anchor, in FP64
    x, anchor, clk, rot = _cloud(pf)
    pos = anchor[None, :] + x[:3].T @ rot
    lw, v, P = O.doppler(pos, st0[:, 4:7], st0[:, 7:], sat, sv, dop, w, L1, 0.4, gain=0.5, max_update=2.0, kf=kf)
    ok, rel = lw_close(pf.get_log_weights(), before + lw, rtol=1e-6)
    assert ok.all(), f"worst {rel.max():.2e}"
    np.testing.assert_allclose(st1[:, 4:7], v, rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(st1[:, 7:], P, rtol=1e-9, atol=1e-12)


def test_velocities_follow_resampling(PFD):
    pf = PFD(n_particles=5000, seed=9, resampling="systematic", sigma_vel=0.5, ess_threshold=0.99)
    pf.initialize(TOKYO_TRUE_POS, clock_bias=TOKYO_TRUE_CB, spread_pos=30.0, spread_cb=20.0,
                  velocity=np.zeros(3), spread_vel=2.0)
    before = pf.get_particle_states()
    pf.update(TOKYO_SATS, TOKYO_PR, None, resample=True)       # resamples (threshold 0.99)
    anc = pf.get_resample_ancestors()
    after = pf.get_particle_states()
    np.testing.assert_array_equal(after[:, 4:], before[anc, 4:])
    np.testing.assert_allclose(after[:, :3], before[anc, :3], atol=1e-4)
    pf.predict(velocity=np.array([1.0, 0, 0]), dt=1.0)
    pf.update(TOKYO_SATS, TOKYO_PR, None)
    assert np.all(np.isfinite(pf.estimate()))


# ------------------------------------------------ forward-backward smoothing
class TestSmoothing:
    def test_smooth_with_dd_pseudorange_and_carrier_smoke(self, PFD):
        """Reference tests/test_cuda_streams.py:775-831, 1002-1079."""
        sat = np.array([[20_200_000.0, 0.0, 0.0], [0.0, 21_000_000.0, 0.0], [0.0, 0.0, 20_600_000.0],
                        [-20_800_000.0, 2_000_000.0, 1_000_000.0]])
        rover = np.array([0.3, -0.2, 0.1])
        base = np.array([120.0, -35.0, 18.0])
        rr, br = np.linalg.norm(sat - rover, axis=1), np.linalg.norm(sat - base, axis=1)
        dd_pr = SimpleNamespace(dd_pseudorange_m=(rr[1:] - rr[0]) - (br[1:] - br[0]), sat_ecef_k=sat[1:],
                                sat_ecef_ref=np.repeat(sat[[0]], 3, axis=0), base_range_k=br[1:],
                                base_range_ref=np.repeat(br[0], 3), dd_weights=np.ones(3), ref_sat_ids=("G01",) * 3,
                                n_dd=3)
        ks, rs = np.array([1, 3, 1]), np.array([0, 2, 2])
        wl = np.array([0.190293673, 0.192039486, 0.190293673])
        dd_cp = SimpleNamespace(dd_carrier_cycles=((rr[ks] - rr[rs]) - (br[ks] - br[rs])) / wl, sat_ecef_k=sat[ks],
                                sat_ecef_ref=sat[rs], base_range_k=br[ks], base_range_ref=br[rs], dd_weights=np.ones(3),
                                wavelengths_m=wl, ref_sat_ids=("G01", "E03", "G03"), n_dd=3)
        pf = PFD(n_particles=20_000, sigma_pos=0.1, sigma_cb=300.0, sigma_pr=5.0, resampling="systematic", seed=SEED)
        pf.initialize(position_ecef=rover, clock_bias=0.0, spread_pos=0.2, spread_cb=10.0)
        pf.enable_smoothing()
        for _ in range(3):
            pf.predict(dt=1.0)
            pf.update_dd_pseudorange(dd_pr, sigma_pr=0.5)
            pf.resample_if_needed()
            pf.update_dd_carrier_afv(dd_cp, sigma_cycles=0.05)
            pf.store_epoch(sat, rr, np.ones(4), None, 1.0, spp_ref=None, dd_pseudorange=dd_pr,
                           dd_pseudorange_sigma=0.5, dd_carrier=dd_cp, dd_carrier_sigma=0.05)
        smoothed, forward = pf.smooth(position_update_sigma=None)
        assert smoothed.shape == (3, 3) and forward.shape == (3, 3)
        assert np.all(np.isfinite(smoothed)) and np.all(np.isfinite(forward))
        with pytest.raises(RuntimeError):
            pf.smooth()  # the stored epochs are consumed

    def test_smoothing_runs_a_noisy_drive(self, PFD):
        rng = np.random.default_rng(11)
        sat, _, _ = _origin_sats(8)
        v = np.array([1.0, 0.5, 0.0])
        truth = [ORIGIN + v * t for t in range(30)]
        pf = PFD(n_particles=50_000, sigma_pos=0.5, sigma_cb=2.0, sigma_pr=5.0, resampling="systematic", seed=5)
        pf.initialize(truth[0], clock_bias=ORIGIN_CB, spread_pos=5.0, spread_cb=5.0)
        pf.enable_smoothing()
        for t, p in enumerate(truth):
            if t:
                pf.predict(velocity=v, dt=1.0)
            pr = np.linalg.norm(sat - p, axis=1) + ORIGIN_CB + rng.normal(0, 5.0, len(sat))
            pf.update(sat, pr)
            pf.store_epoch(sat, pr, np.ones(len(sat)), v, 1.0)
        smoothed, forward = pf.smooth()
        assert smoothed.shape == forward.shape == (30, 3)
        err_f = np.linalg.norm(forward - np.array(truth), axis=1)
        err_s = np.linalg.norm(smoothed - np.array(truth), axis=1)
        # the reference's scheme (an independent backward filter averaged in)
        # guarantees no gain; both passes must track the drive
        assert np.sqrt(np.mean(err_f ** 2)) < 3.0 and np.sqrt(np.mean(err_s ** 2)) < 3.0
