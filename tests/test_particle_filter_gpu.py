"""The reference's ParticleFilter tests (tests/test_particle_filter.py of the
reference project) run against the drop-in: the module-level functions of
gnss_gpu_b200._gnss_gpu_pf and the ParticleFilter class, plus their FP64
parity with the oracle."""
import numpy as np
import pytest

from conftest import N_TEST, SEED
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pfm():
    from gnss_gpu_b200 import _gnss_gpu_pf as m
    return m


@pytest.fixture(scope="module")
def PF():
    from gnss_gpu_b200 import ParticleFilter
    return ParticleFilter


def _arrays(n):
    return [np.empty(n, dtype=np.float64) for _ in range(4)]


# ---------------------------------------------- reference tests, ported
class TestInitialize:
    def test_particles_scattered_around_init(self, pfm):
        N = N_TEST
        init_pos = np.array([-3957199.0, 3310205.0, 3737911.0])
        px, py, pz, pcb = _arrays(N)
        pfm.pf_initialize(px, py, pz, pcb, *init_pos, 3000.0, 50.0, 500.0, N, SEED)
        assert abs(np.mean(px) - init_pos[0]) < 5.0 * 50.0 / np.sqrt(N) * 3
        assert abs(np.mean(pcb) - 3000.0) < 5.0 * 500.0 / np.sqrt(N) * 3
        assert abs(np.std(px) - 50.0) < 5.0
        assert abs(np.std(pcb) - 500.0) < 50.0

    def test_different_seeds_give_different_particles(self, pfm):
        a, b = _arrays(1000), _arrays(1000)
        pfm.pf_initialize(*a, 0, 0, 0, 0, 100, 100, 1000, 1)
        pfm.pf_initialize(*b, 0, 0, 0, 0, 100, 100, 1000, 2)
        assert not np.allclose(a[0], b[0])


class TestPredict:
    def test_mean_shifts_by_velocity(self, pfm):
        px, py, pz, pcb = _arrays(N_TEST)
        pfm.pf_initialize(px, py, pz, pcb, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0, N_TEST, SEED)
        mx, my = px.mean(), py.mean()
        pfm.pf_predict(px, py, pz, pcb, np.array([10.0]), np.array([20.0]), np.array([0.0]), 1.0, 0.1, 0.1,
                       N_TEST, SEED, 1)
        assert abs(px.mean() - mx - 10.0) < 1.0
        assert abs(py.mean() - my - 20.0) < 1.0


class TestWeight:
    def test_near_particles_get_higher_weight(self, pfm, tokyo):
        sat, pr, ws, tp, tcb = tokyo
        N = 1000
        r = np.random.default_rng(42)
        half = N // 2
        px = np.r_[tp[0] + r.normal(0, 1.0, half), tp[0] + 1000.0 + r.normal(0, 1.0, N - half)]
        py = np.r_[tp[1] + r.normal(0, 1.0, half), tp[1] + 1000.0 + r.normal(0, 1.0, N - half)]
        pz = tp[2] + r.normal(0, 1.0, N)
        pcb = tcb + r.normal(0, 10.0, N)
        lw = np.empty(N)
        pfm.pf_weight(px, py, pz, pcb, sat.ravel(), pr, ws, lw, N, len(pr), 5.0)
        assert lw[:half].mean() > lw[half:].mean()


class TestESS:
    def test_uniform_weights_ess_equals_n(self, pfm):
        assert abs(pfm.pf_compute_ess(np.zeros(N_TEST), N_TEST) - N_TEST) < N_TEST * 0.01

    def test_single_dominant_particle(self, pfm):
        lw = np.full(1000, -1000.0)
        lw[0] = 0.0
        assert pfm.pf_compute_ess(lw, 1000) < 2.0

    def test_ess_between_bounds(self, pfm):
        lw = np.random.default_rng(42).normal(0, 1.0, 1000)
        assert 1.0 <= pfm.pf_compute_ess(lw, 1000) <= 1000


class TestResampling:
    @pytest.mark.parametrize("method", ["systematic", "megopolis"])
    def test_particles_cluster_around_high_weight(self, pfm, tokyo, method):
        sat, pr, ws, tp, tcb = tokyo
        N = 1000
        px, py, pz, pcb = _arrays(N)
        pfm.pf_initialize(px, py, pz, pcb, *tp, tcb, 500.0, 2000.0, N, SEED)
        std_before = np.std(px)
        lw = np.empty(N)
        pfm.pf_weight(px, py, pz, pcb, sat.ravel(), pr, ws, lw, N, len(pr), 5.0)
        if method == "systematic":
            pfm.pf_resample_systematic(px, py, pz, pcb, lw, N, SEED)
        else:
            pfm.pf_resample_megopolis(px, py, pz, pcb, lw, N, 15, SEED)
        assert np.std(px) < std_before

    def test_megopolis_more_iterations_runs(self, pfm):
        N = 2000
        lw = np.zeros(N)
        lw[N // 4:] = -10.0
        r = np.random.default_rng(42)
        base = [r.normal(0, 1.0, N) for _ in range(4)]
        few = [b.copy() for b in base]
        many = [b.copy() for b in base]
        pfm.pf_resample_megopolis(*few, lw, N, 2, SEED)
        pfm.pf_resample_megopolis(*many, lw, N, 20, SEED)
        # more iterations: more slots hold a first-quarter particle
        first = set(base[0][: N // 4].tolist())
        assert np.mean([v in first for v in many[0]]) > np.mean([v in first for v in few[0]])


class TestEstimate:
    def test_estimate_with_uniform_weights(self, pfm):
        px, py, pz, pcb = _arrays(N_TEST)
        pfm.pf_initialize(px, py, pz, pcb, 100.0, 200.0, 300.0, 50.0, 10.0, 10.0, N_TEST, SEED)
        res = np.empty(4)
        pfm.pf_estimate(px, py, pz, pcb, np.zeros(N_TEST), res, N_TEST)
        np.testing.assert_allclose(res, [100.0, 200.0, 300.0, 50.0], atol=2.0)


class TestGetParticles:
    def test_get_particles_shape(self, pfm):
        N = 1000
        px = np.arange(N, dtype=np.float64)
        out = np.empty(N * 4)
        pfm.pf_get_particles(px, px * 2, px * 3, px * 4, out, N)
        out = out.reshape(N, 4)
        np.testing.assert_array_equal(out[:, 0], px)
        np.testing.assert_array_equal(out[:, 3], px * 4)


class TestFullPipeline:
    def test_convergence_to_true_position(self, PF, tokyo):
        sat, pr, ws, tp, tcb = tokyo
        pf = PF(n_particles=N_TEST, sigma_pos=0.5, sigma_cb=100.0, sigma_pr=5.0, resampling="megopolis",
                ess_threshold=0.5, seed=SEED)
        pf.initialize(tp + np.array([50.0, -30.0, 40.0]), clock_bias=tcb + 200.0, spread_pos=200.0,
                      spread_cb=1000.0)
        for _ in range(5):
            pf.predict(velocity=None, dt=1.0)
            pf.update(sat, pr, ws)
        est = pf.estimate()
        assert np.linalg.norm(est[:3] - tp) < 50.0
        assert abs(est[3] - tcb) < 500.0

    def test_convergence_systematic_resampling(self, PF, tokyo):
        sat, pr, ws, tp, tcb = tokyo
        pf = PF(n_particles=N_TEST, sigma_pos=0.5, sigma_cb=100.0, sigma_pr=5.0, resampling="systematic",
                ess_threshold=0.5, seed=SEED)
        pf.initialize(tp + np.array([50.0, -30.0, 40.0]), clock_bias=tcb + 200.0, spread_pos=200.0,
                      spread_cb=1000.0)
        for _ in range(15):
            pf.predict(velocity=None, dt=1.0)
            pf.update(sat, pr, ws)
        assert np.linalg.norm(pf.estimate()[:3] - tp) < 100.0

    def test_ess_drops_then_recovers(self, PF, tokyo):
        sat, pr, ws, tp, tcb = tokyo
        pf = PF(n_particles=N_TEST, sigma_pos=0.5, sigma_cb=100.0, sigma_pr=5.0, resampling="megopolis",
                ess_threshold=0.0, seed=SEED)
        pf.initialize(tp, clock_bias=tcb, spread_pos=500.0, spread_cb=2000.0)
        ess0 = pf.get_ess()
        assert abs(ess0 - N_TEST) < N_TEST * 0.01
        pf.update(sat, pr, ws)
        assert pf.get_ess() < ess0 * 0.5

    def test_get_particles_returns_correct_shape(self, PF):
        pf = PF(n_particles=1000, seed=SEED)
        pf.initialize([0, 0, 6_371_000.0], clock_bias=0.0)
        assert pf.get_particles().shape == (1000, 4)

    def test_not_initialized_raises(self, PF):
        pf = PF(n_particles=100, seed=SEED)
        with pytest.raises(RuntimeError):
            pf.predict()
        with pytest.raises(RuntimeError):
            pf.estimate()
        with pytest.raises(RuntimeError):
            pf.get_ess()


# ----------------------------------------------- FP64 parity with the oracle
class TestStatelessParity:
    def test_initialize_and_predict_match_oracle(self, pfm):
        n = 4099
        a = _arrays(n)
        pfm.pf_initialize(*a, 1.0, 2.0, 3.0, 4.0, 50.0, 500.0, n, 77)
        o = O.pf_initialize([1.0, 2.0, 3.0], 4.0, 50.0, 500.0, n, 77)
        for g, w in zip(a, o):
            np.testing.assert_allclose(g, w, rtol=1e-12, atol=1e-9)
        pfm.pf_predict(*a, np.array([1.5]), np.array([-2.0]), np.array([0.25]), 2.0, 0.7, 9.0, n, 77, 3)
        o2 = O.pf_predict(*o, [1.5, -2.0, 0.25], 2.0, 0.7, 9.0, 77, 3)
        for g, w in zip(a, o2):
            np.testing.assert_allclose(g, w, rtol=1e-12, atol=1e-9)

    def test_weight_ess_estimate_match_oracle(self, pfm, tokyo):
        sat, pr, ws, tp, tcb = tokyo
        n = 10_007
        r = np.random.default_rng(1)
        px, py, pz = (tp[i] + r.normal(0, 80, n) for i in range(3))
        pcb = tcb + r.normal(0, 300, n)
        w = r.uniform(0.5, 2, 8)
        lw = np.empty(n)
        pfm.pf_weight(px, py, pz, pcb, sat.ravel(), pr, w, lw, n, 8, 5.0)
        # FP64 on both sides; residuals cancel ~2e7 m ranges, so contraction
        # differences reach ~1e-10 relative
        np.testing.assert_allclose(lw, O.pf_weight(px, py, pz, pcb, sat, pr, w, 5.0), rtol=1e-9, atol=1e-9)
        assert pfm.pf_compute_ess(lw, n) == pytest.approx(O.pf_ess(lw), rel=1e-10)
        res = np.empty(4)
        pfm.pf_estimate(px, py, pz, pcb, lw, res, n)
        np.testing.assert_allclose(res, O.pf_estimate(px, py, pz, pcb, lw), rtol=0, atol=1e-6)

    @pytest.mark.parametrize("n", [1, 3, 1000, 10_000, 100_003])
    def test_systematic_ancestors_bit_exact(self, pfm, n):
        r = np.random.default_rng(n)
        lw = r.normal(0, 4, n)
        idx = np.arange(n, dtype=np.float64)
        a = [idx.copy(), idx.copy(), idx.copy(), idx.copy()]
        pfm.pf_resample_systematic(*a, lw, n, 12345)
        np.testing.assert_array_equal(a[0].astype(np.int64), O.pf_systematic_ancestors(lw, 12345))

    def test_megopolis_reference_chain_bit_exact(self, pfm):
        n = 20_000
        lw = np.random.default_rng(5).normal(0, 2, n)
        idx = np.arange(n, dtype=np.float64)
        a = [idx.copy() for _ in range(4)]
        pfm.pf_resample_megopolis(*a, lw, n, 15, 999)
        got = a[0].astype(np.int64)
        want = O.pf_megopolis_ref_ancestors(lw, 15, 999)
        # identical draws; an accept decision can flip only if exp() of the
        # two libraries differs in the last bit right at the threshold
        assert np.mean(got == want) > 0.999

    def test_invalid_inputs_raise(self, pfm):
        with pytest.raises(ValueError):
            pfm.pf_compute_ess(np.zeros(10), 0)
        lw = np.empty(10, dtype=np.float32)  # wrong dtype for an output
        with pytest.raises(ValueError):
            pfm.pf_weight(np.zeros(10), np.zeros(10), np.zeros(10), np.zeros(10), np.ones(3), np.ones(1),
                          np.ones(1), lw, 10, 1, 5.0)
