"""Building-aware filters on the device: the reference's 3D tests
(tests/test_pf3d.py, tests/test_pf3d_bvh.py of the reference project, the
parts that concern the likelihood and the filter) and parity of the device
ray tracing and likelihood with the FP64 brute-force oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from pfhelp import lw_close
from test_bvh_host import city_mesh

pytestmark = pytest.mark.gpu

N_TEST = 10000
SEED = 12345


@pytest.fixture(scope="module")
def M():
    import gnss_gpu_b200 as g
    from gnss_gpu_b200 import _gnss_gpu_pf3d, _gnss_gpu_pf
    return g, _gnss_gpu_pf3d, _gnss_gpu_pf


def _box(g):
    return g.BuildingModel.create_box(center=[100.0, 0.0, 25.0], width=20.0, depth=20.0, height=50.0)


def _scene():
    sat = np.array([[0.0, 0.0, 20000.0], [200.0, 0.0, 25.0], [0.0, 200.0, 5000.0], [150.0, 0.0, 10.0],
                    [-200.0, 0.0, 5000.0], [0.0, -200.0, 5000.0], [200.0, 200.0, 10000.0], [105.0, 0.0, 25.0]])
    pr = np.linalg.norm(sat, axis=1) + 100.0
    return sat, pr, np.ones(len(sat))


def _w3d(m3, tri, px, sat, pr, sigma_los=3.0, sigma_nlos=30.0, bias=20.0, **kw):
    n = len(px)
    lw = np.zeros(n)
    m3.pf_weight_3d(px[:, 0].copy(), px[:, 1].copy(), px[:, 2].copy(), np.full(n, 100.0), np.ravel(sat), pr,
                    np.ones(len(pr)), tri, lw, n, len(pr), sigma_los, sigma_nlos, bias, **kw)
    return lw


class TestWeight3DKernel:
    def test_los_and_nlos_sigma(self, M):
        g, m3, _ = M
        tri = _box(g).triangles
        px = np.zeros((100, 3))
        up = np.array([[0.0, 0.0, 20000.0]])
        assert np.allclose(_w3d(m3, tri, px, up, np.array([20000.0 + 100.0])), 0.0, atol=1e-10)
        behind = np.array([[200.0, 0.0, 25.0]])
        d = np.linalg.norm(behind)
        assert np.allclose(_w3d(m3, tri, px, behind, np.array([d + 100.0 + 20.0])), 0.0, atol=1e-10)

    def test_nlos_penalises_less_than_los_sigma(self, M):
        g, m3, m = M
        tri = _box(g).triangles
        n = 100
        behind = np.array([200.0, 0.0, 25.0])
        pr = np.array([np.linalg.norm(behind) + 100.0 + 50.0])
        lw3 = _w3d(m3, tri, np.zeros((n, 3)), behind[None], pr)
        lws = np.zeros(n)
        m.pf_weight(np.zeros(n), np.zeros(n), np.zeros(n), np.full(n, 100.0), behind, pr, np.ones(1), lws, n, 1, 3.0)
        assert np.all(lw3 > lws)

    def test_nlos_negative_residual_does_not_apply_bias(self, M):
        g, m3, _ = M
        tri = _box(g).triangles
        behind = np.array([[200.0, 0.0, 25.0]])
        lw = _w3d(m3, tri, np.zeros((32, 3)), behind, np.array([np.linalg.norm(behind) + 100.0 - 20.0]))
        assert np.allclose(lw, -0.5 * 20.0 ** 2 / 30.0 ** 2, atol=1e-10)

    def test_different_particles_different_los(self, M):
        g, m3, _ = M
        tri = _box(g).triangles
        sat = np.array([[0.0, 0.0, 20000.0], [200.0, 0.0, 25.0]])
        pr = np.array([20000.0, np.sqrt(200 ** 2 + 25 ** 2)]) + 100.0
        lw = _w3d(m3, tri, np.array([[0.0, 0.0, 0.0], [50.0, 0.0, 0.0]]), sat, pr)
        assert lw[0] > lw[1]

    def test_no_building_equals_los_weight(self, M):
        g, m3, m = M
        n = 100
        sat = np.array([0.0, 0.0, 20000.0])
        pr = np.array([20100.0])
        lw3 = _w3d(m3, np.zeros((0, 3, 3)), np.zeros((n, 3)), sat[None], pr, sigma_los=5.0)
        lws = np.zeros(n)
        m.pf_weight(np.zeros(n), np.zeros(n), np.zeros(n), np.full(n, 100.0), sat, pr, np.ones(1), lws, n, 1, 5.0)
        np.testing.assert_allclose(lw3, lws, atol=1e-10)

    def test_mixture_priors(self, M):
        g, m3, _ = M
        tri = _box(g).triangles
        sat, pr, _ = _scene()
        px = np.random.default_rng(1).normal(0, 5.0, (500, 3))
        for pb, pc in ((1.0, 0.0), (0.8, 0.1), (0.5, 0.5)):
            got = _w3d(m3, tri, px, sat, pr, blocked_nlos_prob=pb, clear_nlos_prob=pc)
            want, _ = O.weight_3d(px, np.full(len(px), 100.0), np.column_stack([sat, pr, np.ones(len(pr))]), tri,
                                  3.0, 30.0, 20.0, pb, pc)
            np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-9)


class TestParticleFilter3D:
    def test_construction_and_types(self, M):
        g, _, _ = M
        pf = g.ParticleFilter3D(building_model=_box(g), sigma_los=3.0, sigma_nlos=30.0, nlos_bias=20.0,
                                n_particles=1000, sigma_pos=1.0, sigma_cb=300.0)
        assert (pf.sigma_los, pf.sigma_nlos, pf.nlos_bias, pf.n_particles) == (3.0, 30.0, 20.0, 1000)
        with pytest.raises(TypeError):
            g.ParticleFilter3D(building_model="not a model", n_particles=100)
        with pytest.raises(TypeError):
            g.ParticleFilter3DBVH(bvh="not a bvh", n_particles=100)

    @pytest.mark.parametrize("bvh", [False, True])
    def test_estimate_near_truth(self, M, bvh):
        g, _, _ = M
        sat, pr, w = _scene()
        kw = dict(n_particles=N_TEST, sigma_pos=1.0, sigma_cb=300.0, sigma_los=3.0, sigma_nlos=30.0,
                  nlos_bias=20.0, resampling="systematic", seed=SEED)
        pf = (g.ParticleFilter3DBVH(bvh=g.BVHAccelerator.from_building_model(_box(g)), **kw) if bvh
              else g.ParticleFilter3D(building_model=_box(g), **kw))
        pf.initialize(position_ecef=np.zeros(3), clock_bias=100.0, spread_pos=20.0, spread_cb=200.0)
        for _ in range(3):
            pf.predict(dt=0.0)
            pf.update(sat, pr, w)
        assert np.linalg.norm(pf.estimate()[:3]) < 30.0
        assert 0.0 < pf.get_ess() <= N_TEST
        assert pf.get_particles().shape == (N_TEST, 4)

    def test_pf3d_beats_plain_with_nlos(self, M):
        g, _, _ = M
        sat = np.array([[0.0, 0.0, 20000.0], [0.0, 200.0, 5000.0], [-200.0, 0.0, 5000.0], [0.0, -200.0, 5000.0],
                        [200.0, 0.0, 25.0], [150.0, 0.0, 10.0]])
        pr = np.linalg.norm(sat, axis=1) + 100.0
        pr[4:] += 30.0
        std = g.ParticleFilter(n_particles=N_TEST, sigma_pos=1.0, sigma_cb=300.0, sigma_pr=5.0,
                               resampling="systematic", seed=SEED)
        p3 = g.ParticleFilter3D(building_model=_box(g), n_particles=N_TEST, sigma_pos=1.0, sigma_cb=300.0,
                                sigma_los=3.0, sigma_nlos=30.0, nlos_bias=20.0, resampling="systematic", seed=SEED)
        for pf in (std, p3):
            pf.initialize(position_ecef=np.zeros(3), clock_bias=100.0, spread_pos=20.0, spread_cb=200.0)
            for _ in range(3):
                pf.predict(dt=0.0)
                pf.update(sat, pr, np.ones(len(sat)))
        assert np.linalg.norm(p3.estimate()[:3]) < np.linalg.norm(std.estimate()[:3])


# -------------------------------------------------- FP64 oracle parity
def test_los_matches_brute_force_oracle(M):
    g, _, _ = M
    tri, anchor, rot, city = city_mesh(3, 800.0)
    bvh = g.BVHAccelerator(tri)
    rng = np.random.default_rng(4)
    R, S_ = 300, 16
    enu = np.column_stack([rng.uniform(0, 800, R), rng.uniform(0, 800, R), rng.uniform(0.5, 3.0, R)])
    rx = anchor + enu @ rot
    az = rng.uniform(0, 2 * np.pi, (R, S_))
    el = rng.uniform(np.radians(5), np.radians(85), (R, S_))
    u = np.stack([np.cos(el) * np.sin(az), np.cos(el) * np.cos(az), np.sin(el)], axis=-1)
    sats = rx[:, None, :] + 2.2e7 * (u @ rot)
    got = bvh.check_los_batch(rx, sats)
    want = O.los(rx, sats, tri)
    assert got.shape == (R, S_)
    assert 0.05 < 1.0 - want.mean() < 0.95          # the scene has both
    assert np.sum(got != want) <= 3                 # FP32 vs FP64 only at grazing edges
    assert bvh.check_los(rx[0], sats[0]).tolist() == got[0].tolist()
    nan = sats.copy()
    nan[0, 0] = np.nan
    assert not bvh.check_los_batch(rx, nan)[0, 0]


def test_engine_3d_term_matches_oracle(M):
    g, _, _ = M
    from gnss_gpu_b200.engine import Engine, EngineOptions, FilterSpec
    tri, anchor, rot, city = city_mesh(5, 800.0)
    bvh = g.BVHAccelerator(tri)
    rng = np.random.default_rng(6)
    start = anchor + np.array([400.0, 400.0, 1.5]) @ rot
    S_ = 12
    az = rng.uniform(0, 2 * np.pi, S_)
    el = rng.uniform(np.radians(10), np.radians(80), S_)
    sats = start + 2.2e7 * (np.stack([np.cos(el) * np.sin(az), np.cos(el) * np.cos(az), np.sin(el)], 1) @ rot)
    pr = np.linalg.norm(sats - start, axis=1) + 50.0 + rng.exponential(10.0, S_) * (rng.random(S_) < 0.3)
    w = rng.uniform(0.5, 2.0, S_)
    eng = Engine([FilterSpec(n_particles=20_000, seed=3, sigma_pos=(1.0, 1.0, 1.0), sigma_clk=1.0, sigma_pr=3.0)],
                 EngineOptions(n_clk=1, max_sats=16))
    eng.initialize(0, start, 50.0, 60.0, 5.0)
    eng.add_3d_term(0, bvh.mesh, sats, pr, w, 3.0, 30.0, 20.0, 0.9, 0.05)
    x, lw = eng.state_f32(0)
    a, clk, _ = eng.anchor(0)
    frame, _ = eng.frame(0)
    pos = a[None, :] + x[:3].astype(np.float64).T @ frame
    want, blk = O.weight_3d(pos, clk[0] + x[3].astype(np.float64), np.column_stack([sats, pr, w]), tri, 3.0, 30.0,
                            20.0, 0.9, 0.05)
    assert 0.02 < blk.mean() < 0.98
    ok, rel = lw_close(lw, want)
    assert np.mean(ok) >= 1.0 - 1e-3 and np.sum(~ok) <= 5, f"worst {rel.max():.2e}"


def test_bvh_filter_in_a_city(M):
    g, _, _ = M
    tri, anchor, rot, city = city_mesh(7, 800.0)
    bvh = g.BVHAccelerator(tri)
    rng = np.random.default_rng(8)

    def outdoors(e, n):
        b = city.box[city.occ]
        return not np.any((b[:, 0] - 2 <= e) & (e <= b[:, 1] + 2) & (b[:, 2] - 2 <= n) & (n <= b[:, 3] + 2))

    e, n = next((e, n) for e, n in rng.uniform(100.0, 700.0, (200, 2)) if outdoors(e, n))
    truth = anchor + np.array([e, n, 1.5]) @ rot
    S_ = 16
    az = rng.uniform(0, 2 * np.pi, S_)
    el = rng.uniform(np.radians(10), np.radians(80), S_)
    sats = truth + 2.2e7 * (np.stack([np.cos(el) * np.sin(az), np.cos(el) * np.cos(az), np.sin(el)], 1) @ rot)
    blocked = ~bvh.check_los(truth, sats)
    pr = np.linalg.norm(sats - truth, axis=1) + 80.0 + np.where(blocked, 25.0, 0.0) + rng.normal(0, 1.0, S_)
    guess = truth + rng.normal(0, 5.0, 3)
    pf = g.ParticleFilter3DBVH(bvh=bvh, n_particles=50_000, sigma_pos=0.5, sigma_cb=1.0, sigma_los=3.0,
                               sigma_nlos=30.0, nlos_bias=20.0, resampling="systematic", seed=2)
    pf.initialize(guess, clock_bias=80.0, spread_pos=15.0, spread_cb=5.0)
    for _ in range(5):
        pf.predict(dt=1.0)
        pf.update(sats, pr)
    est = pf.estimate()
    assert np.all(np.isfinite(est)) and 0.0 < pf.get_ess() <= 50_000
    # the building-aware likelihood prefers the truth to the initial guess
    _, m3, _ = M
    lw = np.zeros(2)
    pts = np.stack([truth, guess])
    m3.pf_weight_3d(pts[:, 0].copy(), pts[:, 1].copy(), pts[:, 2].copy(), np.full(2, 80.0), sats.ravel(), pr,
                    np.ones(S_), tri, lw, 2, S_, 3.0, 30.0, 20.0)
    assert lw[0] > lw[1]


def test_sort_spatially_is_a_deterministic_permutation():
    """Engine.sort_spatially reorders the particles (a permutation of the
    same states and log-weights), the same way every time, into Morton
    order of their East/North cells."""
    import numpy as np
    from gnss_gpu_b200 import scenario as S
    from gnss_gpu_b200.engine import Engine, EngineOptions, FilterSpec

    tr = S.config0()
    outs = []
    for _ in range(2):
        eng = Engine([FilterSpec(n_particles=50_000, seed=3, sigma_pos=(1.0, 1.0, 1.0), sigma_clk=3.0,
                                 sigma_pr=5.0)], EngineOptions(n_clk=1, max_sats=8))
        eng.initialize(0, tr.anchor, 100.0, 30.0, 50.0)
        st0, lw0 = eng.state_f32(0)
        eng.sort_spatially(0, cell=2.0)
        st1, lw1 = eng.state_f32(0)
        eng.close()
        outs.append(st1)
        a = np.lexsort(st0[::-1]); b = np.lexsort(st1[::-1])
        assert np.array_equal(st0[:, a], st1[:, b])
        # neighbours in the new order are close: median step between consecutive particles
        step = np.hypot(np.diff(st1[0]), np.diff(st1[1]))
        assert np.median(step) < 0.25 * np.median(np.hypot(np.diff(st0[0]), np.diff(st0[1])))
    assert np.array_equal(outs[0], outs[1])
