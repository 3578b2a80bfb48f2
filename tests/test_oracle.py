"""CPU tests: the FP64 oracle pinned against the reference's own code and
fixtures, plus properties of the exact systematic predicate."""
import numpy as np
import pytest

from conftest import TOKYO_SATS, TOKYO_PR, TOKYO_TRUE_POS, TOKYO_TRUE_CB
from oracle import oracle as O

GOLD = np.load(__import__("pathlib").Path(__file__).parent / "golden" / "simple_pf_cpu.npz")


# --------------------------------------------------------------- Philox
# Known-answer vectors of Philox4x32-10 published with the Random123 library
# of Salmon et al. (SC'11).
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,want", PHILOX_KAT)
def test_philox_known_answers(ctr, key, want):
    assert tuple(int(v) for v in O.philox10(ctr, key)) == want


def test_philox_matches_curand_fixture_if_present():
    """Words of cuRAND's Philox4_32_10 (the reference's generator,
    predict.cu:14-20) recorded on a GPU by tests/golden/make_curand_fixture.py."""
    import json
    from pathlib import Path
    p = Path(__file__).parent / "golden" / "curand_philox.json"
    if not p.exists():
        pytest.skip("cuRAND fixture not generated yet")
    d = json.loads(p.read_text())
    for rec in d["records"]:
        seed, subseq = rec["seed"], rec["subsequence"]
        key = (seed & 0xFFFFFFFF, seed >> 32)
        ctr = (0, 0, subseq & 0xFFFFFFFF, subseq >> 32)
        words = []
        c = list(ctr)
        for _ in range(len(rec["words"]) // 4):
            words.extend(int(v) for v in O.philox10(c, key))
            c[0] = (c[0] + 1) & 0xFFFFFFFF
        assert words == rec["words"], f"seed {seed} subsequence {subseq}"


# ------------------------------------------------------------ weights
def test_weight_matches_reference_simple_pf_cpu():
    """Shifted log-likelihoods equal the reference CPU filter's
    (experiments/evaluate.py:735-749) to FP64 round-off."""
    for c in range(3):
        parts = GOLD[f"c{c}_particles"]
        ws = GOLD[f"c{c}_wsat"]
        lw = O.pf_weight(parts[:, 0], parts[:, 1], parts[:, 2], parts[:, 3], TOKYO_SATS, TOKYO_PR, ws, 5.0)
        got = lw - lw.max()
        want = GOLD[f"c{c}_shifted_loglik"]
        np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-7 * max(1.0, np.abs(want).max()) * 1e-3)


def test_ess_and_estimate_match_reference_simple_pf_cpu():
    for c in range(3):
        parts = GOLD[f"c{c}_particles"]
        lw = GOLD[f"c{c}_lw_rand"]
        assert O.pf_ess(lw) == pytest.approx(float(GOLD[f"c{c}_ess"]), rel=1e-12)
        est = O.pf_estimate(parts[:, 0], parts[:, 1], parts[:, 2], parts[:, 3], lw)
        np.testing.assert_allclose(est, GOLD[f"c{c}_estimate"], rtol=1e-13, atol=1e-7)


def test_gaussian_and_huber_known_answers():
    """A 100 m outlier at sigma 5: Gaussian -200, Huber (k = 1.5) -28.875
    (reference tests/test_cuda_streams.py:668-693)."""
    sats = TOKYO_SATS[:5]
    rng = np.linalg.norm(sats - TOKYO_TRUE_POS, axis=1)
    pr = rng + TOKYO_TRUE_CB
    pr[0] += 100.0
    rot = np.eye(3)
    x = np.zeros((4, 1))
    rows = np.column_stack([sats, pr, np.ones(5)])
    clk = np.zeros(5, np.int32)
    g = O.weight(x, TOKYO_TRUE_POS, [TOKYO_TRUE_CB], rot, rows, clk, 5.0, mode=0)
    h = O.weight(x, TOKYO_TRUE_POS, [TOKYO_TRUE_CB], rot, rows, clk, 5.0, mode=1, huber_k=1.5)
    assert g[0] == pytest.approx(-200.0, abs=1e-6)
    assert h[0] == pytest.approx(-28.875, abs=1e-6)


def test_reference_scenario_near_beats_far():
    """tests/test_particle_filter.py:136-168 of the reference, on the oracle."""
    r = np.random.default_rng(42)
    n = 1000
    half = n // 2
    px = np.r_[TOKYO_TRUE_POS[0] + r.normal(0, 1, half), TOKYO_TRUE_POS[0] + 1000 + r.normal(0, 1, half)]
    py = np.r_[TOKYO_TRUE_POS[1] + r.normal(0, 1, half), TOKYO_TRUE_POS[1] + 1000 + r.normal(0, 1, half)]
    pz = TOKYO_TRUE_POS[2] + r.normal(0, 1, n)
    pcb = TOKYO_TRUE_CB + r.normal(0, 10, n)
    lw = O.pf_weight(px, py, pz, pcb, TOKYO_SATS, TOKYO_PR, np.ones(8), 5.0)
    assert lw[:half].mean() > lw[half:].mean()


# -------------------------------------------------------- systematic
def _slow_systematic(lw32, max_lw, u32):
    """Pure-Python restatement of resampling.cu:60-83 on exact integers."""
    q = [int(v) for v in O.quantize(lw32, max_lw)]
    n = len(q)
    C = np.cumsum(np.array(q, dtype=object))
    W = int(C[-1])
    anc = []
    for k in range(n):
        T = (k << 32) | u32
        lo, hi = 0, n - 1
        while lo < hi:
            mid = (lo + hi) // 2
            if (int(C[mid]) * n << 32) < T * W:
                lo = mid + 1
            else:
                hi = mid
        anc.append(lo)
    return np.array(anc)


@pytest.mark.parametrize("n", [1, 2, 3, 7, 64, 257, 1000])
def test_systematic_matches_slow_restatement(n):
    r = np.random.default_rng(n)
    lw = r.normal(0, 3, n).astype(np.float32)
    u = int(r.integers(0, 2 ** 32))
    anc, _ = O.systematic(lw, lw.max(), u)
    np.testing.assert_array_equal(anc, _slow_systematic(lw, lw.max(), u))


def test_systematic_agrees_with_float64_cdf_search():
    """Away from exact ties the integer predicate reproduces the
    reference's FP64 search (resampling.cu:143-158)."""
    r = np.random.default_rng(7)
    n = 5000
    lw = r.normal(0, 2, n)
    anc = O.pf_systematic_ancestors(lw, 12345)
    w = np.exp(lw - lw.max())
    cdf = np.cumsum(w / w.sum())
    u0 = (12345 % 1000000) / (1000000.0 * n)
    target = (u0 + np.arange(n)) / n
    ref = np.minimum(np.searchsorted(cdf, target, side="left"), n - 1)
    assert np.mean(anc == ref) > 0.999


def test_systematic_offspring_counts_are_floor_or_ceil():
    """Systematic resampling gives every particle floor(N w) or ceil(N w)
    offspring (up to quantisation of w)."""
    r = np.random.default_rng(3)
    n = 4096
    lw = r.normal(0, 1.5, n).astype(np.float32)
    anc, W = O.systematic(lw, lw.max(), int(r.integers(0, 2 ** 32)))
    q = O.quantize(lw, lw.max()).astype(np.float64)
    expect = n * q / q.sum()
    cnt = np.bincount(anc, minlength=n)
    assert np.all(cnt >= np.floor(expect) - 1) and np.all(cnt <= np.ceil(expect) + 1)
    assert np.all(np.diff(anc) >= 0)


def test_quantiser_properties():
    n = 1 << 20
    K = O.quant_exponent(n)
    assert K == 40
    q = O.quantize(np.array([0.0, -0.5, -1.0, -27.0, -28.0, -100.0, np.nan], np.float32), 0.0)
    assert q[0] == 1 << K
    assert q[0] > q[1] > q[2] > q[3] > 0
    assert q[5] == 0 and q[6] == 0
    assert abs(q[2] / q[0] - np.exp(-1.0)) < 2e-6


# ----------------------------------------------------------- megopolis
def test_megopolis_prefers_heavy_particles():
    n = 2000
    lw = np.full(n, -10.0, np.float32)
    lw[: n // 4] = 0.0
    anc = O.megopolis(lw, 32, seed=5, epoch=0)
    frac = np.mean(anc < n // 4)
    # weight mass of the first quarter: 500 / (500 + 1500 e^-10) ~ 1
    assert frac > 0.99


def test_reference_megopolis_chain_prefers_heavy_particles():
    n = 2000
    lw = np.full(n, -10.0)
    lw[: n // 4] = 0.0
    anc = O.pf_megopolis_ref_ancestors(lw, 20, 12345)
    assert np.mean(anc < n // 4) > 0.9


# ------------------------------------------------ device-filter likelihoods
def _outlier_case(n_out, n_sat=5):
    sats = TOKYO_SATS[:n_sat]
    pr = np.linalg.norm(sats - TOKYO_TRUE_POS, axis=1) + TOKYO_TRUE_CB
    pr[:n_out] += 100.0
    return np.column_stack([sats, pr, np.ones(n_sat)])


def _generic(rows, x=None, **kw):
    x = np.zeros((4, 1)) if x is None else x
    lw, _ = O.weight_generic(x, TOKYO_TRUE_POS, [TOKYO_TRUE_CB], np.eye(3), rows, 5.0, **kw)
    return lw


def test_generic_gaussian_and_huber_match_pinned_oracle():
    """weight_generic agrees with the C oracle (pinned against the
    reference) on a cloud of particles, Gaussian and Huber."""
    rng = np.random.default_rng(5)
    x = np.vstack([rng.normal(0, 30, (3, 500)), rng.normal(0, 20, (1, 500))])
    rows = np.column_stack([TOKYO_SATS, TOKYO_PR, rng.uniform(0.5, 2.0, len(TOKYO_PR))])
    clk = np.zeros(len(rows), np.int32)
    for kind, mode in (("gaussian", 0), ("huber", 1)):
        want = O.weight(x, TOKYO_TRUE_POS, [TOKYO_TRUE_CB], np.eye(3), rows, clk, 5.0, mode=mode, huber_k=1.5)
        got, _ = O.weight_generic(x, TOKYO_TRUE_POS, [TOKYO_TRUE_CB], np.eye(3), rows, 5.0, kind=kind, huber_k=1.5)
        np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-7)


def test_generic_known_answers():
    """A 100 m outlier at sigma 5 (reference tests/test_cuda_streams.py:
    668-693 for Gaussian / Huber, 569-600 for the gate); Student's t and the
    GMM from their closed forms (pf_device.cu:265-266, 415-428)."""
    one = _outlier_case(1)
    assert _generic(one, kind="gaussian")[0] == pytest.approx(-200.0, abs=1e-6)
    assert _generic(one, kind="huber", huber_k=1.5)[0] == pytest.approx(-28.875, abs=1e-6)
    assert _generic(one, kind="student_t", nu=4.0)[0] == pytest.approx(-2.5 * np.log(101.0), abs=1e-9)
    a = np.log(0.7) - np.log(5.0)
    gmm_clean = np.logaddexp(a, np.log(0.3) - np.log(30.0) - 0.5 * 15.0 ** 2 / 900.0)
    gmm_out = np.logaddexp(a - 0.5 * 100.0 ** 2 / 25.0, np.log(0.3) - np.log(30.0) - 0.5 * 85.0 ** 2 / 900.0)
    want = 4 * gmm_clean + gmm_out
    got = _generic(one, kind="gmm", w_los=0.7, mu_nlos=15.0, sigma_nlos=30.0)[0]
    assert got == pytest.approx(want, abs=1e-6)
    # gate: one outlier of five is dropped, five of five keep the gate off
    assert abs(_generic(one, kind="gaussian", gate_m=30.0)[0]) < 1e-6
    assert _generic(_outlier_case(5), kind="gaussian", gate_m=30.0)[0] < -900.0
    # two outliers of five: three inside < min(5, 4), gate off
    assert _generic(_outlier_case(2), kind="gaussian", gate_m=30.0)[0] == pytest.approx(-400.0, abs=1e-6)
    # three satellites: min(3, 4) = 3 must stay inside
    assert _generic(_outlier_case(1, 3), kind="gaussian", gate_m=30.0)[0] == pytest.approx(-200.0, abs=1e-6)


def test_generic_weight_zero_satellite_contributes_nothing():
    rows = _outlier_case(1)
    rows[0, 4] = 0.0
    for kind in ("gaussian", "student_t", "huber", "gmm"):
        full = _generic(rows, kind=kind, nu=3.0)
        drop = _generic(rows[1:], kind=kind, nu=3.0)
        assert full[0] == pytest.approx(drop[0], abs=1e-12)


# ------------------------------------ differenced / carrier-phase terms
def _dd_case(outlier, carrier=False):
    """Receiver at the ECEF origin, base 120/-35/18 m away, 5 satellites
    20,000 km out; pair 0 carries the outlier (reference
    tests/test_cuda_streams.py:600-660, 694-773)."""
    rng = np.random.RandomState(123)
    d = rng.randn(5, 3)
    sats = d / np.linalg.norm(d, axis=1, keepdims=True) * 20_000_000.0
    rover = np.zeros(3)
    base = np.array([120.0, -35.0, 18.0])
    rr = np.linalg.norm(sats - rover, axis=1)
    br = np.linalg.norm(sats - base, axis=1)
    dd = (rr[1:] - rr[0]) - (br[1:] - br[0])
    wl = np.full(4, 0.190293673)
    if carrier:
        dd = dd / wl
    dd[0] += outlier
    return dict(sat_k=sats[1:], sat_ref=np.repeat(sats[[0]], 4, axis=0), obs=dd, weight=np.ones(4),
                base_k=br[1:], base_ref=np.repeat(br[0], 4), wavelength=wl)


def _obs(kind, case, **kw):
    lw, _ = O.obs_term(np.zeros((4, 1)), np.zeros(3), [0.0], np.eye(3), kind, **case, **kw)
    return lw[0]


def test_obs_term_known_answers():
    pr = _dd_case(50.0)
    assert _obs(O.OBS_DD_PSEUDORANGE, pr, sigma=0.5) == pytest.approx(-5000.0, rel=1e-9)
    assert _obs(O.OBS_DD_PSEUDORANGE, pr, sigma=0.5, huber_k=1.5) == pytest.approx(-148.875, rel=1e-9)
    assert abs(_obs(O.OBS_DD_PSEUDORANGE, pr, sigma=0.5, gate=10.0)) < 1e-6
    cp = _dd_case(0.45, carrier=True)
    assert _obs(O.OBS_DD_CARRIER_AFV, cp, sigma=0.05) == pytest.approx(-40.5, abs=1e-6)
    assert _obs(O.OBS_DD_CARRIER_AFV, cp, sigma=0.05, huber_k=1.5) == pytest.approx(-12.375, abs=1e-6)
    assert abs(_obs(O.OBS_DD_CARRIER_AFV, cp, sigma=0.05, gate=0.3)) < 1e-6
    # integer cycle slips leave the fractional residual unchanged
    slip = dict(cp, obs=cp["obs"] + np.array([0.0, 7.0, -3.0, 120.0]))
    assert _obs(O.OBS_DD_CARRIER_AFV, slip, sigma=0.05) == pytest.approx(-40.5, abs=1e-6)
    # undifferenced carrier at the true clock: only the planted fraction costs
    rng = np.random.RandomState(123)
    d = rng.randn(5, 3)
    sats = d / np.linalg.norm(d, axis=1, keepdims=True) * 20_000_000.0
    wl = np.full(5, 0.190293673)
    cb = 100.0
    cyc = (np.linalg.norm(sats, axis=1) + cb) / wl + np.array([0.2, 3.0, -8.0, 0.0, 1e6])
    lw, _ = O.obs_term(np.zeros((4, 1)), np.zeros(3), [cb], np.eye(3), O.OBS_CARRIER_AFV, sat_k=sats, obs=cyc,
                       weight=np.ones(5), wavelength=wl, sigma=0.05)
    assert lw[0] == pytest.approx(-0.5 * 0.2 ** 2 / 0.05 ** 2, abs=1e-5)


# ---------------------------------------------- velocity states, Doppler
L1 = 0.19029367279836488


def doppler_case():
    """Receiver, satellites and a known receiver velocity and clock drift
    (reference tests/test_cuda_streams.py:61-88)."""
    rx = np.array([-3957199.0, 3310205.0, 3737911.0])
    true_vel = np.array([0.3, -0.5, 0.8])
    sat = np.array([[-14985000.0, -3988000.0, 21474000.0], [-9575000.0, 15498000.0, 19457000.0],
                    [7624000.0, -16218000.0, 19843000.0], [16305000.0, 12037000.0, 17183000.0],
                    [-20889000.0, 13759000.0, 8291000.0], [5463000.0, 24413000.0, 8934000.0]])
    sv = np.array([[1200.0, -2800.0, 500.0], [-800.0, 1500.0, -2700.0], [2500.0, 1800.0, -900.0],
                   [-1100.0, -2200.0, 2100.0], [600.0, 2900.0, 1300.0], [-2600.0, 400.0, -1800.0]])
    los = (sat - rx) / np.linalg.norm(sat - rx, axis=1)[:, None]
    dop = -(np.sum((sv - true_vel) * los, axis=1) + 5.0) / L1
    return rx, sat, sv, dop, true_vel


def test_doppler_oracle_known_answers():
    """The reference's Doppler tests (tests/test_cuda_streams.py:285-337):
    WLS blend with gain 1 recovers the velocity to 1e-3, the velocity KF
    from sigma 10 to 2e-2 with the variances shrinking."""
    rx, sat, sv, dop, tv = doppler_case()
    pos = np.tile(rx, (4, 1))
    _, v, _ = O.doppler(pos, np.zeros((4, 3)), np.zeros((4, 9)), sat, sv, dop, np.ones(6), L1, 0.5, gain=1.0,
                        max_update=100.0)
    np.testing.assert_allclose(v, np.tile(tv, (4, 1)), atol=1e-3)
    lw, v, P = O.doppler(pos, np.zeros((4, 3)), np.tile(100.0 * np.eye(3).ravel(), (4, 1)), sat, sv, dop, np.ones(6),
                         L1, 0.5, kf=True)
    np.testing.assert_allclose(v, np.tile(tv, (4, 1)), atol=2e-2)
    assert np.all(P[:, [0, 4, 8]] < 100.0) and np.all(P[:, [0, 4, 8]] > 0.0)
    # the likelihood prefers the true velocity
    lw_true, _, _ = O.doppler(pos[:1], tv[None], np.zeros((1, 9)), sat, sv, dop, np.ones(6), L1, 0.5)
    lw_off, _, _ = O.doppler(pos[:1], (tv + 1.0)[None], np.zeros((1, 9)), sat, sv, dop, np.ones(6), L1, 0.5)
    assert lw_true[0] == pytest.approx(0.0, abs=1e-9) and lw_off[0] < -1.0


def test_velocity_predict_oracle_known_answers():
    """Reference tests/test_cuda_streams.py:239-283: the guide becomes every
    particle's velocity and moves it by v dt; in KF mode the positions spread
    by sqrt(sigma_pos^2 + dt^2 var) and the variances grow by q dt."""
    n = 400
    pos, v, P = O.vel_predict(np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 9)), [2.0, -1.0, 0.5], 0.25, 0.0, 0.0,
                              1.0, False, 0.0, 1, 42)
    np.testing.assert_allclose(pos, np.tile([0.5, -0.25, 0.125], (n, 1)), atol=1e-12)
    np.testing.assert_allclose(v, np.tile([2.0, -1.0, 0.5], (n, 1)))
    P0 = np.tile(4.0 * np.eye(3).ravel(), (n, 1))
    pos, v, P = O.vel_predict(np.zeros((n, 3)), np.tile([1.0, 0, 0], (n, 1)), P0, [1.0, 0.0, 0.0], 1.0, 1.0, 100.0,
                              1.0, True, 0.5, 1, 42)
    np.testing.assert_allclose(v, np.tile([1.0, 0.0, 0.0], (n, 1)))
    assert 1.9 < np.std(pos[:, 0] - 1.0) < 2.6 and 1.9 < np.std(pos[:, 1]) < 2.6
    np.testing.assert_allclose(P[:, [0, 4, 8]], 4.5)
