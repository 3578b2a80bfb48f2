"""The NLOS network's FP64 oracle: analytic gradient against finite
differences (no BF16 rounding), and BF16 rounding itself."""
import numpy as np

from oracle import mlp_oracle as M


def _data(n=64, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.normal(0, 1, (n, M.FEAT))
    Y = np.column_stack([rng.random(n) < 0.3, rng.exponential(20.0, n)]).astype(np.float64)
    return X, Y


def test_gradient_matches_finite_differences():
    X, Y = _data()
    prm = M.init_params(3).astype(np.float64)
    _, g = M.loss_grad(prm, X, Y, bf=False)
    rng = np.random.default_rng(1)
    idx = np.concatenate([rng.choice(np.arange(M.OFF_W1, M.OFF_B1).reshape(M.H, M.IN)[:, :M.FEAT].ravel(), 8),
                          rng.integers(M.OFF_B1, M.N_PARAMS, 24)])
    for i in idx:
        h = 1e-6
        p1, p2 = prm.copy(), prm.copy()
        p1[i] += h
        p2[i] -= h
        fd = (M.loss_only(p1, X, Y) - M.loss_only(p2, X, Y)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_nearest_even():
    # BF16 keeps 7 mantissa bits: spacing 2^-7 just above 1
    x = np.array([1.0, 1 + 2 ** -8, 1 + 2 ** -9, 1 + 3 * 2 ** -9, 1 + 3 * 2 ** -8, -3.0e-3, 65504.0], np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                    # halfway, ties to the even mantissa
    assert r[2] == 1.0                    # below halfway
    assert r[3] == 1 + 2 ** -7            # above halfway
    assert r[4] == 1 + 2 ** -6            # halfway between odd and even: to even
    assert abs(r[5] + 3.0e-3) < 3.0e-3 * 2 ** -8
    assert r[6] == 65536.0
