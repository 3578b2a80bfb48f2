"""The NLOS network's tensor-core kernels (through the C ABI) against the
FP64 oracle with the same BF16 rounding points."""
import ctypes as C

import numpy as np
import pytest

from gnss_gpu_b200 import _native as N
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def _dev(a, torch):
    return torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda")


def _data(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.normal(0, 1, (n, M.FEAT)).astype(np.float32)
    nl = (X[:, 0] + 0.5 * X[:, 1] + 0.3 * rng.normal(0, 1, n) > 0.3).astype(np.float32)
    b = np.where(nl > 0, 10.0 + 15.0 * np.abs(X[:, 2]), 0.0).astype(np.float32)
    return X, np.column_stack([nl, b]).astype(np.float32)


def test_param_count_matches_oracle():
    assert N.load().pf_mlp_param_count() == M.N_PARAMS


def test_forward_matches_oracle():
    import torch
    L = N.load()
    X, _ = _data(1000, 1)
    prm = M.init_params(2)
    out = torch.zeros(2 * len(X), device="cuda")
    dx, dp = _dev(X, torch), _dev(prm, torch)  # keep the buffers alive across the call
    N.check(L.pf_mlp_forward(dx.data_ptr(), len(X), dp.data_ptr(), out.data_ptr(), None))
    torch.cuda.synchronize()
    o = out.cpu().numpy().reshape(-1, 2)
    p, mu = M.predict(prm, X)
    assert np.max(np.abs(o[:, 0] - p)) < 2e-3
    assert np.max(np.abs(o[:, 1] - mu) / np.maximum(1.0, mu)) < 2e-3


@pytest.mark.parametrize("n", [1, 100, 4096, 20_000])
def test_gradient_matches_oracle(n):
    import torch
    L = N.load()
    X, Y = _data(n, 5 + n)
    prm = M.init_params(7)
    grad = torch.zeros(M.N_PARAMS, device="cuda")
    loss = torch.zeros(1, device="cuda")
    scratch = torch.zeros(L.pf_mlp_scratch_bytes(), dtype=torch.uint8, device="cuda")
    dx, dy, dp = _dev(X, torch), _dev(Y, torch), _dev(prm, torch)
    N.check(L.pf_mlp_grad(dx.data_ptr(), dy.data_ptr(), n, dp.data_ptr(), grad.data_ptr(), loss.data_ptr(),
                          scratch.data_ptr(), scratch.numel(), None))
    torch.cuda.synchronize()
    g = grad.cpu().numpy().astype(np.float64)
    lo, go = M.loss_grad(prm, X, Y, bf=True)
    assert float(loss.item()) == pytest.approx(lo, rel=2e-3)
    scale = np.abs(go).max()
    err = np.abs(g - go)
    # FP32 accumulation in a different order on BF16-rounded operands; an
    # occasional BF16 rounding of a backward signal can differ by one ulp
    assert np.max(err) <= 2e-2 * scale, (np.max(err), scale)
    assert np.mean(err) <= 1e-3 * scale
    # and close to the unrounded FP64 gradient
    _, g64 = M.loss_grad(prm, X, Y, bf=False)
    assert np.linalg.norm(g - g64) <= 5e-2 * np.linalg.norm(g64)


def test_adam_training_lowers_loss():
    import torch
    L = N.load()
    X, Y = _data(16_384, 11)
    prm = _dev(M.init_params(1), torch)
    m = torch.zeros_like(prm)
    v = torch.zeros_like(prm)
    loss = torch.zeros(1, device="cuda")
    scratch = torch.zeros(L.pf_mlp_scratch_bytes(), dtype=torch.uint8, device="cuda")
    dx, dy = _dev(X, torch), _dev(Y, torch)
    losses = []
    for step in range(1, 301):
        N.check(L.pf_mlp_adam_step(dx.data_ptr(), dy.data_ptr(), len(X), prm.data_ptr(), m.data_ptr(), v.data_ptr(),
                                   step, C.c_float(3e-3), loss.data_ptr(), scratch.data_ptr(), scratch.numel(), None))
        if step in (1, 300):
            torch.cuda.synchronize()
            losses.append(float(loss.item()))
    assert losses[1] < 0.5 * losses[0], losses
    # the trained network separates the classes
    p, _ = M.predict(prm.cpu().numpy(), X)
    acc = np.mean((p > 0.5) == (Y[:, 0] > 0.5))
    assert acc > 0.85, acc
