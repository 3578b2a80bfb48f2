"""pf_compute_ess_noalloc: the entry point for callers that cannot call
cudaMalloc -- real-time loops that must not allocate after start-up, hosts
whose device memory belongs to another allocator.  It takes caller-owned device input and output and keeps
its scratch in a fixed device array of the library.

This file is collected last on purpose (its name sorts after the others), so
a run that stops at the first failure has already run every other test.  The
test passes alone in a fresh process and after the other tests: every call
clears the shared ticket itself.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ess_noalloc(lib, lw_host, torch):
    d_lw = torch.from_numpy(np.ascontiguousarray(lw_host, np.float64)).cuda()
    d_out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    st = lib.pf_compute_ess_noalloc(C.c_void_p(d_lw.data_ptr()), len(lw_host), C.c_void_p(d_out.data_ptr()),
                                    C.c_void_p(stream.cuda_stream))
    assert st == 0, lib.pf_last_error().decode()
    stream.synchronize()
    return float(d_out.item())


def test_noalloc_ess_matches_pf_compute_ess_on_two_calls_in_a_row():
    import torch
    from gnss_gpu_b200 import _native as N
    from gnss_gpu_b200 import _gnss_gpu_pf as pfm

    lib = N.load()
    r = np.random.default_rng(2024)
    # two calls in a row with different sizes and weights: the second must not
    # see anything left in the shared scratch by the first
    cases = [r.normal(0.0, 3.0, 1_000_003), r.normal(-50.0, 0.5, 70_001)]
    for lw in cases:
        got = _ess_noalloc(lib, lw, torch)
        want = pfm.pf_compute_ess(lw, len(lw))   # the existing, allocating entry point
        assert got == pytest.approx(want, rel=1e-12), (got, want)


def test_noalloc_ess_at_its_limit_and_without_allocating():
    """n = PF_NOALLOC_MAX_PARTICLES fills every row of the scratch array (the
    last block writes the last row).  A warmed-up call must leave the
    device's free memory unchanged: the entry point allocates nothing."""
    import torch
    from gnss_gpu_b200 import _native as N
    from gnss_gpu_b200 import _gnss_gpu_pf as pfm

    lib = N.load()
    n = N.PF_NOALLOC_MAX_PARTICLES
    lw = np.random.default_rng(7).normal(-3.0, 2.0, n)
    d_lw = torch.from_numpy(lw).cuda()
    d_out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()

    def call():
        st = lib.pf_compute_ess_noalloc(C.c_void_p(d_lw.data_ptr()), n, C.c_void_p(d_out.data_ptr()),
                                        C.c_void_p(stream.cuda_stream))
        assert st == 0, lib.pf_last_error().decode()
        stream.synchronize()

    call()  # warm-up: module load and the one-time symbol lookup
    free_before, _ = torch.cuda.mem_get_info()
    call()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before, (free_before, free_after)
    want = pfm.pf_compute_ess(lw, n)
    assert float(d_out.item()) == pytest.approx(want, rel=1e-12)


def test_noalloc_ess_rejects_sizes_beyond_its_scratch():
    import torch
    from gnss_gpu_b200 import _native as N

    lib = N.load()
    n = N.PF_NOALLOC_MAX_PARTICLES + 1
    d = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = lib.pf_compute_ess_noalloc(C.c_void_p(d.data_ptr()), n, C.c_void_p(d.data_ptr()), None)
    assert st == N.PF_ECAP
    assert b"no-allocation limit" in lib.pf_last_error()
