"""Allocation failures made on the host (pf_test_fail_alloc): the call that
meets one returns PF_ENOMEM with a message, releases what it had allocated,
and the library keeps working.  No GPU fault is involved: the failure is
decided before the allocation is attempted."""
import numpy as np
import pytest

from gnss_gpu_b200 import _native as N
from gnss_gpu_b200 import scenario as S

import pfhelp as H

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nth", [1, 2, 3])
def test_engine_creation_survives_an_allocation_failure(nth):
    lib = N.load()
    assert lib.pf_test_fail_alloc(nth) == 0
    try:
        with pytest.raises(RuntimeError, match="injected") as ei:
            H.make_engine([4096], n_clk=4)
        assert ei.value.status == N.PF_ENOMEM
    finally:
        lib.pf_test_fail_alloc(0)
    # the next engine is created and steps normally
    tr = S.config1(n_epochs=2)
    eng = H.make_engine([4096], n_clk=4)
    eng.initialize(0, tr.anchor, tr.truth_clk[0], 10.0, 30.0)
    fe, sv = eng.pack_epoch([{"disp": tr.disp_enu[0], "sats": tr.sats[0], "pr": tr.pr[0], "clk": tr.clk_idx[0]}])
    eng.upload(0, fe, sv)
    eng.step()
    assert np.all(np.isfinite(eng.results()[0]["est_ecef"]))
    eng.close()


def test_stateless_workspace_growth_survives_an_allocation_failure():
    from gnss_gpu_b200 import _gnss_gpu_pf as pfm
    lib = N.load()
    n = 1 << 24  # larger than any other stateless call of the suite: the workspace must grow
    lw = np.random.default_rng(3).normal(-2.0, 1.5, n)
    assert lib.pf_test_fail_alloc(1) == 0
    try:
        with pytest.raises(RuntimeError, match="injected") as ei:
            pfm.pf_compute_ess(lw, n)
        assert ei.value.status == N.PF_ENOMEM
    finally:
        lib.pf_test_fail_alloc(0)
    w = np.exp(lw - lw.max())
    assert pfm.pf_compute_ess(lw, n) == pytest.approx(w.sum() ** 2 / (w ** 2).sum(), rel=1e-10)
