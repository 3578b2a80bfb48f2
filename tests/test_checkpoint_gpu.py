"""Checkpoint and resume of a filter (pfe_checkpoint_save / _load): a filter
restored into a fresh engine continues bit for bit like the uninterrupted
one -- the same states, log-weights, ancestors and estimates over the
following epochs, resampling included (the reference's closest facility,
pf_device_get/set_particle_states and get/set_log_weights in
include/gnss_gpu/pf_device.h:211-222, restores particles and weights only)."""
import numpy as np
import pytest

from gnss_gpu_b200 import _native as N
from gnss_gpu_b200 import scenario as S

import pfhelp as H

pytestmark = pytest.mark.gpu


def _rec(tr, t, flags):
    return {"disp": tr.disp_enu[t], "sats": tr.sats[t], "pr": tr.pr[t], "clk": tr.clk_idx[t], "flags": flags}


def _run(eng, tr, t0, t1, flags):
    out = []
    for t in range(t0, t1):
        fe, sv = eng.pack_epoch([_rec(tr, t, flags)])
        eng.upload(0, fe, sv)
        eng.step()
        x, lw = eng.state_f32(0, raw=True)
        r = eng.results()[0]
        out.append((x.copy(), lw.copy(), eng.ancestors(0).copy(), r["est_ecef"].copy(), r["est_clk"].copy(),
                    r["ess"], r["epoch"]))
    return out


@pytest.mark.parametrize("resampler", ["systematic", "megopolis"])
def test_resume_from_checkpoint_is_bit_exact(resampler):
    tr = S.config1(n_epochs=12)
    fl = N.PF_EP_PREDICT | N.PF_EP_WEIGHT | N.PF_EP_FORCE_RESAMPLE
    a = H.make_engine([20_000], n_clk=4, resampler=resampler, seeds=[777])
    a.initialize(0, tr.anchor, tr.truth_clk[0], 10.0, 30.0)
    _run(a, tr, 0, 5, fl)
    blob = a.checkpoint(0)
    want = _run(a, tr, 5, 10, fl)
    b = H.make_engine([20_000], n_clk=4, resampler=resampler, seeds=[777])
    b.restore(0, blob)
    got = _run(b, tr, 5, 10, fl)
    for w, g in zip(want, got):
        for wi, gi in zip(w, g):
            assert np.array_equal(np.asarray(wi), np.asarray(gi))
    a.close()
    b.close()


def test_checkpoint_rejects_mismatched_filters():
    tr = S.config1(n_epochs=2)
    a = H.make_engine([4096], n_clk=4, seeds=[5])
    a.initialize(0, tr.anchor, tr.truth_clk[0], 10.0, 30.0)
    blob = a.checkpoint(0)
    for ns, nclk, seed in [([4097], 4, 5), ([4096], 3, 5), ([4096], 4, 6)]:
        b = H.make_engine(ns, n_clk=nclk, seeds=[seed])
        with pytest.raises(ValueError):
            b.restore(0, blob)
        b.close()
    b = H.make_engine([4096], n_clk=4, seeds=[5])
    with pytest.raises(ValueError):
        b.restore(0, blob[:100])
    with pytest.raises(ValueError):
        b.restore(0, b"\0" * len(blob))
    with pytest.raises(RuntimeError):
        b.checkpoint(0)  # never initialized
    bad = bytearray(blob)
    bad[-4:] = (4096 + 5).to_bytes(4, "little", signed=True)  # last slot's ancestor out of range
    with pytest.raises(ValueError, match="ancestor"):
        b.restore(0, bytes(bad))
    b.close()
    a.close()
