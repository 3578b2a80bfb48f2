"""Offspring runs of every length class around the 128-slot segments.

Systematic resampling in the epoch kernel writes a run of up to 128 slots
slot by slot (lane) and a longer one (warp) as one marker word per 128-slot
segment it covers, plus the slots of the segments it covers in part.  The
filter's log-weights are set so that chosen particles get runs of 1, 63-65,
127-130, 255-257, ... slots and one run takes the rest, at filter sizes
whose last segment is partial.  Checked:

* the ancestors (host read, markers merged) equal the FP64 oracle's tiled
  integer CDF on the same log-weights and offset, slot for slot;
* the next step's device gather, which reads the markers, moves exactly
  state[ancestor] (no predict, no weight pass, no re-centring: the copy is
  bit-exact);
* a checkpoint taken after the resample restores into a fresh engine whose
  next gather gives the same states (the restore writes every slot and
  clears the markers).
"""
import numpy as np
import pytest

from gnss_gpu_b200 import _native as N
from gnss_gpu_b200 import scenario as S
from oracle import oracle as O

import pfhelp as H

pytestmark = pytest.mark.gpu

RUNS = [1, 2, 63, 64, 65, 127, 128, 129, 130, 255, 256, 257, 1000, 4095, 4096, 4097]


def _engine(n):
    eng = H.make_engine([n], lw_mode="accumulate", recenter=False)
    tr = S.config0()
    eng.initialize(0, tr.anchor, tr.truth_clk[0], 10.0, 30.0)
    return eng, tr


def _step(eng, tr, flags):
    fe, sv = eng.pack_epoch([{"disp": np.zeros(3), "sats": tr.sats[0], "pr": tr.pr[0], "clk": tr.clk_idx[0],
                              "flags": flags}])
    eng.upload(0, fe, sv)
    eng.step()


@pytest.mark.parametrize("n", [70_001, 131_075, 1_000_003])
def test_runs_around_segments_match_oracle_and_gather(n):
    rng = np.random.default_rng(n)
    eng, tr = _engine(n)
    st, _ = eng.state_f32(0)
    # particles and run lengths: the listed classes, one particle taking
    # the rest of the slots (a run over many whole segments)
    owners = np.sort(rng.choice(n, size=len(RUNS) + 1, replace=False))
    lengths = np.array(RUNS + [n - sum(RUNS)], np.float64)
    rng.shuffle(lengths)
    lw = np.full(n, -1e5, np.float32)
    lw[owners] = np.log(lengths).astype(np.float32)
    eng.set_state_f32(0, st, lw)
    _step(eng, tr, N.PF_EP_RESAMPLE_CHECK | N.PF_EP_FORCE_RESAMPLE)
    assert eng.results()[0]["resampled"]

    anc = eng.ancestors(0)
    u, W, _ = eng.resample_info(0)
    _, lw_raw = eng.state_f32(0, raw=True)
    want, w_want = O.systematic_tiled(lw_raw, u)[:2]
    assert np.array_equal(want, anc)
    assert W == w_want
    counts = np.bincount(anc, minlength=n)[owners]
    assert (counts > 128).sum() >= 8 and (counts <= 128).sum() >= 6, counts  # both write paths ran

    # the host export gathers through the merged ancestors
    x_host, _ = eng.state_f32(0)
    assert np.array_equal(x_host, st[:, anc])

    # a checkpoint of the resampled filter, restored into a fresh engine
    blob = eng.checkpoint(0)

    # the device gather of the next step reads the markers
    _step(eng, tr, 0)
    x_dev, _ = eng.state_f32(0, raw=True)
    assert np.array_equal(x_dev, st[:, anc])

    eng2, _ = _engine(n)
    eng2.restore(0, blob)
    assert np.array_equal(eng2.ancestors(0), anc)
    _step(eng2, tr, 0)
    x2, _ = eng2.state_f32(0, raw=True)
    assert np.array_equal(x2, st[:, anc])
