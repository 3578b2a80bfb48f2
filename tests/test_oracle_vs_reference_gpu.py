"""CPU tests: the oracle against outputs of the reference's OWN GPU module
(src/particle_filter/*.cu + _particle_filter_bindings.cpp of the reference,
compiled by oracle/build_ref.py and run on a B200 by
tests/golden/make_ref_gpu_fixtures.py), and the project's Philox against
cuRAND words (tests/golden/make_curand_fixture.py)."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

G = Path(__file__).parent / "golden"
FIX = G / "ref_gpu_fixtures.npz"

pytestmark = pytest.mark.skipif(not FIX.exists(), reason="reference GPU fixtures not generated")


@pytest.fixture(scope="module")
def ref():
    return np.load(FIX)


@pytest.fixture(scope="module")
def scen():
    fx = json.loads((G / "tokyo_fixture.json").read_text())
    return np.array(fx["sat_ecef"]), np.array(fx["pseudoranges"])


CASES = [0, 1, 2]


@pytest.mark.parametrize("c", CASES)
def test_weight_matches_reference_gpu(ref, scen, c):
    sat, pr = scen
    px, py, pz, pcb, ws = (ref[f"c{c}_{k}"] for k in ("px", "py", "pz", "pcb", "wsat"))
    lw = O.pf_weight(px, py, pz, pcb, sat, pr, ws, 5.0)
    want = ref[f"c{c}_lw"]
    # FP64 on both sides; the residual pr - |sat - p| - cb cancels ~2e7 m
    assert np.max(np.abs(lw - want) / np.maximum(1.0, np.abs(want))) < 1e-8


@pytest.mark.parametrize("c", CASES)
def test_ess_and_estimate_match_reference_gpu(ref, c):
    lw = ref[f"c{c}_lw"]
    assert O.pf_ess(lw) == pytest.approx(float(ref[f"c{c}_ess"]), rel=1e-12)
    px, py, pz, pcb = (ref[f"c{c}_{k}"] for k in ("px", "py", "pz", "pcb"))
    est = O.pf_estimate(px, py, pz, pcb, lw)
    np.testing.assert_allclose(est, ref[f"c{c}_est"], rtol=0, atol=1e-6)


@pytest.mark.parametrize("c", CASES)
def test_get_particles_layout_matches_reference_gpu(ref, c):
    parts = ref[f"c{c}_particles"].reshape(-1, 4)
    for j, k in enumerate(("px", "py", "pz", "pcb")):
        np.testing.assert_array_equal(parts[:, j], ref[f"c{c}_{k}"])


@pytest.mark.parametrize("c", CASES)
def test_systematic_ancestors_match_reference_gpu(ref, c):
    """The exact integer predicate on 2^40-scaled weights reproduces the
    reference's FP64 thrust-scan search (resampling.cu:143-158) slot for slot
    (a tie would need a CDF value within ~1e-12 of a target)."""
    lw = ref[f"c{c}_lw"]
    anc = O.pf_systematic_ancestors(lw, 12345)
    np.testing.assert_array_equal(anc, ref[f"c{c}_sys_anc"])


@pytest.mark.parametrize("c", CASES)
def test_reference_megopolis_offspring_distribution(ref, c):
    """The reference's Megopolis (cuRAND draws) and the oracle's restatement
    of the same chain (Philox draws) give offspring counts from the same
    distribution (two-sample KS, p > 0.01)."""
    from scipy import stats
    lw = ref[f"c{c}_lw"]
    n = len(lw)
    got = np.bincount(O.pf_megopolis_ref_ancestors(lw, 15, 12345), minlength=n)
    want = np.bincount(ref[f"c{c}_mego_anc"], minlength=n)
    assert stats.ks_2samp(got, want).pvalue > 0.01


def test_reference_ess_known_cases(ref):
    assert float(ref["ess_uniform_10000"]) == pytest.approx(10_000)
    assert float(ref["ess_dominant_1000"]) < 2.0
    assert O.pf_ess(np.zeros(10_000)) == pytest.approx(float(ref["ess_uniform_10000"]), rel=1e-12)
    dom = np.full(1000, -1000.0)
    dom[0] = 0.0
    assert O.pf_ess(dom) == pytest.approx(float(ref["ess_dominant_1000"]), rel=1e-12)
