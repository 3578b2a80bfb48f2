"""The oracle's restatements of the device filter's likelihoods against the
reference's own device code: tests/golden/ref_device_fixtures.npz holds the
log-weights (and Doppler velocity states) that the reference's
_gnss_gpu_pf_device module (src/particle_filter/pf_device.cu,
python/gnss_gpu/_pf_device_bindings.cpp) produced on a B200 for seeded
particle sets (tests/golden/make_ref_device_fixtures.py).  The particles are
given to the oracle in ECEF (anchor 0, identity frame).

Tolerances: 1e-8 relative for the pseudorange and Doppler terms (FP64 on
both sides); 1e-6 for the carrier-phase AFV terms, whose phases are about
1e8 cycles, so the order of FP64 operations shows at 1e-8 cycles."""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

FX = np.load(Path(__file__).resolve().parent / "golden" / "ref_device_fixtures.npz")
ST = FX["states"]
X = np.vstack([ST[:, 0], ST[:, 1], ST[:, 2], ST[:, 3]])
A0, ROT, CA = np.zeros(3), np.eye(3), np.zeros(4)
WL = 0.190293673


def rel(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b))))


@pytest.mark.parametrize("name,kw", [
    ("gauss", {}),                                            # pf_device.cu:273-275
    ("student_t", dict(kind="student_t", nu=4.0)),           # pf_device.cu:265-266
    ("huber", dict(kind="huber", huber_k=1.5)),               # pf_device.cu:19-26,267-268
    ("gate", dict(gate_m=15.0)),                              # pf_device.cu:236-258
    ("gmm", dict(kind="gmm")),                                # pf_device.cu:415-428
])
def test_pseudorange_likelihoods_match_reference_device(name, kw):
    rows = np.column_stack([FX["sat"], FX["pr"], FX["w"]])
    lw, _ = O.weight_generic(X, A0, CA, ROT, rows, 5.0, **kw)
    assert rel(lw, FX["lw_" + name]) < 1e-8


def test_carrier_afv_matches_reference_device():  # pf_device.cu:439-494
    lw, _ = O.obs_term(X, A0, CA, ROT, O.OBS_CARRIER_AFV, FX["sat"], FX["cp"], FX["w"],
                       wavelength=np.full(len(FX["cp"]), WL), sigma=0.05)
    assert rel(lw, FX["lw_carrier_afv"]) < 1e-6


@pytest.mark.parametrize("name,kind,sigma,kw,tol", [
    ("dd_pr", O.OBS_DD_PSEUDORANGE, 2.0, {}, 1e-8),                                       # pf_device.cu:282-368
    ("dd_pr_gate_huber", O.OBS_DD_PSEUDORANGE, 2.0, dict(gate=10.0, huber_k=1.5), 1e-8),
    ("dd_carrier", O.OBS_DD_CARRIER_AFV, 0.05, {}, 1e-6),                                 # pf_device.cu:496-604
    ("dd_carrier_gate_huber", O.OBS_DD_CARRIER_AFV, 0.05, dict(gate=0.3, huber_k=1.5), 1e-6),
])
def test_double_differences_match_reference_device(name, kind, sigma, kw, tol):
    obs = FX["dd"] if kind == O.OBS_DD_PSEUDORANGE else FX["ddc"]
    wl = None if kind == O.OBS_DD_PSEUDORANGE else FX["dd_wl"]
    lw, _ = O.obs_term(X, A0, CA, ROT, kind, FX["dd_sat_k"].reshape(-1, 3), obs, FX["w_dd"],
                       sat_ref=FX["dd_ref"].reshape(-1, 3), base_k=FX["dd_base_k"], base_ref=FX["dd_base_ref"],
                       wavelength=wl, sigma=sigma, **kw)
    assert rel(lw, FX["lw_" + name]) < tol


@pytest.mark.parametrize("kf", [False, True])  # pf_device.cu:610-748 and 750-887
def test_doppler_matches_reference_device(kf):
    pos, v, P = ST[:, :3], ST[:, 4:7], ST[:, 7:16]
    kw = dict(kf=True) if kf else dict(gain=0.25, max_update=10.0)
    lw, v2, P2 = O.doppler(pos, v, P, FX["sat"], FX["sat_vel"], FX["doppler_hz"], FX["w"], WL, 0.5, **kw)
    out = FX["states_doppler_kf" if kf else "states_doppler"]
    assert rel(lw, FX["lw_doppler_kf" if kf else "lw_doppler"]) < 1e-8
    assert np.max(np.abs(v2 - out[:, 4:7])) < 1e-9
    assert np.max(np.abs(P2 - out[:, 7:16])) < 1e-9
