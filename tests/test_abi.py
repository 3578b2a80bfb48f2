"""CPU tests of the C ABI: the library loads, exports every function that
include/gnss_pf_b200.h declares, and its record layouts match the header.
(No compute call: this environment may have no GPU.)"""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "gnss_pf_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_\s\*]*?\b((?:pf|pfe)_[A-Za-z0-9_]+)\s*\(", text, re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from gnss_gpu_b200 import build, _native
    build.build()
    return _native.load()


def test_header_declares_the_reference_functions():
    names = declared_functions()
    for ref_name in ["pf_initialize", "pf_predict", "pf_weight", "pf_compute_ess", "pf_resample_systematic",
                     "pf_resample_megopolis", "pf_estimate", "pf_get_particles"]:
        assert ref_name in names


def test_library_exports_every_declared_function(lib):
    from gnss_gpu_b200 import _native
    out = subprocess.run(["nm", "-D", "--defined-only", str(_native.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        getattr(lib, n)  # resolvable through ctypes


def test_python_binding_covers_every_declared_function():
    from gnss_gpu_b200 import _native
    assert set(declared_functions()) <= set(_native.EXPORTED)


def test_record_layouts(lib):
    from gnss_gpu_b200 import _native as N
    assert C.sizeof(N.FilterEpoch) == 40 and C.sizeof(N.Sat) == 56
    assert C.sizeof(N.EngineConfig) == 56
    assert C.sizeof(N.FilterParams) == 56
    assert lib.pf_abi_version() == 2
    assert lib.pf_last_error() == b""


def test_workspace_size_and_validation_without_gpu(lib):
    """pfe_workspace_bytes is host-only: sizes and argument checks."""
    from gnss_gpu_b200 import _native as N
    cfg = N.EngineConfig(n_filters=2, n_clk=4, resampler=0, megopolis_iters=32, weight_mode=0, lw_mode=0,
                         sys_offset=0, max_sats=32, obs_slots=4, flags=3, ess_threshold=0.5, huber_k=1.5)
    fp = (N.FilterParams * 2)()
    for k, n in enumerate([1_000_000, 5]):
        fp[k].n_particles = n
        fp[k].seed = 1
        for a in range(3):
            fp[k].sigma_pos[a] = 1.0
        fp[k].sigma_clk = 0.5
        fp[k].sigma_pr = 3.0
    b = C.c_size_t(0)
    assert lib.pfe_workspace_bytes(C.byref(cfg), fp, C.byref(b)) == N.PF_OK
    # two 7-component FP32 state buffers dominate: 2 * 7 * 4 B per particle
    assert b.value > 2 * 7 * 4 * 1_000_000
    cfg.max_sats = 65
    assert lib.pfe_workspace_bytes(C.byref(cfg), fp, C.byref(b)) == N.PF_ECAP
    assert b"max_sats" in lib.pf_last_error()
    cfg.max_sats = 32
    fp[1].sigma_pr = 0.0
    assert lib.pfe_workspace_bytes(C.byref(cfg), fp, C.byref(b)) == N.PF_EINVAL
    fp[1].sigma_pr = 3.0
    cfg.n_clk = 5
    assert lib.pfe_workspace_bytes(C.byref(cfg), fp, C.byref(b)) == N.PF_EINVAL


def test_particle_filter_raises_before_initialize(lib):
    """particle_filter.py:112-113,141-142,185-186 of the reference: calls on an
    uninitialised filter raise RuntimeError (no GPU touched)."""
    from gnss_gpu_b200 import ParticleFilter
    pf = ParticleFilter(n_particles=100, seed=12345)
    for call in (pf.predict, pf.estimate, pf.get_ess, pf.get_particles):
        with pytest.raises(RuntimeError):
            call()
    with pytest.raises(RuntimeError):
        pf.update(__import__("numpy").zeros((1, 3)), [1.0])
