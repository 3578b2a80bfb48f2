"""The checked build (libgnsspf_b200_checked.so, -DPF_CHECKED) tests every
data-dependent index (ancestors of the gather, offspring-run ends, queued
chunk descriptors) before use and reports a bad one through the error word.
On valid inputs its checks must never fire and its results must equal the
release build's bit for bit: both run the same epochs, the checked one in a
child process (a process loads one of the two libraries)."""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from gnss_gpu_b200 import _native as N

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
CHECKED = ROOT / "gnss_gpu_b200" / "lib" / "libgnsspf_b200_checked.so"

RUN = r"""
import sys, numpy as np
sys.path[:0] = [{root!r}, {tests!r}]
from gnss_gpu_b200 import _native as N
from gnss_gpu_b200 import scenario as S
import pfhelp as H
out = {{"lib": str(N.LIB_PATH)}}
tr = S.config1(n_epochs=7)
for res in ("systematic", "megopolis"):
    for k, fl in enumerate([N.PF_EP_PREDICT | N.PF_EP_WEIGHT, N.PF_EP_PREDICT | N.PF_EP_WEIGHT | N.PF_EP_FORCE_RESAMPLE]):
        eng = H.make_engine([30_001, 777], n_clk=4, resampler=res, seeds=[3, 4])
        for f in range(2):
            eng.initialize(f, tr.anchor, tr.truth_clk[0], 10.0, 30.0)
        for t in range(6):
            rec = {{"disp": tr.disp_enu[t], "sats": tr.sats[t], "pr": tr.pr[t], "clk": tr.clk_idx[t], "flags": fl}}
            fe, sv = eng.pack_epoch([rec, rec])
            eng.upload(0, fe, sv)
            eng.step()
        for f in range(2):
            x, lw = eng.state_f32(f, raw=True)
            out[f"{{res}}{{k}}_{{f}}_x"] = x
            out[f"{{res}}{{k}}_{{f}}_lw"] = lw
            out[f"{{res}}{{k}}_{{f}}_anc"] = eng.ancestors(f)
            out[f"{{res}}{{k}}_{{f}}_est"] = eng.results()[f]["est_ecef"]
        out[f"{{res}}{{k}}_err"] = np.array([eng.error_word()])
        eng.close()
np.savez({path!r}, **out)
"""


def _run(path, lib=None):
    env = dict(os.environ)
    if lib:
        env["PF_B200_LIB"] = str(lib)
    else:
        env.pop("PF_B200_LIB", None)
    code = RUN.format(root=str(ROOT), tests=str(ROOT / "tests"), path=str(path))
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.load(path)


def test_checked_build_equals_release_and_stays_quiet(tmp_path):
    assert CHECKED.exists(), "build() makes the checked library"
    rel = _run(tmp_path / "release.npz")
    chk = _run(tmp_path / "checked.npz", CHECKED)
    assert str(chk["lib"]).endswith("libgnsspf_b200_checked.so")
    assert str(rel["lib"]).endswith("libgnsspf_b200.so")
    for k in rel.files:
        if k == "lib":
            continue
        if k.endswith("_err"):
            assert int(chk[k][0]) == 0 and int(rel[k][0]) == 0, k
        else:
            assert np.array_equal(rel[k], chk[k]), k
