"""Run the reference's own GPU particle-filter functions (its _gnss_gpu_pf
module compiled by oracle/build_ref.py into oracle/_ref) on seeded inputs and
save their outputs, so the CPU oracle can be pinned to the reference itself.

Needs a GPU: python tests/golden/make_ref_gpu_fixtures.py
Writes tests/golden/ref_gpu_fixtures.npz.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "oracle" / "_ref"))


def main():
    import gnss_gpu._gnss_gpu_pf as ref  # the reference's module, built from its sources
    fx = json.loads((HERE / "tokyo_fixture.json").read_text())
    sat = np.array(fx["sat_ecef"])
    pr = np.array(fx["pseudoranges"])
    tp = np.array(fx["true_pos"])
    tcb = fx["true_cb"]
    out = {}
    rng = np.random.default_rng(31337)
    for c, (n, sp, scb) in enumerate([(1000, 30.0, 60.0), (10_000, 200.0, 400.0), (100_003, 5.0, 10.0)]):
        px = tp[0] + rng.normal(0, sp, n)
        py = tp[1] + rng.normal(0, sp, n)
        pz = tp[2] + rng.normal(0, sp, n)
        pcb = tcb + rng.normal(0, scb, n)
        ws = rng.uniform(0.5, 2.0, len(pr))
        lw = np.empty(n)
        ref.pf_weight(px, py, pz, pcb, sat.ravel(), pr, ws, lw, n, len(pr), 5.0)
        ess = ref.pf_compute_ess(lw, n)
        est = np.empty(4)
        ref.pf_estimate(px, py, pz, pcb, lw, est, n)
        parts = np.empty(4 * n)
        ref.pf_get_particles(px, py, pz, pcb, parts, n)
        idx = [np.arange(n, dtype=np.float64) for _ in range(4)]
        ref.pf_resample_systematic(*idx, lw, n, 12345)
        midx = [np.arange(n, dtype=np.float64) for _ in range(4)]
        ref.pf_resample_megopolis(*midx, lw, n, 15, 12345)
        out.update({
            f"c{c}_px": px, f"c{c}_py": py, f"c{c}_pz": pz, f"c{c}_pcb": pcb, f"c{c}_wsat": ws,
            f"c{c}_lw": lw, f"c{c}_ess": np.array(ess), f"c{c}_est": est, f"c{c}_particles": parts,
            f"c{c}_sys_anc": idx[0].astype(np.int64), f"c{c}_mego_anc": midx[0].astype(np.int64),
        })
    # ESS known cases of the reference tests (tests/test_particle_filter.py:174-193)
    out["ess_uniform_10000"] = np.array(ref.pf_compute_ess(np.zeros(10_000), 10_000))
    dom = np.full(1000, -1000.0)
    dom[0] = 0.0
    out["ess_dominant_1000"] = np.array(ref.pf_compute_ess(dom, 1000))
    np.savez_compressed(HERE / "ref_gpu_fixtures.npz", **out)
    print("wrote", HERE / "ref_gpu_fixtures.npz")


if __name__ == "__main__":
    main()
