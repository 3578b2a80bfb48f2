"""Generate golden fixtures from the reference's own Python code.

Runs only where the reference tree is mounted (it is read-only input, not a
dependency): python tests/golden/make_golden.py /path/to/gnss_gpu

Writes, next to this script:
  tokyo_fixture.json   -- the reference test scenario, obtained by calling
                          _make_test_scenario() of tests/test_particle_filter.py
  simple_pf_cpu.npz    -- log-likelihoods, ESS and weighted means computed by
                          the reference's CPU particle filter SimplePFCPU
                          (experiments/evaluate.py:701-775) on seeded particles
"""
from __future__ import annotations

import importlib.util
import json
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _load(path: Path, name: str):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main(ref_root: str):
    ref = Path(ref_root)
    sys.path.insert(0, str(ref / "python"))
    # the reference's PF test module; its GPU import fails here and is caught
    tmod = _load(ref / "tests" / "test_particle_filter.py", "ref_test_particle_filter")
    sat, pr, w, true_pos, true_cb = tmod._make_test_scenario()
    (HERE / "tokyo_fixture.json").write_text(json.dumps({
        "source": "tests/test_particle_filter.py:24-48 (_make_test_scenario)",
        "sat_ecef": np.asarray(sat).tolist(), "pseudoranges": np.asarray(pr).tolist(),
        "weights": np.asarray(w).tolist(), "true_pos": np.asarray(true_pos).tolist(),
        "true_cb": float(true_cb), "n_test": int(tmod.N_TEST), "seed": int(tmod.SEED),
    }, indent=1))

    # experiments/evaluate.py imports gnss_gpu.range_model at module level;
    # SimplePFCPU itself only needs numpy.
    evmod = _load(ref / "experiments" / "evaluate.py", "ref_evaluate")
    SimplePFCPU = evmod.SimplePFCPU
    rng = np.random.default_rng(20240611)
    cases = {}
    for case, (n, spread, cb_spread) in enumerate([(64, 30.0, 50.0), (257, 200.0, 400.0), (1000, 5.0, 5.0)]):
        pf = SimplePFCPU(n_particles=n, sigma_pr=5.0, seed=case)
        parts = np.column_stack([
            true_pos[0] + rng.normal(0, spread, n), true_pos[1] + rng.normal(0, spread, n),
            true_pos[2] + rng.normal(0, spread, n), true_cb + rng.normal(0, cb_spread, n)])
        ws = rng.uniform(0.5, 2.0, len(pr))
        # log-likelihood: update() with log_w = 0 turns log_w into
        # loglik - max(loglik); when it resamples (ESS < N/2) it calls
        # rng.choice(...) first and zeroes log_w afterwards, so a stand-in rng
        # records log_w at that moment.  Otherwise log_w keeps the value.
        sat_ = np.asarray(sat, dtype=np.float64)
        pf_ll = SimplePFCPU(n_particles=n, sigma_pr=5.0, seed=case)
        pf_ll.particles = parts.copy()
        pf_ll.log_w = np.zeros(n)
        seen = []

        def _choice(m, size=None, p=None, _pf=pf_ll, _seen=seen):
            _seen.append((_pf.log_w.copy(), np.asarray(p).copy()))
            return np.arange(m)

        pf_ll.rng = types.SimpleNamespace(choice=_choice)
        pf_ll.update(sat_, pr, ws)
        shifted = seen[0][0] if seen else pf_ll.log_w.copy()
        # a filter whose ESS stays above N/2 keeps its weights: use the
        # estimate/ESS of the shifted log-weights directly
        pf_e = SimplePFCPU(n_particles=n, seed=case)
        pf_e.particles = parts.copy()
        lw_rand = rng.normal(0.0, 1.5, n)
        pf_e.log_w = lw_rand.copy()
        cases[f"c{case}_particles"] = parts
        cases[f"c{case}_wsat"] = ws
        cases[f"c{case}_shifted_loglik"] = shifted
        cases[f"c{case}_resampled"] = np.array(bool(seen))
        cases[f"c{case}_lw_rand"] = lw_rand
        cases[f"c{case}_ess"] = np.array(pf_e.get_ess())
        cases[f"c{case}_estimate"] = pf_e.estimate()
    np.savez(HERE / "simple_pf_cpu.npz", **cases)
    print("wrote", HERE / "tokyo_fixture.json", HERE / "simple_pf_cpu.npz")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["GNSS_GPU_REFERENCE"])
