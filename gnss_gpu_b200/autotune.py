"""Autotuner of the engine's launch configuration, keyed on (N, n_sat).

For a workload shape it times, on the GPU and with synthetic observations
of that shape, every candidate of

  * path          -- one cooperative kernel per epoch ("epoch") or one kernel
                     per phase ("chain"),
  * ctas_per_sm   -- how many CTAs per SM the cooperative kernel launches
                     (1 or every CTA that fits),
  * resampler     -- when the caller allows either ("any"), systematic or
                     Megopolis,

and keeps the fastest.  Tiles are fixed at 1024 particles (256 threads x 4
particles, one float4 per state component), so tile size and particles per
thread are not free parameters of this engine.  Results are cached per key
(particle count rounded to a power of two, satellite count, clock count,
filter count, resampler choice) in a JSON file, by default
$XDG_CACHE_HOME/gnss_gpu_b200/autotune.json.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import asdict, dataclass, replace
from pathlib import Path

import numpy as np

from . import _native as N
from . import scenario as S
from .engine import Engine, EngineOptions, FilterSpec


@dataclass(frozen=True)
class Choice:
    path: str = "epoch"
    ctas_per_sm: int = 0       # 0: every CTA that fits
    resampler: str = "systematic"


def cache_path() -> Path:
    base = os.environ.get("XDG_CACHE_HOME") or str(Path.home() / ".cache")
    return Path(base) / "gnss_gpu_b200" / "autotune.json"


def key(n_particles: int, n_sat: int, n_clk: int, n_filters: int, resampler: str) -> str:
    nb = 1 << max(0, int(math.ceil(math.log2(max(1, n_particles)))))
    return f"N{nb}_S{n_sat}_C{n_clk}_F{n_filters}_{resampler}"


def _time_choice(ch: Choice, n_particles: int, n_sat: int, n_clk: int, n_filters: int, steps: int, warmup: int):
    tr = S.single_filter(n_epochs=steps + warmup + 1, n_const=n_clk, sats_per_const=max(1, n_sat // n_clk),
                         nlos_frac=0.25, seed=3)
    specs = [FilterSpec(n_particles=n_particles, seed=11 + k, sigma_pos=(1.0, 1.0, 0.5), sigma_clk=0.5,
                        sigma_pr=3.0) for k in range(n_filters)]
    eng = Engine(specs, EngineOptions(n_clk=n_clk, resampler=ch.resampler, max_sats=max(n_sat, 1),
                                      obs_slots=steps + warmup, kernel_chain=ch.path == "chain"))
    try:
        if ch.path == "epoch":
            eng.set_epoch_ctas_per_sm(ch.ctas_per_sm)
        for k in range(n_filters):
            eng.initialize(k, tr.truth_ecef[0], tr.truth_clk[0], 10.0, 30.0)
        flags = N.PF_EP_PREDICT | N.PF_EP_WEIGHT
        for t in range(steps + warmup):
            rec = {"disp": tr.disp_enu[t], "sats": tr.sats[t], "pr": tr.pr[t], "clk": tr.clk_idx[t], "flags": flags}
            fe, sv = eng.pack_epoch([rec] * n_filters)
            eng.upload(t, fe, sv)
        for _ in range(warmup):
            eng.step()
        eng.enable_timing(steps)
        for _ in range(steps):
            eng.step()
        _, whole = eng.read_timing()
        return float(np.median(whole))
    finally:
        eng.close()


def tune(n_particles: int, n_sat: int, n_clk: int = 1, n_filters: int = 1, resampler: str = "systematic",
         steps: int = 12, warmup: int = 4, use_cache: bool = True):
    """Best Choice for the shape, and the timings (ms per step) of every
    candidate.  resampler: "systematic", "megopolis" or "any"."""
    k = key(n_particles, n_sat, n_clk, n_filters, resampler)
    path = cache_path()
    cache = {}
    if use_cache and path.exists():
        try:
            cache = json.loads(path.read_text())
        except ValueError:
            cache = {}
        if k in cache:
            return Choice(**cache[k]["choice"]), cache[k]["ms"]
    resamplers = ["systematic", "megopolis"] if resampler == "any" else [resampler]
    cands = []
    for r in resamplers:
        cands.append(Choice("chain", 0, r))
        cands.append(Choice("epoch", 0, r))
        cands.append(Choice("epoch", 1, r))
    ms = {}
    for c in cands:
        ms[f"{c.path}/{c.ctas_per_sm}/{c.resampler}"] = _time_choice(c, n_particles, n_sat, n_clk, n_filters, steps,
                                                                     warmup)
    best = min(cands, key=lambda c: ms[f"{c.path}/{c.ctas_per_sm}/{c.resampler}"])
    if use_cache:
        cache[k] = {"choice": asdict(best), "ms": ms}
        path.parent.mkdir(parents=True, exist_ok=True)
        path.write_text(json.dumps(cache, indent=1))
    return best, ms


def apply(choice: Choice, options: EngineOptions) -> EngineOptions:
    """EngineOptions with the tuned path and resampler (the CTA cap is set on
    the engine with Engine.set_epoch_ctas_per_sm(choice.ctas_per_sm))."""
    return replace(options, kernel_chain=choice.path == "chain", resampler=choice.resampler)
