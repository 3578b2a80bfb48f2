"""The launch-configuration autotuner: cache keys (CPU) and one tuning run
on the GPU."""
import json

import pytest

from gnss_gpu_b200 import autotune as A
from gnss_gpu_b200.engine import EngineOptions


def test_key_buckets_particle_counts_by_power_of_two():
    assert A.key(1000, 8, 1, 1, "systematic") == A.key(1024, 8, 1, 1, "systematic") == "N1024_S8_C1_F1_systematic"
    assert A.key(1025, 8, 1, 1, "systematic").startswith("N2048_")
    assert A.key(1000, 9, 1, 1, "systematic") != A.key(1000, 8, 1, 1, "systematic")


def test_apply_sets_path_and_resampler():
    o = A.apply(A.Choice("chain", 0, "megopolis"), EngineOptions(n_clk=1))
    assert o.kernel_chain and o.resampler == "megopolis"
    o = A.apply(A.Choice("epoch", 1, "systematic"), EngineOptions(n_clk=1))
    assert not o.kernel_chain and o.resampler == "systematic"


@pytest.mark.gpu
def test_tune_times_every_candidate_and_caches(tmp_path, monkeypatch):
    monkeypatch.setenv("XDG_CACHE_HOME", str(tmp_path))
    best, ms = A.tune(50_000, 16, n_clk=2, n_filters=2, resampler="any", steps=4, warmup=2)
    assert len(ms) == 6 and all(v > 0 for v in ms.values())
    assert ms[f"{best.path}/{best.ctas_per_sm}/{best.resampler}"] == min(ms.values())
    cached = json.loads((tmp_path / "gnss_gpu_b200" / "autotune.json").read_text())
    assert A.key(50_000, 16, 2, 2, "any") in cached
    again, ms2 = A.tune(50_000, 16, n_clk=2, n_filters=2, resampler="any")
    assert again == best and ms2 == ms
