"""B200 (sm_100a) implementation of the gnss_gpu particle-filter step.

`ParticleFilter` is the drop-in for gnss_gpu.particle_filter.ParticleFilter
and `ParticleFilterDevice` for gnss_gpu.particle_filter_device.ParticleFilterDevice;
`_gnss_gpu_pf` mirrors the reference's pybind11 module; `Engine` advances many
filters together.  All compute runs in libgnsspf_b200.so (hand-written CUDA).
"""
from .particle_filter import ParticleFilter
from .particle_filter_device import ParticleFilterDevice
from .engine import Engine, EngineOptions, FilterSpec

__all__ = ["ParticleFilter", "ParticleFilterDevice", "Engine", "EngineOptions", "FilterSpec"]
