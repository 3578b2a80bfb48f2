"""B200 (sm_100a) implementation of the gnss_gpu particle-filter step.

`ParticleFilter` is the drop-in for gnss_gpu.particle_filter.ParticleFilter,
`ParticleFilterDevice` for gnss_gpu.particle_filter_device.ParticleFilterDevice
and `ParticleFilter3D` / `ParticleFilter3DBVH` (with `BVHAccelerator`) for
the building-aware filters; `_gnss_gpu_pf` mirrors the reference's pybind11 module; `Engine` advances many
filters together.  All compute runs in libgnsspf_b200.so (hand-written CUDA).
"""
from .particle_filter import ParticleFilter
from .particle_filter_device import ParticleFilterDevice
from .particle_filter_3d import ParticleFilter3D, ParticleFilter3DBVH
from .bvh import BVHAccelerator, BuildingModel
from .engine import Engine, EngineOptions, FilterSpec
from .ephemeris import Ephemeris
from .nav_rinex import NavMessage, read_nav_rinex, read_nav_rinex_multi
from .nmea import NMEAWriter, ecef_to_nmea, parse_nmea, positions_to_nmea
from .rinex_obs import read_rinex_obs

__all__ = ["ParticleFilter", "Ephemeris", "NavMessage", "read_nav_rinex", "read_nav_rinex_multi", "read_rinex_obs", "parse_nmea",
           "NMEAWriter", "positions_to_nmea", "ecef_to_nmea", "ParticleFilterDevice", "ParticleFilter3D", "ParticleFilter3DBVH", "BVHAccelerator",
           "BuildingModel", "Engine", "EngineOptions", "FilterSpec"]
