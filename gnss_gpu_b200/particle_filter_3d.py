"""Drop-ins for python/gnss_gpu/particle_filter_3d.py (ParticleFilter3D) and
python/gnss_gpu/particle_filter_3d_bvh.py (ParticleFilter3DBVH).

update() casts, for every particle and satellite, a ray from the particle
to the satellite through the building mesh (pfe_add_3d_term: BVH traversal
in FP32 in the mesh frame, ranges and likelihood in FP64) and weights the
pseudorange with a tight LOS Gaussian or a wide NLOS Gaussian whose positive
residuals are reduced by nlos_bias, mixed by the blocked / clear NLOS priors
(weight_3d.cu:86-177).  Then, as in the reference, the ESS decides the
resample.  Both classes trace through a hierarchy: the reference's
ParticleFilter3D scans every triangle, which gives the same blocked flags.
"""
from __future__ import annotations

import numpy as np

from . import _native as N
from .bvh import BVHAccelerator
from .particle_filter import ParticleFilter


class ParticleFilter3D(ParticleFilter):
    """Particle filter with building-aware NLOS handling (reference
    constructor: building_model, sigma_los, sigma_nlos, nlos_bias,
    blocked_nlos_prob, clear_nlos_prob, **ParticleFilter kwargs)."""

    def __init__(self, building_model, sigma_los=3.0, sigma_nlos=30.0, nlos_bias=20.0, blocked_nlos_prob=1.0,
                 clear_nlos_prob=0.0, **kwargs):
        super().__init__(**kwargs)
        if not hasattr(building_model, "triangles"):
            raise TypeError("building_model must hold a triangles array")
        self.building_model = building_model
        self._bvh = BVHAccelerator(building_model.triangles)
        self.sigma_los = sigma_los
        self.sigma_nlos = sigma_nlos
        self.nlos_bias = nlos_bias
        self.blocked_nlos_prob = blocked_nlos_prob
        self.clear_nlos_prob = clear_nlos_prob

    def initialize(self, position_ecef, clock_bias=0.0, spread_pos=100.0, spread_cb=1000.0):
        """As ParticleFilter.initialize, then the particles are put in
        spatial order (Engine.sort_spatially) so that the ray casts of
        neighbouring threads take similar paths through the buildings."""
        super().initialize(position_ecef, clock_bias, spread_pos, spread_cb)
        self._engine.sort_spatially(0)

    def update(self, sat_ecef, pseudoranges, weights=None):
        """Building-aware weight update, ESS and ESS-triggered resampling."""
        if not self._initialized:
            raise RuntimeError(f"{type(self).__name__} not initialized. Call initialize() first.")
        sat = np.asarray(sat_ecef, dtype=np.float64).reshape(-1, 3)
        pr = np.asarray(pseudoranges, dtype=np.float64).ravel()
        if len(sat) != len(pr):
            raise ValueError("sat_ecef and pseudoranges disagree on the satellite count")
        w = np.ones(len(pr)) if weights is None else np.asarray(weights, dtype=np.float64).ravel()
        self._flush_predict()
        self._engine.add_3d_term(0, self._bvh.mesh, sat, pr, w, float(self.sigma_los), float(self.sigma_nlos),
                                 float(self.nlos_bias), float(self.blocked_nlos_prob), float(self.clear_nlos_prob))
        self._sync_params()
        self._launch(np.zeros(3), N.PF_EP_RESAMPLE_CHECK)


class ParticleFilter3DBVH(ParticleFilter3D):
    """ParticleFilter3D over a prebuilt BVHAccelerator (reference
    constructor: bvh, sigma_los, ..., **ParticleFilter kwargs)."""

    def __init__(self, bvh, sigma_los=3.0, sigma_nlos=30.0, nlos_bias=20.0, blocked_nlos_prob=1.0,
                 clear_nlos_prob=0.0, **kwargs):
        if not isinstance(bvh, BVHAccelerator):
            raise TypeError("bvh must be a BVHAccelerator instance")
        ParticleFilter.__init__(self, **kwargs)
        self.bvh = bvh
        self._bvh = bvh
        self.building_model = None
        self.sigma_los = sigma_los
        self.sigma_nlos = sigma_nlos
        self.nlos_bias = nlos_bias
        self.blocked_nlos_prob = blocked_nlos_prob
        self.clear_nlos_prob = clear_nlos_prob
