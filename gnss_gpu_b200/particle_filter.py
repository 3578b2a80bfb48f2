"""Drop-in ParticleFilter for python/gnss_gpu/particle_filter.py:10-222.

Same constructor arguments, methods, return shapes and exceptions as the
reference class.  The particles live on the GPU as FP32 offsets in a local
E/N/U frame about an FP64 anchor (re-centred every epoch on the weighted
mean), and every call runs the engine's sm_100a kernels:

* predict() records the motion; the next update() fuses it with the weight
  pass (one kernel reads the state once), as the reference's
  predict -> update sequence (particle_filter.py:102-161) would compute.
* update() evaluates the pseudorange likelihood, the ESS and, when
  ESS < ess_threshold * N, resamples -- the decision is taken on the device,
  so update() does not synchronise with the host.
* estimate(), get_particles(), get_ess() return host values as the
  reference does.

Extensions (keyword-only, reference behaviour by default): per-axis position
noise, Huber likelihood, accumulating log-weights, Megopolis iteration count,
reference or random systematic offset.
"""
from __future__ import annotations

import numpy as np

from . import _native as N
from .engine import Engine, EngineOptions, FilterSpec


class ParticleFilter:
    """Mega particle filter for GNSS positioning in ECEF coordinates.

    Parameters are those of the reference class (particle_filter.py:31-33):
    n_particles, sigma_pos, sigma_cb, sigma_pr, resampling ("megopolis" or
    "systematic"), ess_threshold, seed.
    """

    def __init__(self, n_particles=1_000_000, sigma_pos=1.0, sigma_cb=300.0,
                 sigma_pr=5.0, resampling="megopolis", ess_threshold=0.5,
                 seed=42, *, megopolis_iterations=15, weight_mode="gaussian",
                 huber_k=1.5, log_weight_mode="overwrite",
                 systematic_offset="reference", max_sats=N.PF_MAX_SATS,
                 recenter=True):
        N.load()  # the reference imports its extension here (particle_filter.py:34-43)
        self.n_particles = n_particles
        self.sigma_pos = sigma_pos
        self.sigma_cb = sigma_cb
        self.sigma_pr = sigma_pr
        self.resampling = resampling
        self.ess_threshold = ess_threshold
        self.seed = seed
        self.megopolis_iterations = megopolis_iterations
        self.weight_mode = weight_mode
        self.huber_k = huber_k
        self.log_weight_mode = log_weight_mode
        self.systematic_offset = systematic_offset
        self.max_sats = max_sats
        self.recenter = recenter
        self._engine = None
        self._initialized = False
        self._step = 0
        self._pending_disp = None
        self._rot = None
        self._spec = None

    # ------------------------------------------------------------------
    def _require_init(self):
        if not self._initialized:
            raise RuntimeError("ParticleFilter not initialized. Call initialize() first.")

    def _filter_spec(self):
        sp = self.sigma_pos
        sp3 = tuple(float(v) for v in (np.broadcast_to(np.asarray(sp, dtype=np.float64), (3,))))
        return FilterSpec(n_particles=int(self.n_particles), seed=int(self.seed), sigma_pos=sp3,
                          sigma_clk=float(self.sigma_cb), sigma_pr=float(self.sigma_pr))

    def _sync_params(self):
        spec = self._filter_spec()
        if spec != self._spec:
            self._engine.set_filter_params(0, spec)
            self._spec = spec

    def initialize(self, position_ecef, clock_bias=0.0, spread_pos=100.0, spread_cb=1000.0):
        """Scatter particles N(position, spread_pos) / N(clock_bias, spread_cb)."""
        pos = np.asarray(position_ecef, dtype=np.float64).ravel()
        if pos.size < 3 or not np.all(np.isfinite(pos[:3])):
            raise ValueError("position_ecef must hold 3 finite values")
        if self.resampling not in ("megopolis", "systematic"):
            raise ValueError(f"unknown resampling method {self.resampling!r}")
        if self._engine is not None:
            self._engine.close()
        opts = EngineOptions(
            n_clk=1,
            resampler=self.resampling,
            megopolis_iters=int(self.megopolis_iterations),
            weight_mode=self.weight_mode,
            huber_k=float(self.huber_k),
            lw_mode=self.log_weight_mode,
            sys_offset=self.systematic_offset,
            max_sats=int(self.max_sats),
            obs_slots=1,
            covariance=True,
            recenter=bool(self.recenter),
            ess_threshold=float(self.ess_threshold),
        )
        self._spec = self._filter_spec()
        self._engine = Engine([self._spec], opts)
        self._engine.initialize(0, pos[:3], float(clock_bias), float(spread_pos), float(spread_cb))
        self._rot, _ = self._engine.frame(0)
        self._initialized = True
        self._step = 0
        self._pending_disp = None

    def _launch(self, disp_local, flags, sats=None, pr=None, w=None):
        eng = self._engine
        rec = {"disp": disp_local, "flags": flags}
        if sats is not None:
            rec.update(sats=sats, pr=pr, w=w)
        fe, sv = eng.pack_epoch([rec])
        eng.upload(0, fe, sv)
        eng.step()

    def _flush_predict(self):
        if self._pending_disp is not None:
            self._sync_params()
            self._launch(self._pending_disp, N.PF_EP_PREDICT)
            self._pending_disp = None

    def predict(self, velocity=None, dt=1.0):
        """Constant-velocity motion (ECEF m/s) plus N(0, sigma_pos) / N(0, sigma_cb)."""
        self._require_init()
        if velocity is None:
            velocity = [0.0, 0.0, 0.0]
        vel = np.asarray(velocity, dtype=np.float64).ravel()
        if vel.size < 3 or not np.all(np.isfinite(vel[:3])) or not np.isfinite(dt):
            raise ValueError("velocity must hold 3 finite values and dt must be finite")
        self._flush_predict()
        self._step += 1
        self._pending_disp = self._rot @ (vel[:3] * float(dt))

    def update(self, sat_ecef, pseudoranges, weights=None):
        """Pseudorange likelihood, ESS and ESS-triggered resampling."""
        self._require_init()
        sat = np.asarray(sat_ecef, dtype=np.float64).reshape(-1, 3)
        pr = np.asarray(pseudoranges, dtype=np.float64).ravel()
        n_sat = len(pr)
        if len(sat) != n_sat:
            raise ValueError("sat_ecef and pseudoranges disagree on the satellite count")
        if weights is None:
            weights = np.ones(n_sat, dtype=np.float64)
        else:
            weights = np.asarray(weights, dtype=np.float64).ravel()
        self._sync_params()
        flags = N.PF_EP_WEIGHT
        disp = np.zeros(3)
        if self._pending_disp is not None:
            flags |= N.PF_EP_PREDICT
            disp = self._pending_disp
            self._pending_disp = None
        self._launch(disp, flags, sat, pr, weights)

    def estimate(self):
        """Weighted mean [x, y, z, clock_bias] (ECEF, m) of the current particles."""
        self._require_init()
        self._flush_predict()
        return self._engine.estimate(0)

    def get_particles(self):
        """All particles as an (n_particles, 4) FP64 array [x, y, z, clock_bias]."""
        self._require_init()
        self._flush_predict()
        return self._engine.particles(0)

    def get_ess(self):
        """Effective sample size of the current log-weights."""
        self._require_init()
        return self._engine.ess(0)

    # ---------------------------------------------------------- extensions
    def get_log_weights(self):
        """Current log-weights as FP64 (zeros right after a resample)."""
        self._require_init()
        self._flush_predict()
        _, lw = self._engine.state_f32(0)
        return lw.astype(np.float64)

    def last_step(self):
        """Fused per-step outputs: pre-resample weighted mean, covariance, ESS."""
        self._require_init()
        return self._engine.results()[0]
