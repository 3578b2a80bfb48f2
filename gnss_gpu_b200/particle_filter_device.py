"""Drop-in ParticleFilterDevice for python/gnss_gpu/particle_filter_device.py.

The reference's device-resident filter keeps (x, y, z, clock) per particle
on the GPU and offers robust likelihoods (Student's t, Huber, a per-particle
NLOS gate), a fixed two-component GMM, position-domain constraints, clock
and position shifts, and access to particle states, log-weights and
resampling ancestors.  This class offers the same constructor and those
methods on the engine's sm_100a kernels (weight mode "generic"):

* predict() records the motion; the next update() fuses it with the weight
  pass.  update()/update_gmm() overwrite the log-weights as the reference
  does (pf_device.cu:278) and, with resample=True, resample on the device
  when ESS < ess_threshold * N.
* position_update(), position_mixture_update() add a position term to the
  log-weights on the device; shift_clock_bias(), recenter_position() and
  correct_clock_bias() move the filter's anchor (O(1), no particle pass).
* resample_if_needed() tests the ESS of the current weights on the device
  and resamples when needed.

* update_dd_pseudorange(), update_carrier_afv(), update_dd_carrier_afv()
  evaluate the differenced / carrier-phase terms in FP64 on the device.

* Per-particle velocity states (velocity and its covariance, FP64) come into
  being when a call needs them (sigma_vel > 0, velocity_guide_alpha < 1,
  rbpf_velocity_kf, a velocity spread, a Doppler update); until then every
  particle's velocity is the last guide.  update_doppler() and
  update_doppler_kf() work on them.

* enable_smoothing(), store_epoch() and smooth() run the reference's
  forward-backward scheme: a second filter over the stored epochs in
  reverse, averaged with the forward estimates.
"""
from __future__ import annotations

import numpy as np

from . import _native as N
from .engine import Engine, EngineOptions, FilterSpec


class ParticleFilterDevice:
    """GPU-resident GNSS particle filter (reference constructor arguments)."""

    def __init__(self, n_particles=1_000_000, sigma_pos=1.0, sigma_cb=300.0,
                 sigma_pr=5.0, nu=0.0, resampling="megopolis", ess_threshold=0.5,
                 seed=42, per_particle_nlos_gate=False,
                 per_particle_nlos_dd_pr_threshold_m=10.0,
                 per_particle_nlos_dd_carrier_threshold_cycles=0.5,
                 per_particle_nlos_undiff_pr_threshold_m=30.0,
                 per_particle_huber=False,
                 per_particle_huber_dd_pr_k=1.5,
                 per_particle_huber_dd_carrier_k=1.5,
                 per_particle_huber_undiff_pr_k=1.5,
                 sigma_vel=0.0,
                 velocity_guide_alpha=1.0,
                 rbpf_velocity_kf=False,
                 velocity_process_noise=0.0, *, megopolis_iterations=15, max_sats=N.PF_MAX_SATS):
        N.load()
        self.n_particles = n_particles
        self.sigma_pos = sigma_pos
        self.sigma_cb = sigma_cb
        self.sigma_pr = sigma_pr
        self.nu = nu
        self.resampling = resampling
        self.ess_threshold = ess_threshold
        self.seed = seed
        self.per_particle_nlos_gate = bool(per_particle_nlos_gate)
        self.per_particle_nlos_dd_pr_threshold_m = float(per_particle_nlos_dd_pr_threshold_m)
        self.per_particle_nlos_dd_carrier_threshold_cycles = float(per_particle_nlos_dd_carrier_threshold_cycles)
        self.per_particle_nlos_undiff_pr_threshold_m = float(per_particle_nlos_undiff_pr_threshold_m)
        self.per_particle_huber = bool(per_particle_huber)
        self.per_particle_huber_dd_pr_k = float(per_particle_huber_dd_pr_k)
        self.per_particle_huber_dd_carrier_k = float(per_particle_huber_dd_carrier_k)
        self.per_particle_huber_undiff_pr_k = float(per_particle_huber_undiff_pr_k)
        self.sigma_vel = float(sigma_vel)
        self.velocity_guide_alpha = float(velocity_guide_alpha)
        self.rbpf_velocity_kf = bool(rbpf_velocity_kf)
        self.velocity_process_noise = float(velocity_process_noise)
        self.megopolis_iterations = int(megopolis_iterations)
        self.max_sats = int(max_sats)
        self._engine = None
        self._initialized = False
        self._step = 0
        self._pending = None        # (disp_local, sigma_pos) of a recorded predict
        self._spec = None
        self._rot = None
        self._vel = None            # per-particle velocity states, once any call needs them
        self._v_shared = np.zeros(3)
        self._var_shared = 0.0

    # ------------------------------------------------------------------
    def _require_init(self):
        if not self._initialized:
            raise RuntimeError("ParticleFilterDevice not initialized. Call initialize() first.")

    def _per_particle_threshold(self, value):
        if not self.per_particle_nlos_gate:
            return 0.0
        value = float(value)
        return value if np.isfinite(value) and value > 0.0 else 0.0

    @staticmethod
    def _per_particle_huber_k(value):
        value = float(value)
        return value if np.isfinite(value) and value > 0.0 else 1.5

    def _gate(self):
        return self._per_particle_threshold(self.per_particle_nlos_undiff_pr_threshold_m)

    def _huber_k(self):
        return self._per_particle_huber_k(self.per_particle_huber_undiff_pr_k)

    def _spec_for(self, sigma_pos, sigma_pr):
        sp = float(self.sigma_pos if sigma_pos is None else sigma_pos)
        return FilterSpec(n_particles=int(self.n_particles), seed=int(self.seed), sigma_pos=(sp, sp, sp),
                          sigma_clk=float(self.sigma_cb),
                          sigma_pr=float(self.sigma_pr if sigma_pr is None else sigma_pr))

    def _set_spec(self, spec):
        if spec != self._spec:
            self._engine.set_filter_params(0, spec)
            self._spec = spec

    def _launch(self, disp_local, flags, sats=None, pr=None, w=None):
        rec = {"disp": disp_local, "flags": flags}
        if sats is not None:
            rec.update(sats=sats, pr=pr, w=w)
        fe, sv = self._engine.pack_epoch([rec])
        self._engine.upload(0, fe, sv)
        self._engine.step()
        if self._vel is not None:
            self._vel.follow()

    def _flush(self):
        """Apply a recorded predict on its own (no weighting, no resampling)."""
        if self._pending is not None:
            disp, sp = self._pending
            self._pending = None
            self._set_spec(self._spec_for(sp, None))
            self._launch(disp, N.PF_EP_PREDICT)

    def _refresh(self, flags=0):
        """A step without motion or satellites: statistics of the current
        weights (and with PF_EP_RESAMPLE_CHECK the resample test)."""
        self._flush()
        self._launch(np.zeros(3), flags)

    # ------------------------------------------------------------------
    def initialize(self, position_ecef, clock_bias=0.0, spread_pos=100.0,
                   spread_cb=1000.0, velocity=None, spread_vel=0.0,
                   velocity_init_sigma=0.0):
        """Scatter particles N(position, spread_pos) / N(clock_bias, spread_cb);
        velocities `velocity` (+ N(0, spread_vel)), velocity covariance
        velocity_init_sigma^2 I."""
        v0 = np.zeros(3) if velocity is None else np.asarray(velocity, dtype=np.float64).ravel()[:3]
        if v0.size < 3 or not np.all(np.isfinite(v0)) or not (float(spread_vel) >= 0.0):
            raise ValueError("velocity must hold 3 finite values and spread_vel must be >= 0")
        pos = np.asarray(position_ecef, dtype=np.float64).ravel()
        if pos.size < 3 or not np.all(np.isfinite(pos[:3])):
            raise ValueError("position_ecef must hold 3 finite values")
        if self.resampling not in ("megopolis", "systematic"):
            raise ValueError(f"unknown resampling method {self.resampling!r}")
        if self._engine is not None:
            self._engine.close()
        opts = EngineOptions(n_clk=1, resampler=self.resampling, megopolis_iters=self.megopolis_iterations,
                             weight_mode="generic", huber_k=self._huber_k(), lw_mode="overwrite",
                             sys_offset="reference", max_sats=self.max_sats, obs_slots=1, covariance=True,
                             recenter=True, ess_threshold=float(self.ess_threshold))
        self._spec = self._spec_for(None, None)
        self._engine = Engine([self._spec], opts)
        self._engine.initialize(0, pos[:3], float(clock_bias), float(spread_pos), float(spread_cb))
        self._rot, _ = self._engine.frame(0)
        self._initialized = True
        self._step = 0
        self._pending = None
        self._vel = None
        self._v_shared = v0.copy()
        self._var_shared = float(velocity_init_sigma) ** 2
        if float(spread_vel) > 0.0 or self._per_particle_velocity():
            self._ensure_vel(spread_vel)

    def _per_particle_velocity(self, sigma_vel=None, alpha=None, kf=None):
        sv = self.sigma_vel if sigma_vel is None else float(sigma_vel)
        a = self.velocity_guide_alpha if alpha is None else float(alpha)
        k = self.rbpf_velocity_kf if kf is None else bool(kf)
        return sv > 0.0 or a != 1.0 or k

    def _ensure_vel(self, spread_vel=0.0):
        """Per-particle velocity states, started from the shared velocity and
        covariance every particle has had so far."""
        if self._vel is None:
            self._vel = self._engine.velocity_states(0)
            self._vel.init(self._v_shared, float(spread_vel), np.sqrt(self._var_shared), step=0)
        return self._vel

    def predict(self, velocity=None, dt=1.0, sigma_pos=None, sigma_vel=None, velocity_guide_alpha=None,
                rbpf_velocity_kf=None, velocity_process_noise=None):
        """Motion with the velocity guide (ECEF m/s) plus N(0, sigma_pos) /
        N(0, sigma_cb).  With per-particle velocities (sigma_vel > 0,
        velocity_guide_alpha < 1, rbpf_velocity_kf, a Doppler update, a
        velocity spread) every particle moves by its own velocity
        (pf_device.cu:106-187); otherwise every particle's velocity is the
        guide and the motion is fused into the next update."""
        self._require_init()
        vel = np.zeros(3) if velocity is None else np.asarray(velocity, dtype=np.float64).ravel()[:3]
        if vel.size < 3 or not np.all(np.isfinite(vel)) or not np.isfinite(dt):
            raise ValueError("velocity must hold 3 finite values and dt must be finite")
        self._flush()
        self._step += 1
        sp = float(self.sigma_pos if sigma_pos is None else sigma_pos)
        if self._vel is None and not self._per_particle_velocity(sigma_vel, velocity_guide_alpha, rbpf_velocity_kf):
            self._v_shared = vel.copy()
            self._pending = (self._rot @ (vel * float(dt)), sp)
            return
        sv = self.sigma_vel if sigma_vel is None else float(sigma_vel)
        a = self.velocity_guide_alpha if velocity_guide_alpha is None else float(velocity_guide_alpha)
        kf = self.rbpf_velocity_kf if rbpf_velocity_kf is None else bool(rbpf_velocity_kf)
        q = self.velocity_process_noise if velocity_process_noise is None else float(velocity_process_noise)
        self._ensure_vel().predict(vel, float(dt), sp, sv, a, kf, q, self._step)
        self._pending = (np.zeros(3), 0.0)  # the clocks' noise rides on the next update

    def _weight(self, sat_ecef, pseudoranges, weights, sigma_pr, resample, **lik):
        self._require_init()
        sat = np.asarray(sat_ecef, dtype=np.float64).reshape(-1, 3)
        pr = np.asarray(pseudoranges, dtype=np.float64).ravel()
        if len(sat) != len(pr):
            raise ValueError("sat_ecef and pseudoranges disagree on the satellite count")
        w = np.ones(len(pr)) if weights is None else np.asarray(weights, dtype=np.float64).ravel()
        self._engine.set_likelihood(**lik)
        flags = N.PF_EP_WEIGHT | (0 if resample else N.PF_EP_NO_RESAMPLE)
        disp, sp = np.zeros(3), None
        if self._pending is not None:
            disp, sp = self._pending
            self._pending = None
            flags |= N.PF_EP_PREDICT
        self._set_spec(self._spec_for(sp, sigma_pr))
        self._launch(disp, flags, sat, pr, w)

    def update(self, sat_ecef, pseudoranges, weights=None, sigma_pr=None, resample=True):
        """Pseudorange likelihood: Student's t when nu > 0, else Huber when
        per_particle_huber, else Gaussian; per-particle NLOS gate when
        per_particle_nlos_gate.  Overwrites the log-weights."""
        if float(self.nu) > 0.0:
            lik = dict(kind="student_t", nu=float(self.nu))
        elif self.per_particle_huber:
            lik = dict(kind="huber", huber_k=self._huber_k())
        else:
            lik = dict(kind="gaussian")
        self._weight(sat_ecef, pseudoranges, weights, sigma_pr, resample, gate_m=self._gate(), **lik)

    def update_gmm(self, sat_ecef, pseudoranges, weights=None, sigma_pr=None,
                   w_los=0.7, mu_nlos=15.0, sigma_nlos=30.0, resample=True):
        """LOS/NLOS Gaussian-mixture likelihood (pf_device.cu:373-436)."""
        self._weight(sat_ecef, pseudoranges, weights, sigma_pr, resample, kind="gmm", w_los=float(w_los),
                     mu_nlos=float(mu_nlos), sigma_nlos=float(sigma_nlos))

    @staticmethod
    def _dd_rows(dd_result, obs, wavelengths=None):
        n = int(dd_result.n_dd)
        rows = np.zeros(n, N.OBS_ROW_DTYPE)
        rows["sat_k"] = np.asarray(dd_result.sat_ecef_k, dtype=np.float64).reshape(-1, 3)[:n]
        rows["sat_ref"] = np.asarray(dd_result.sat_ecef_ref, dtype=np.float64).reshape(-1, 3)[:n]
        rows["obs"] = np.asarray(obs, dtype=np.float64).ravel()[:n]
        rows["base_k"] = np.asarray(dd_result.base_range_k, dtype=np.float64).ravel()[:n]
        rows["base_ref"] = np.asarray(dd_result.base_range_ref, dtype=np.float64).ravel()[:n]
        rows["weight"] = np.asarray(dd_result.dd_weights, dtype=np.float64).ravel()[:n]
        rows["wavelength"] = 1.0 if wavelengths is None else np.asarray(wavelengths, dtype=np.float64).ravel()[:n]
        return rows

    def _obs_update(self, kind, rows, sigma, gate, huber_k, accumulate, resample):
        self._require_init()
        self._flush()
        self._engine.add_obs_term(0, kind, rows, sigma, gate, huber_k, accumulate)
        if resample:
            self.resample_if_needed()

    def update_dd_pseudorange(self, dd_result, sigma_pr=0.75, resample=True):
        """Double-differenced pseudorange likelihood (clock-free); overwrites
        the log-weights (pf_device.cu:282-368).  dd_result: the reference's
        DDPseudorangeResult fields (sat_ecef_k, sat_ecef_ref,
        dd_pseudorange_m, base_range_k, base_range_ref, dd_weights, n_dd)."""
        rows = self._dd_rows(dd_result, dd_result.dd_pseudorange_m)
        huber = self._per_particle_huber_k(self.per_particle_huber_dd_pr_k) if self.per_particle_huber else 0.0
        self._obs_update(N.PF_OBS_DD_PSEUDORANGE, rows, float(sigma_pr),
                         self._per_particle_threshold(self.per_particle_nlos_dd_pr_threshold_m), huber, False,
                         resample)

    def update_carrier_afv(self, sat_ecef, carrier_phase_cycles, weights=None, wavelength=0.190293673,
                           sigma_cycles=0.05, resample=True):
        """Carrier-phase ambiguity-function likelihood on the fractional cycle
        residual; adds to the log-weights (pf_device.cu:439-494)."""
        sat = np.asarray(sat_ecef, dtype=np.float64).reshape(-1, 3)
        cp = np.asarray(carrier_phase_cycles, dtype=np.float64).ravel()
        rows = np.zeros(len(cp), N.OBS_ROW_DTYPE)
        rows["sat_k"] = sat
        rows["obs"] = cp
        rows["weight"] = 1.0 if weights is None else np.asarray(weights, dtype=np.float64).ravel()
        rows["wavelength"] = float(wavelength)
        self._obs_update(N.PF_OBS_CARRIER_AFV, rows, float(sigma_cycles), 0.0, 0.0, True, resample)

    def update_dd_carrier_afv(self, dd_result, wavelength=None, sigma_cycles=0.05, resample=True):
        """Double-differenced carrier-phase AFV likelihood; adds to the
        log-weights (pf_device.cu:496-604).  Per-pair wavelengths come from
        dd_result.wavelengths_m unless `wavelength` overrides them."""
        n = int(dd_result.n_dd)
        if wavelength is None:
            wl = getattr(dd_result, "wavelengths_m", None)
            wl = np.full(n, 0.190293673) if wl is None else np.asarray(wl, dtype=np.float64).ravel()
        else:
            wl = np.full(n, float(wavelength))
        rows = self._dd_rows(dd_result, dd_result.dd_carrier_cycles, wl)
        huber = self._per_particle_huber_k(self.per_particle_huber_dd_carrier_k) if self.per_particle_huber else 0.0
        self._obs_update(N.PF_OBS_DD_CARRIER_AFV, rows, float(sigma_cycles),
                         self._per_particle_threshold(self.per_particle_nlos_dd_carrier_threshold_cycles), huber,
                         True, resample)

    def _doppler_args(self, sat_ecef, sat_vel, doppler_hz, weights):
        sat = np.asarray(sat_ecef, dtype=np.float64).reshape(-1, 3)
        sv = np.asarray(sat_vel, dtype=np.float64).reshape(-1, 3)
        dop = np.asarray(doppler_hz, dtype=np.float64).ravel()
        if sat.shape != sv.shape:
            raise ValueError("sat_ecef and sat_vel must have the same shape")
        if dop.size != len(sat):
            raise ValueError("doppler_hz length must match sat_ecef rows")
        w = np.ones(dop.size) if weights is None else np.asarray(weights, dtype=np.float64).ravel()
        if w.size != dop.size:
            raise ValueError("weights length must match doppler_hz")
        return sat, sv, dop, w

    def update_doppler(self, sat_ecef, sat_vel, doppler_hz, weights=None, wavelength=0.19029367279836488,
                       sigma_mps=0.5, velocity_update_gain=0.25, max_velocity_update_mps=10.0, resample=True):
        """Doppler likelihood of each particle's velocity (with its own clock
        drift), then a blend of velocity_update_gain toward its Doppler WLS
        velocity (pf_device.cu:610-748); adds to the log-weights."""
        self._require_init()
        sat, sv, dop, w = self._doppler_args(sat_ecef, sat_vel, doppler_hz, weights)
        self._flush()
        self._ensure_vel().doppler(sat, sv, dop, w, float(wavelength), float(sigma_mps),
                                   float(velocity_update_gain), float(max_velocity_update_mps), kf=False)
        if resample:
            self.resample_if_needed()

    def update_doppler_kf(self, sat_ecef, sat_vel, doppler_hz, weights=None, wavelength=0.19029367279836488,
                          sigma_mps=0.5, resample=True):
        """Sequential Kalman update of each particle's velocity by the
        Doppler rows, with the innovation likelihood added to the
        log-weights (pf_device.cu:750-887)."""
        self._require_init()
        sat, sv, dop, w = self._doppler_args(sat_ecef, sat_vel, doppler_hz, weights)
        self._flush()
        self._ensure_vel().doppler(sat, sv, dop, w, float(wavelength), float(sigma_mps), kf=True)
        if resample:
            self.resample_if_needed()

    # ------------------------------------------------ forward-backward smoothing
    def enable_smoothing(self):
        """Store each epoch's observations for an offline forward-backward
        pass (particle_filter_device.py:892-899): call before the forward
        pass, store_epoch() after each epoch, smooth() at the end."""
        self._smooth_epochs = []
        self._smooth_enabled = True

    @staticmethod
    def _f64(a):
        return None if a is None else np.array(a, dtype=np.float64, copy=True)

    def store_epoch(self, sat_ecef, pseudoranges, weights, velocity, dt, spp_ref=None, dd_pseudorange=None,
                    dd_pseudorange_sigma=None, dd_pseudorange_source=None, dd_carrier=None, dd_carrier_sigma=None,
                    carrier_anchor_pseudorange=None, carrier_anchor_sigma=None, carrier_afv=None,
                    carrier_afv_sigma=None, carrier_afv_wavelength=None, doppler_update=None, doppler_sigma_mps=None,
                    doppler_velocity_update_gain=None, doppler_max_velocity_update_mps=None):
        """Record the epoch just processed (the arrays given to update(), the
        predict velocity and dt, optional references and the other
        observation updates) with the current estimate
        (particle_filter_device.py:901-1070)."""
        if not getattr(self, "_smooth_enabled", False):
            return
        f = self._f64

        def dd(res, extra):
            if res is None:
                return None
            d = {k: f(getattr(res, k)) for k in ("sat_ecef_k", "sat_ecef_ref", "base_range_k", "base_range_ref",
                                                 "dd_weights") + extra}
            d["ref_sat_ids"] = tuple(getattr(res, "ref_sat_ids", ()))
            d["n_dd"] = int(res.n_dd)
            return d

        def rows(src, keys):
            return None if src is None else {k: f(src[k]) for k in keys}

        dop = rows(doppler_update, ("sat_ecef", "sat_vel", "doppler_hz", "weights"))
        if dop is not None:
            dop["wavelength_m"] = float(doppler_update.get("wavelength_m", 0.19029367279836488))
        opt = lambda v: None if v is None else float(v)  # noqa: E731
        self._smooth_epochs.append({
            "estimate": np.asarray(self.estimate(), dtype=np.float64)[:3].copy(),
            "sat_ecef": f(sat_ecef), "pseudoranges": f(pseudoranges), "weights": f(weights),
            "velocity": f(velocity), "dt": float(dt), "spp_ref": f(spp_ref),
            "dd_pseudorange": dd(dd_pseudorange, ("dd_pseudorange_m",)),
            "dd_pseudorange_sigma": opt(dd_pseudorange_sigma),
            "dd_pseudorange_source": None if dd_pseudorange_source is None else str(dd_pseudorange_source),
            "dd_carrier": dd(dd_carrier, ("dd_carrier_cycles", "wavelengths_m")),
            "dd_carrier_sigma": opt(dd_carrier_sigma),
            "carrier_anchor_pseudorange": rows(carrier_anchor_pseudorange, ("sat_ecef", "pseudoranges", "weights")),
            "carrier_anchor_sigma": opt(carrier_anchor_sigma),
            "carrier_afv": rows(carrier_afv, ("sat_ecef", "carrier_phase_cycles", "weights")),
            "carrier_afv_sigma": opt(carrier_afv_sigma), "carrier_afv_wavelength": opt(carrier_afv_wavelength),
            "doppler_update": dop, "doppler_sigma_mps": opt(doppler_sigma_mps),
            "doppler_velocity_update_gain": opt(doppler_velocity_update_gain),
            "doppler_max_velocity_update_mps": opt(doppler_max_velocity_update_mps),
        })

    def smooth(self, position_update_sigma=None, skip_widelane_dd_pseudorange=False):
        """Backward pass over the stored epochs with a second filter (seed +
        1, reversed velocities, the same updates in the same order), then the
        equal-weight average of forward and backward estimates
        (particle_filter_device.py:1072-1251).  Returns (smoothed, forward),
        each (n_epochs, 3) ECEF."""
        from types import SimpleNamespace
        if not getattr(self, "_smooth_enabled", False) or not self._smooth_epochs:
            raise RuntimeError("No stored epochs. Call enable_smoothing() before forward pass.")
        stored = self._smooth_epochs
        n_ep = len(stored)
        forward = np.array([e["estimate"] for e in stored])
        last = stored[-1]
        init_cb = float(np.median(last["pseudoranges"] - np.linalg.norm(
            last["sat_ecef"].reshape(-1, 3) - last["estimate"], axis=1)))
        bwd = ParticleFilterDevice(
            n_particles=self.n_particles, sigma_pos=self.sigma_pos, sigma_cb=self.sigma_cb, sigma_pr=self.sigma_pr,
            nu=self.nu, resampling=self.resampling, ess_threshold=self.ess_threshold, seed=self.seed + 1,
            per_particle_nlos_gate=self.per_particle_nlos_gate,
            per_particle_nlos_dd_pr_threshold_m=self.per_particle_nlos_dd_pr_threshold_m,
            per_particle_nlos_dd_carrier_threshold_cycles=self.per_particle_nlos_dd_carrier_threshold_cycles,
            per_particle_nlos_undiff_pr_threshold_m=self.per_particle_nlos_undiff_pr_threshold_m,
            per_particle_huber=self.per_particle_huber, per_particle_huber_dd_pr_k=self.per_particle_huber_dd_pr_k,
            per_particle_huber_dd_carrier_k=self.per_particle_huber_dd_carrier_k,
            per_particle_huber_undiff_pr_k=self.per_particle_huber_undiff_pr_k, sigma_vel=self.sigma_vel,
            velocity_guide_alpha=self.velocity_guide_alpha, rbpf_velocity_kf=self.rbpf_velocity_kf,
            velocity_process_noise=self.velocity_process_noise, megopolis_iterations=self.megopolis_iterations,
            max_sats=self.max_sats)
        bwd.initialize(last["estimate"], clock_bias=init_cb, spread_pos=10.0, spread_cb=100.0,
                       velocity_init_sigma=np.sqrt(self._var_shared) if self._vel is None else 0.0)
        backward = np.zeros((n_ep, 3))
        for i in range(n_ep - 1, -1, -1):
            ep = stored[i]
            bwd.predict(velocity=None if ep["velocity"] is None else -ep["velocity"], dt=ep["dt"])
            sat, pr, w = ep["sat_ecef"].reshape(-1, 3), ep["pseudoranges"], ep["weights"]
            dd_ep = ep["dd_pseudorange"]
            if dd_ep is not None and not (skip_widelane_dd_pseudorange and ep["dd_pseudorange_source"] == "widelane"):
                bwd.update_dd_pseudorange(SimpleNamespace(**dd_ep), sigma_pr=(
                    ep["dd_pseudorange_sigma"] if ep["dd_pseudorange_sigma"] is not None else self.sigma_pr))
            else:
                bwd.correct_clock_bias(sat, pr)
                bwd.update(sat, pr, weights=w)
            if ep["dd_carrier"] is not None:
                bwd.resample_if_needed()
                bwd.update_dd_carrier_afv(SimpleNamespace(**ep["dd_carrier"]), sigma_cycles=(
                    ep["dd_carrier_sigma"] if ep["dd_carrier_sigma"] is not None else 0.05))
            ca = ep["carrier_anchor_pseudorange"]
            if ca is not None:
                bwd.update(ca["sat_ecef"], ca["pseudoranges"], weights=ca["weights"], sigma_pr=(
                    ep["carrier_anchor_sigma"] if ep["carrier_anchor_sigma"] is not None else self.sigma_pr))
            cafv = ep["carrier_afv"]
            if cafv is not None:
                bwd.resample_if_needed()
                bwd.update_carrier_afv(cafv["sat_ecef"], cafv["carrier_phase_cycles"], weights=cafv["weights"],
                                       wavelength=(ep["carrier_afv_wavelength"]
                                                   if ep["carrier_afv_wavelength"] is not None else 0.190293673),
                                       sigma_cycles=ep["carrier_afv_sigma"] if ep["carrier_afv_sigma"] is not None
                                       else 0.05)
            # Doppler rows constrain the forward-time velocity: the backward
            # filter runs with reversed velocities, so (as in the reference)
            # they are not replayed
            if position_update_sigma is not None and ep["spp_ref"] is not None:
                bwd.position_update(ep["spp_ref"][:3], sigma_pos=position_update_sigma)
            backward[i] = bwd.estimate()[:3]
        smoothed = (forward + backward) / 2.0
        self._smooth_enabled = False
        self._smooth_epochs = []
        if bwd._engine is not None:
            bwd._engine.close()
        return smoothed, forward

    # ------------------------------------------------------------------
    def position_update(self, ref_ecef, sigma_pos=30.0):
        """log-weights += -|p - ref|^2 / (2 sigma_pos^2) (pf_device.cu:889-900)."""
        self._require_init()
        ref = np.asarray(ref_ecef, dtype=np.float64).ravel()[:3]
        self._flush()
        self._engine.add_position_term(0, ref[None, :], float(sigma_pos))

    def position_mixture_update(self, refs_ecef, sigma_pos=1.0, mixture_weights=None):
        """log-weights += log sum_j pi_j exp(-|p - ref_j|^2 / (2 sigma^2)),
        pi normalised (at most 64 references, one device pass)."""
        self._require_init()
        refs = np.asarray(refs_ecef, dtype=np.float64).reshape(-1, 3)
        refs_ok = np.all(np.isfinite(refs), axis=1)
        if mixture_weights is None:
            mix = np.full(len(refs), 1.0 / max(1, len(refs)))
        else:
            mix = np.asarray(mixture_weights, dtype=np.float64).reshape(-1)
            if mix.size != len(refs):
                raise ValueError("mixture_weights length must match refs_ecef")
        refs, mix = refs[refs_ok], mix[refs_ok]
        if len(refs) == 0:
            return
        mix = np.where(np.isfinite(mix) & (mix > 0.0), mix, 0.0)
        mix = mix / mix.sum() if mix.sum() > 0 else np.full(len(refs), 1.0 / len(refs))
        if len(refs) > 64:
            raise ValueError("at most 64 mixture references are supported")
        keep = mix > 0
        self._flush()
        with np.errstate(divide="ignore"):
            self._engine.add_position_term(0, refs[keep], max(float(sigma_pos), 1.0e-6), np.log(mix[keep]))

    def shift_clock_bias(self, shift: float):
        """Add `shift` (m) to every particle's clock bias."""
        self._require_init()
        self._flush()
        self._engine.shift(0, np.zeros(3), [float(shift)])

    def recenter_position(self, ref_ecef, max_shift_m=10000.0):
        """Move the cloud's weighted mean to ref_ecef when within the cap;
        returns (shift norm, applied)."""
        self._require_init()
        ref = np.asarray(ref_ecef, dtype=np.float64).ravel()
        if ref.size != 3:
            raise ValueError("ref_ecef must have shape (3,)")
        if not np.all(np.isfinite(ref)):
            return float("inf"), False
        est = self.estimate()
        delta = ref - est[:3]
        norm = float(np.linalg.norm(delta))
        if float(max_shift_m) > 0.0 and norm > float(max_shift_m):
            return norm, False
        self._engine.shift(0, delta)
        return norm, True

    def correct_clock_bias(self, sat_ecef, pseudoranges, quantile=0.5):
        """Shift every clock bias so the estimate's clock equals the chosen
        quantile of the pseudorange residuals at the estimated position."""
        self._require_init()
        est = self.estimate()
        sat = np.asarray(sat_ecef, dtype=np.float64).reshape(-1, 3)
        pr = np.asarray(pseudoranges, dtype=np.float64).ravel()
        res = pr - np.linalg.norm(sat - est[:3], axis=1)
        expected = float(np.quantile(res, float(np.clip(quantile, 0.0, 1.0))))
        self._engine.shift(0, np.zeros(3), [expected - est[3]])

    def _resample(self):
        """Resample now, whatever the ESS."""
        self._require_init()
        self._refresh(N.PF_EP_RESAMPLE_CHECK | N.PF_EP_FORCE_RESAMPLE)

    def resample_if_needed(self):
        """Resample when the ESS of the current weights is below
        ess_threshold * n_particles; returns whether it did."""
        self._require_init()
        self._refresh(N.PF_EP_RESAMPLE_CHECK)
        return bool(self._engine.results()[0]["resampled"])

    # ------------------------------------------------------------------
    def estimate(self):
        """Weighted mean [x, y, z, clock_bias] (ECEF, m) of the current particles."""
        self._require_init()
        self._flush()
        return self._engine.estimate(0)

    def get_particles(self):
        """All particles as an (n_particles, 4) FP64 array [x, y, z, clock_bias]."""
        self._require_init()
        self._flush()
        return self._engine.particles(0)

    def get_particle_states(self):
        """(n_particles, 16) rows [x, y, z, clock_bias, vx, vy, vz, 3x3
        velocity covariance row-major] (ECEF, m, m/s)."""
        p = self.get_particles()
        out = np.zeros((len(p), 16))
        out[:, :4] = p
        if self._vel is not None:
            self._vel.follow()
            out[:, 4:] = self._vel.host()
        else:
            out[:, 4:7] = self._v_shared
            out[:, [7, 11, 15]] = self._var_shared
        return out

    def set_particle_states(self, states):
        """Replace the particles (rows [x, y, z, clock_bias, ...]) and reset
        the weights."""
        self._require_init()
        arr = np.asarray(states, dtype=np.float64)
        if arr.ndim != 2 or arr.shape[0] != self.n_particles or arr.shape[1] not in (4, 16):
            raise ValueError(f"states shape {arr.shape} != ({self.n_particles}, 16)")
        self._flush()
        anchor, clk, _ = self._engine.anchor(0)
        st = np.empty((4, self.n_particles), np.float32)
        st[:3] = ((arr[:, :3] - anchor) @ self._rot.T).T
        st[3] = arr[:, 3] - clk[0]
        self._engine.set_state_f32(0, st, np.zeros(self.n_particles, np.float32))
        if arr.shape[1] == 16:
            self._ensure_vel().set_host(arr[:, 4:])

    def get_log_weights(self):
        """Current log-weights as FP64."""
        self._require_init()
        self._flush()
        _, lw = self._engine.state_f32(0)
        return lw.astype(np.float64)

    def set_log_weights(self, log_weights):
        """Replace the log-weights of the current particles."""
        self._require_init()
        lw = np.asarray(log_weights, dtype=np.float64).reshape(-1)
        if lw.size != self.n_particles:
            raise ValueError(f"log_weights size {lw.size} != {self.n_particles}")
        self._flush()
        st, _ = self._engine.state_f32(0)
        self._engine.set_state_f32(0, st, lw.astype(np.float32))

    def get_resample_ancestors(self):
        """Slot j of the last systematic resample copied particle out[j]."""
        self._require_init()
        if self.resampling != "systematic":
            raise RuntimeError("get_resample_ancestors requires resampling='systematic'")
        return self._engine.ancestors(0)

    def get_ess(self):
        """Effective sample size of the current log-weights (device pass)."""
        self._require_init()
        self._flush()
        return self._engine.current_ess(0)

    def get_position_spread(self, center=None):
        """Weighted RMS distance of the particles from `center` (default: the
        weighted mean), m, from one device pass."""
        self._require_init()
        c = None
        if center is not None:
            c = np.asarray(center, dtype=np.float64).ravel()
            if c.size != 3:
                raise ValueError("center must have shape (3,)")
        self._flush()
        return self._engine.position_spread(0, c)

    def sync(self):
        if self._engine is not None:
            self._engine.synchronize()
