"""Device-resident particle-filter engine (one or many filters).

Python side of the pfe_* C ABI.  PyTorch supplies the device workspace and the
CUDA stream; every step runs the library's sm_100a kernels.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _native as N


@dataclass
class FilterSpec:
    n_particles: int
    seed: int = 42
    sigma_pos: Sequence[float] = (1.0, 1.0, 1.0)
    sigma_clk: float = 300.0
    sigma_pr: float = 5.0


@dataclass
class EngineOptions:
    n_clk: int = 1
    resampler: str = "systematic"          # "systematic" | "megopolis"
    megopolis_iters: int = 15
    weight_mode: str = "gaussian"          # "gaussian" | "huber" | "mixture" (learned, set_mlp) | "generic"
    huber_k: float = 1.5
    lw_mode: str = "overwrite"             # "overwrite" (reference) | "accumulate"
    sys_offset: str = "random"             # "random" | "reference"
    max_sats: int = 64
    obs_slots: int = 1
    covariance: bool = True
    recenter: bool = True
    ess_threshold: float = 0.5
    kernel_chain: bool = False             # one kernel per phase (comparison path)


def _torch():
    import torch  # noqa: WPS433 (import on use: torch is only the buffer/stream provider)
    if not torch.cuda.is_available():
        raise RuntimeError("CUDA is not available: the B200 particle filter has no CPU path")
    return torch


class Engine:
    """Many independent filters advanced together by fused kernels."""

    def __init__(self, filters: Sequence[FilterSpec], options: EngineOptions | None = None,
                 stream=None, device=None):
        torch = _torch()
        self._torch = torch
        self.lib = N.load()
        self.opt = options or EngineOptions()
        self.filters = list(filters)
        o = self.opt
        cfg = N.EngineConfig()
        cfg.n_filters = len(self.filters)
        cfg.n_clk = int(o.n_clk)
        cfg.resampler = {"systematic": N.PF_RESAMPLE_SYSTEMATIC, "megopolis": N.PF_RESAMPLE_MEGOPOLIS}[o.resampler]
        cfg.megopolis_iters = int(o.megopolis_iters)
        cfg.weight_mode = {"gaussian": N.PF_WEIGHT_GAUSSIAN, "huber": N.PF_WEIGHT_HUBER,
                           "mixture": N.PF_WEIGHT_MIXTURE, "generic": N.PF_WEIGHT_GENERIC}[o.weight_mode]
        cfg.lw_mode = {"overwrite": N.PF_LW_OVERWRITE, "accumulate": N.PF_LW_ACCUMULATE}[o.lw_mode]
        cfg.sys_offset = {"random": N.PF_SYS_OFFSET_RANDOM, "reference": N.PF_SYS_OFFSET_REFERENCE}[o.sys_offset]
        cfg.max_sats = int(o.max_sats)
        cfg.obs_slots = int(o.obs_slots)
        cfg.flags = ((N.PF_FLAG_COVARIANCE if o.covariance else 0) | (N.PF_FLAG_RECENTER if o.recenter else 0)
                     | (N.PF_FLAG_KERNEL_CHAIN if o.kernel_chain else 0))
        cfg.ess_threshold = float(o.ess_threshold)
        cfg.huber_k = float(o.huber_k)
        self.cfg = cfg
        self.D = 3 + cfg.n_clk
        self.params = (N.FilterParams * len(self.filters))()
        for k, f in enumerate(self.filters):
            self._fill_params(self.params[k], f)
        nbytes = C.c_size_t(0)
        N.check(self.lib.pfe_workspace_bytes(C.byref(cfg), self.params, C.byref(nbytes)))
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.workspace = torch.empty(int(nbytes.value), dtype=torch.uint8, device=self.device)
        self.stream = stream if stream is not None else torch.cuda.Stream(device=self.device)
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            N.check(self.lib.pfe_create(C.byref(cfg), self.params, C.c_void_p(self.workspace.data_ptr()),
                                        nbytes, C.c_void_p(self.stream.cuda_stream), C.byref(h)))
        self.h = h
        slot = C.c_size_t(0)
        N.check(self.lib.pfe_obs_slot_bytes(self.h, C.byref(slot)))
        self.obs_slot_bytes = int(slot.value)
        self._results = (N.FilterResult * len(self.filters))()

    @staticmethod
    def _fill_params(p, f: FilterSpec):
        p.n_particles = int(f.n_particles)
        p.seed = int(f.seed) & 0xFFFFFFFFFFFFFFFF
        sp = list(f.sigma_pos) if np.ndim(f.sigma_pos) else [float(f.sigma_pos)] * 3
        for a in range(3):
            p.sigma_pos[a] = float(sp[a])
        p.sigma_clk = float(f.sigma_clk)
        p.sigma_pr = float(f.sigma_pr)

    # ------------------------------------------------------------ lifecycle
    def close(self):
        if getattr(self, "h", None):
            self.lib.pfe_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_filter_params(self, k: int, f: FilterSpec):
        self.filters[k] = f
        self._fill_params(self.params[k], f)
        N.check(self.lib.pfe_set_filter_params(self.h, k, C.byref(self.params[k])))

    def initialize(self, k: int, anchor_ecef, clk0=0.0, spread_pos=100.0, spread_clk=1000.0):
        a = np.ascontiguousarray(anchor_ecef, dtype=np.float64).ravel()[:3].copy()
        c = np.zeros(N.PF_MAX_CLK)
        c[: self.cfg.n_clk] = np.broadcast_to(np.asarray(clk0, dtype=np.float64), (self.cfg.n_clk,))
        N.check(self.lib.pfe_initialize(self.h, k, N.dptr(a), N.dptr(c), float(spread_pos), float(spread_clk)))

    def frame(self, k: int):
        rot = np.zeros(9)
        anchor = np.zeros(3)
        N.check(self.lib.pfe_get_frame(self.h, k, N.dptr(rot), N.dptr(anchor)))
        return rot.reshape(3, 3), anchor

    # ---------------------------------------------------------------- inputs
    def pack_epoch(self, per_filter):
        """per_filter: list of dicts with keys disp (3,), sats (S,3), pr (S,),
        w (S,) [optional], clk (S,) [optional], cn0 / blocked (S,)
        [optional], flags (int).  One pass gathers the fields, then each
        column is filled for all filters at once (an optional column given by
        only some filters is filled filter by filter)."""
        F = len(self.filters)
        fe = np.zeros(F, N.FILTER_EPOCH_DTYPE)
        opt = ("w", "clk", "cn0", "blocked")
        sats_l, pr_l, counts = [], [], []
        given = {k: [] for k in opt}
        off = 0
        for k, r in enumerate(per_filter):
            d = r.get("disp")
            if d is not None:
                fe["disp"][k] = d
            fe["flags"][k] = int(r.get("flags", N.PF_EP_PREDICT | N.PF_EP_WEIGHT))
            sats = r.get("sats")
            s = 0 if sats is None else len(sats)
            fe["n_sat"][k] = s
            fe["sat_offset"][k] = off
            if s:
                sats_l.append(sats)
                pr_l.append(r["pr"])
                for key in opt:
                    v = r.get(key)
                    if v is not None:
                        given[key].append((off, s, v))
                off += s
        out = np.zeros(off, N.SAT_DTYPE)
        if off:
            xyz = np.concatenate([np.asarray(a, dtype=np.float64).reshape(-1, 3) for a in sats_l])
            out["x"], out["y"], out["z"] = xyz[:, 0], xyz[:, 1], xyz[:, 2]
            out["pr"] = np.concatenate([np.asarray(a, dtype=np.float64).ravel() for a in pr_l])
            out["w"] = 1.0
            out["cn0"] = 45.0
            for key in opt:
                g = given[key]
                if len(g) == len(sats_l) and g:
                    out[key] = np.concatenate([np.asarray(v).ravel() for _, _, v in g])
                else:
                    for a, n, v in g:
                        out[key][a:a + n] = np.asarray(v).ravel()
        return fe, out

    def upload(self, slot: int, fe: np.ndarray, sats: np.ndarray):
        fe = np.ascontiguousarray(fe, dtype=N.FILTER_EPOCH_DTYPE)
        sats = np.ascontiguousarray(sats, dtype=N.SAT_DTYPE)
        N.check(self.lib.pfe_upload_obs(self.h, int(slot), N.vptr(fe), N.vptr(sats) if len(sats) else None,
                                        len(sats)))

    # ------------------------------------------------------------------ steps
    def set_epoch_ctas_per_sm(self, ctas_per_sm: int) -> int:
        """Cap the epoch kernel's CTAs per SM (0 = all that fit); returns how
        many fit."""
        r = C.c_int(0)
        N.check(self.lib.pfe_set_epoch_ctas_per_sm(self.h, int(ctas_per_sm), C.byref(r)))
        return int(r.value)

    def set_likelihood(self, kind: str = "gaussian", nu: float = 0.0, huber_k: float = 1.5, w_los: float = 0.7,
                       mu_nlos: float = 15.0, sigma_nlos: float = 30.0, gate_m: float = 0.0):
        """Likelihood of a "generic" engine for the following steps: "gaussian",
        "student_t" (nu), "huber" (huber_k) or "gmm" (w_los, mu_nlos,
        sigma_nlos); gate_m > 0 adds the per-particle NLOS gate."""
        lk = N.Likelihood()
        lk.type = {"gaussian": N.PF_LIK_GAUSSIAN, "student_t": N.PF_LIK_STUDENT_T, "huber": N.PF_LIK_HUBER,
                   "gmm": N.PF_LIK_GMM}[kind]
        lk.nu, lk.huber_k, lk.w_los, lk.mu_nlos, lk.sigma_nlos, lk.gate_m = (
            float(nu), float(huber_k), float(w_los), float(mu_nlos), float(sigma_nlos), float(gate_m))
        N.check(self.lib.pfe_set_likelihood(self.h, C.byref(lk)))

    def shift(self, k: int, dpos_ecef, dclk=None):
        """Move every particle of filter k by dpos_ecef and its clocks by dclk."""
        dp = np.ascontiguousarray(dpos_ecef, dtype=np.float64).reshape(3)
        dc = None if dclk is None else np.ascontiguousarray(np.broadcast_to(np.asarray(dclk, np.float64),
                                                                              (self.cfg.n_clk,)))
        N.check(self.lib.pfe_shift(self.h, int(k), dp.ctypes.data_as(C.POINTER(C.c_double)),
                                   None if dc is None else dc.ctypes.data_as(C.POINTER(C.c_double))))

    def add_position_term(self, k: int, refs_ecef, sigma: float, log_pi=None):
        """log-weights += log sum_j pi_j N(p; ref_j, sigma^2 I) for filter k."""
        refs = np.ascontiguousarray(refs_ecef, dtype=np.float64).reshape(-1, 3)
        lp = None if log_pi is None else np.ascontiguousarray(log_pi, dtype=np.float64).ravel()
        N.check(self.lib.pfe_add_position_term(self.h, int(k), refs.ctypes.data_as(C.POINTER(C.c_double)),
                                               None if lp is None else lp.ctypes.data_as(C.POINTER(C.c_double)),
                                               len(refs), float(sigma)))

    def add_obs_term(self, k: int, kind: int, rows, sigma: float, gate: float = 0.0, huber_k: float = 0.0,
                     accumulate: bool = True):
        """Differenced / carrier-phase observation term over filter k's
        current particles (FP64 on the device).  rows: structured array of
        N.OBS_ROW_DTYPE."""
        r = np.ascontiguousarray(rows, dtype=N.OBS_ROW_DTYPE)
        N.check(self.lib.pfe_add_obs_term(self.h, int(k), int(kind), N.vptr(r) if len(r) else None, len(r),
                                          float(sigma), float(gate), float(huber_k), 1 if accumulate else 0))

    def add_3d_term(self, k: int, mesh, sats_ecef, pr, w, sigma_los: float, sigma_nlos: float, nlos_bias: float,
                    p_blocked: float, p_clear: float, accumulate: bool = False):
        """Building-aware pseudorange likelihood of filter k through `mesh`
        (an N.Mesh of a BVHAccelerator); overwrites the log-weights unless
        accumulate."""
        sats = np.ascontiguousarray(np.column_stack([np.asarray(sats_ecef, np.float64).reshape(-1, 3),
                                                     np.asarray(pr, np.float64).ravel(),
                                                     np.asarray(w, np.float64).ravel()]))
        N.check(self.lib.pfe_add_3d_term(self.h, int(k), C.byref(mesh), N.dptr(sats.reshape(-1)), len(sats),
                                         float(sigma_los), float(sigma_nlos), float(nlos_bias), float(p_blocked),
                                         float(p_clear), 1 if accumulate else 0))

    # ------------------------------------------------------ velocity states
    def velocity_states(self, k: int) -> "VelocityStates":
        """Per-particle velocity states of filter k (device memory allocated
        here, initialised by VelocityStates.init)."""
        return VelocityStates(self, k)

    def set_mlp(self, params):
        """Upload the NLOS network's parameters (mixture mode)."""
        prm = np.ascontiguousarray(params, dtype=np.float32)
        if prm.size != self.lib.pf_mlp_param_count():
            raise ValueError(f"expected {self.lib.pf_mlp_param_count()} parameters, got {prm.size}")
        N.check(self.lib.pfe_set_mlp(self.h, N.vptr(prm)))

    def sat_debug(self, k: int):
        """(n_sat, 16) per satellite of filter k's last weighted epoch: the 12
        features, p_nlos, mu, mode, residual against the prior mean."""
        out = np.zeros((self.cfg.max_sats, 16), np.float32)
        n = C.c_int(0)
        N.check(self.lib.pfe_get_sat_debug(self.h, int(k), N.vptr(out), self.cfg.max_sats, C.byref(n)))
        return out[: n.value]

    def step(self):
        N.check(self.lib.pfe_step(self.h))

    def step_io(self, fe: np.ndarray, sats: np.ndarray):
        """One epoch from host records to host results in one library call
        (upload into slot 0, step, read); returns the raw per-filter
        N.FilterResult array (reused by the next call).  Needs obs_slots == 1."""
        N.check(self.lib.pfe_step_io(self.h, N.vptr(fe), N.vptr(sats) if len(sats) else None, len(sats),
                                     C.byref(self._results)))
        return self._results

    def step_per_filter(self):
        N.check(self.lib.pfe_step_per_filter(self.h))

    def capture(self, per_filter: bool = False):
        N.check(self.lib.pfe_graph_capture(self.h, 1 if per_filter else 0))

    def replay(self, n: int = 1):
        N.check(self.lib.pfe_graph_launch(self.h, int(n)))

    def last_launch_count(self) -> int:
        c = C.c_int(0)
        N.check(self.lib.pfe_last_launch_count(self.h, C.byref(c)))
        return int(c.value)

    def synchronize(self):
        self.stream.synchronize()

    # ---------------------------------------------------------------- outputs
    def results(self):
        N.check(self.lib.pfe_read_results(self.h, self._results))
        out = []
        for r in self._results:
            out.append({
                "est_ecef": np.array(r.est_ecef[:]), "est_clk": np.array(r.est_clk[: self.cfg.n_clk]),
                "cov_enu": np.array(r.cov_enu[:]), "ess": r.ess, "sum_w": r.sum_w, "max_lw": r.max_lw,
                "resampled": bool(r.resampled), "epoch": r.epoch,
            })
        return out

    def results_array(self) -> np.ndarray:
        """The per-filter results as one structured array (fields est_ecef,
        est_clk, cov_enu, ess, sum_w, max_lw, resampled, epoch, initialized),
        a copy of pfe_read_results' records."""
        N.check(self.lib.pfe_read_results(self.h, self._results))
        return np.ctypeslib.as_array(self._results).copy()

    def result_bytes(self) -> int:
        b = C.c_size_t(0)
        N.check(self.lib.pfe_result_bytes(self.h, C.byref(b)))
        return int(b.value)

    def estimate(self, k: int) -> np.ndarray:
        out = np.zeros(self.D)
        N.check(self.lib.pfe_estimate(self.h, k, N.dptr(out)))
        return out

    def ess(self, k: int) -> float:
        v = C.c_double(0)
        N.check(self.lib.pfe_get_ess(self.h, k, C.byref(v)))
        return float(v.value)

    def current_ess(self, k: int) -> float:
        """ESS of filter k's current log-weights, recomputed on the device."""
        v = C.c_double(0)
        N.check(self.lib.pfe_current_ess(self.h, k, C.byref(v)))
        return float(v.value)

    def position_spread(self, k: int, center_ecef=None) -> float:
        """Weighted RMS distance of filter k's particles from center_ecef
        (default: their weighted mean), computed on the device."""
        v = C.c_double(0)
        c = None if center_ecef is None else np.ascontiguousarray(center_ecef, dtype=np.float64).reshape(3)
        N.check(self.lib.pfe_position_spread(self.h, k, None if c is None else N.vptr(c), C.byref(v)))
        return float(v.value)

    def particles(self, k: int) -> np.ndarray:
        n = self.filters[k].n_particles
        out = np.zeros((n, self.D))
        N.check(self.lib.pfe_get_particles(self.h, k, N.dptr(out)))
        return out

    def state_f32(self, k: int, raw: bool = False):
        """(state [D][N] FP32 local offsets, lw [N] FP32).  raw=True returns
        the buffers as the last step wrote them (before the resample gather)."""
        n = self.filters[k].n_particles
        st = np.zeros((self.D, n), np.float32)
        lw = np.zeros(n, np.float32)
        N.check(self.lib.pfe_get_state_f32(self.h, k, N.vptr(st), N.vptr(lw), 1 if raw else 0))
        return st, lw

    def anchor(self, k: int):
        """(anchor ECEF (3,), clock anchors (n_clk,), pending shift (D,))."""
        a = np.zeros(3)
        c = np.zeros(N.PF_MAX_CLK)
        sh = np.zeros(8, np.float32)
        N.check(self.lib.pfe_get_anchor(self.h, k, N.dptr(a), N.dptr(c), sh.ctypes.data_as(C.POINTER(C.c_float))))
        return a, c[: self.cfg.n_clk].copy(), sh[: self.D].copy()

    def set_state_f32(self, k: int, state, lw=None):
        st = np.ascontiguousarray(state, dtype=np.float32)
        assert st.shape == (self.D, self.filters[k].n_particles)
        lwa = None if lw is None else np.ascontiguousarray(lw, dtype=np.float32)
        N.check(self.lib.pfe_set_state_f32(self.h, k, N.vptr(st), None if lwa is None else N.vptr(lwa)))

    def checkpoint(self, k: int) -> bytes:
        """Filter k's complete state (control block with the FP64 anchors and
        the step counter of its random numbers, FP32 offsets, log-weights,
        ancestors) as bytes; restore() continues the filter bit for bit in an
        engine of the same configuration, particle count and seed."""
        nb = C.c_size_t(0)
        N.check(self.lib.pfe_checkpoint_bytes(self.h, k, C.byref(nb)))
        buf = np.empty(int(nb.value), np.uint8)
        N.check(self.lib.pfe_checkpoint_save(self.h, k, N.vptr(buf), buf.nbytes))
        return buf.tobytes()

    def restore(self, k: int, blob: bytes):
        buf = np.frombuffer(blob, np.uint8).copy()
        N.check(self.lib.pfe_checkpoint_load(self.h, k, N.vptr(buf), buf.nbytes))

    def sort_spatially(self, k: int, cell: float = 1.0):
        """Reorder filter k's particles (with their log-weights) by a Morton
        code of their East/North offsets in cells of `cell` metres, stably
        (ties keep their index order), so the order is deterministic.
        Particles are exchangeable, so the filter's distribution does not
        change; per-particle ray casts then run in spatially coherent
        warps, and since systematic resampling keeps ancestors in index
        order the population stays close to this order afterwards."""
        st, lw = self.state_f32(k)
        q = []
        for a in (st[0], st[1]):
            v = np.nan_to_num(a.astype(np.float64), nan=0.0)
            q.append(np.clip(np.floor((v - v.min()) / cell), 0, 65535).astype(np.uint64))
        key = np.zeros(len(lw), np.uint64)
        for b in range(16):
            one = np.uint64(1)
            key |= ((q[0] >> np.uint64(b)) & one) << np.uint64(2 * b)
            key |= ((q[1] >> np.uint64(b)) & one) << np.uint64(2 * b + 1)
        order = np.argsort(key, kind="stable")
        self.set_state_f32(k, np.ascontiguousarray(st[:, order]), np.ascontiguousarray(lw[order]))

    def ancestors(self, k: int) -> np.ndarray:
        out = np.zeros(self.filters[k].n_particles, np.int32)
        N.check(self.lib.pfe_get_ancestors(self.h, k, N.vptr(out)))
        return out

    def resample_info(self, k: int):
        u = C.c_uint32(0)
        w = C.c_uint64(0)
        m = C.c_float(0)
        N.check(self.lib.pfe_get_resample_info(self.h, k, C.byref(u), C.byref(w), C.byref(m)))
        return int(u.value), int(w.value), float(m.value)

    def error_word(self) -> int:
        w = C.c_uint(0)
        N.check(self.lib.pfe_error_word(self.h, C.byref(w)))
        return int(w.value)

    def set_spin_limit(self, limit: int):
        N.check(self.lib.pfe_set_spin_limit(self.h, int(limit)))

    def poison_lookback(self, on: bool):
        N.check(self.lib.pfe_test_poison_lookback(self.h, 1 if on else 0))

    def enable_timing(self, slots: int, detailed: bool = False):
        """Record CUDA events around the fused step kernel of each eager step
        (detailed: also after every resampling kernel, which serialises them)."""
        N.check(self.lib.pfe_enable_timing(self.h, int(slots), 1 if detailed else 0))
        self._timing_slots = int(slots)

    def read_timing(self):
        """(fused step kernel ms, whole step ms) per step since the last read."""
        n = max(1, getattr(self, "_timing_slots", 0))
        a = (C.c_float * n)()
        b = (C.c_float * n)()
        c = C.c_int(0)
        N.check(self.lib.pfe_read_timing(self.h, a, b, n, C.byref(c)))
        return np.array(a[: c.value]), np.array(b[: c.value])

    def read_timing_kernels(self):
        """Per-kernel ms of the steps returned by the last read_timing():
        (steps, 4) = fused step kernel, scan, offspring ends, merge path."""
        n = max(1, getattr(self, "_timing_slots", 0))
        a = (C.c_float * (4 * n))()
        c = C.c_int(0)
        N.check(self.lib.pfe_read_timing_kernels(self.h, a, n, C.byref(c)))
        return np.array(a[: 4 * c.value]).reshape(-1, 4)


class VelocityStates:
    """Per-particle ECEF velocity and 3x3 covariance (FP64) of one engine
    filter, in device memory beside the engine's particles (pfe_vel_*)."""

    NCOMP = 12

    def __init__(self, eng: Engine, k: int):
        torch = eng._torch
        self.eng, self.k = eng, int(k)
        self.n = eng.filters[k].n_particles
        # no fill: init() writes buffer 0, the resample gather writes buffer 1
        self.buf = torch.empty(2 * self.NCOMP * self.n, dtype=torch.float64, device=eng.device)
        self.vs = N.VelState()
        self.vs.buf = C.c_void_p(self.buf.data_ptr())
        self.vs.sel = 0
        self.vs.seq = 0

    def init(self, v0_ecef, spread_vel=0.0, init_sigma=0.0, step=0):
        v = np.ascontiguousarray(v0_ecef, dtype=np.float64).reshape(3)
        N.check(self.eng.lib.pfe_vel_init(self.eng.h, self.k, C.byref(self.vs), N.dptr(v), float(spread_vel),
                                          float(init_sigma), int(step) & 0xFFFFFFFF))

    def follow(self):
        N.check(self.eng.lib.pfe_vel_follow(self.eng.h, self.k, C.byref(self.vs)))

    def predict(self, guide_ecef, dt, sigma_pos, sigma_vel, alpha, kf, q, step):
        g = np.ascontiguousarray(guide_ecef, dtype=np.float64).reshape(3)
        N.check(self.eng.lib.pfe_vel_predict(self.eng.h, self.k, C.byref(self.vs), N.dptr(g), float(dt),
                                             float(sigma_pos), float(sigma_vel), float(alpha), 1 if kf else 0,
                                             float(q), int(step) & 0xFFFFFFFF))

    def doppler(self, sat_ecef, sat_vel, doppler_hz, weights, wavelength, sigma_mps, gain=0.0, max_update=0.0,
                kf=False):
        rows = np.zeros(len(doppler_hz), N.DOPPLER_ROW_DTYPE)
        rows["sat"] = np.asarray(sat_ecef, dtype=np.float64).reshape(-1, 3)
        rows["sat_vel"] = np.asarray(sat_vel, dtype=np.float64).reshape(-1, 3)
        rows["doppler_hz"] = np.asarray(doppler_hz, dtype=np.float64).ravel()
        rows["weight"] = np.asarray(weights, dtype=np.float64).ravel()
        N.check(self.eng.lib.pfe_vel_doppler(self.eng.h, self.k, C.byref(self.vs), N.vptr(rows), len(rows),
                                             float(wavelength), float(sigma_mps), float(gain), float(max_update),
                                             1 if kf else 0))

    def host(self):
        """(n, 12) FP64: velocity (3) then covariance row-major (9), current
        particle order (call follow() first after a resampling step)."""
        self.eng.synchronize()
        cur = self.buf[self.vs.sel * self.NCOMP * self.n:(self.vs.sel + 1) * self.NCOMP * self.n]
        return cur.view(self.NCOMP, self.n).t().cpu().numpy().copy()

    def set_host(self, arr):
        a = np.ascontiguousarray(np.asarray(arr, dtype=np.float64).reshape(self.n, self.NCOMP).T)
        torch = self.eng._torch
        cur = self.buf[self.vs.sel * self.NCOMP * self.n:(self.vs.sel + 1) * self.NCOMP * self.n]
        src = torch.from_numpy(a.reshape(-1))
        with torch.cuda.stream(self.eng.stream):
            cur.copy_(src.to(cur.device, non_blocking=False))
        self.eng.synchronize()
