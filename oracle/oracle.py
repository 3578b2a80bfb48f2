"""ctypes wrapper of the FP64 CPU oracle (oracle/pf_oracle.c).

Test infrastructure only: imported by tests/, by __graft_entry__.smoke() as the
checker, and by bench.py's CPU-baseline leg.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "pf_oracle.c"
LIB = HERE / "liboracle.so"

_lib = None

F64 = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
F32 = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
I32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
U64 = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
U32 = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")

TAG_SYS_U = 0x03000000


def build(force: bool = False) -> Path:
    if force or not LIB.exists() or LIB.stat().st_mtime < SRC.stat().st_mtime:
        tmp = LIB.with_suffix(".so.tmp")
        subprocess.run(["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
                        "-std=gnu11", str(SRC), "-o", str(tmp), "-lm"], check=True)
        os.replace(tmp, LIB)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        u32, i32, f32, f64 = C.c_uint32, C.c_int, C.c_float, C.c_double
        P = C.c_void_p
        L.orc_philox10.argtypes = [U32, u32, u32, U32]
        L.orc_quant_exponent.argtypes = [i32]
        L.orc_quant_exponent.restype = i32
        L.orc_quantize.argtypes = [f64, i32]
        L.orc_quantize.restype = C.c_uint64
        L.orc_quantize_all.argtypes = [F32, i32, f32, U64]
        L.orc_quantize_all64.argtypes = [F64, i32, f64, U64]
        L.orc_systematic64.argtypes = [F64, i32, f64, u32, I32, C.POINTER(C.c_uint64)]
        L.orc_systematic64.restype = i32
        L.orc_systematic.argtypes = [F32, i32, f32, u32, I32, C.POINTER(C.c_uint64)]
        L.orc_systematic.restype = i32
        L.orc_systematic_tiled.argtypes = [F32, i32, u32, I32, C.POINTER(C.c_uint64), C.POINTER(C.c_float)]
        L.orc_systematic_tiled.restype = i32
        L.orc_det_expf.argtypes = [f32]
        L.orc_det_expf.restype = f32
        L.orc_quantize_f32.argtypes = [f32, i32]
        L.orc_quantize_f32.restype = C.c_uint64
        L.orc_megopolis.argtypes = [F32, i32, i32, u32, u32, u32, u32, I32]
        L.orc_init.argtypes = [i32, i32, f32, f32, u32, u32, u32, F64]
        L.orc_predict.argtypes = [i32, i32, F64, P, F64, F64, F32, i32, u32, u32, u32, u32, F64]
        L.orc_weight.argtypes = [i32, i32, F64, F64, F64, F64, i32, F64, I32, f64, i32, f64, P, F64]
        L.orc_stats.argtypes = [i32, i32, F64, F64, F64, F64, F64, F64]
        L.orc_epoch.argtypes = [i32, i32, F64, F64, F64, F32, I32, F64, F64, F64, F64, F32, u32, u32,
                                u32, i32, F64, I32, f64, f64, F64]
        L.orc_epoch.restype = i32
        L.orc_pf_initialize.argtypes = [F64, F64, F64, F64, f64, f64, f64, f64, f64, f64, i32, C.c_ulonglong]
        L.orc_pf_predict.argtypes = [F64, F64, F64, F64, f64, f64, f64, f64, f64, f64, i32, C.c_ulonglong, i32]
        L.orc_pf_weight.argtypes = [F64, F64, F64, F64, F64, F64, F64, F64, i32, i32, f64]
        L.orc_pf_ess.argtypes = [F64, i32]
        L.orc_pf_ess.restype = f64
        L.orc_pf_estimate.argtypes = [F64, F64, F64, F64, F64, F64, i32]
        L.orc_pf_systematic_ancestors.argtypes = [F64, i32, C.c_ulonglong, I32]
        L.orc_pf_systematic_ancestors.restype = i32
        L.orc_pf_megopolis_ref_ancestors.argtypes = [F64, i32, i32, C.c_ulonglong, I32]
        L.orc_num_threads.restype = i32
        L.orc_set_threads.argtypes = [i32]
        U8 = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
        L.orc_los.argtypes = [F64, F64, i32, i32, F64, i32, U8]
        L.orc_weight_3d.argtypes = [i32, F64, F64, i32, F64, F64, i32, f64, f64, f64, f64, f64, F64, P]
        _lib = L
    return _lib


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


# ------------------------------------------------------------------ RNG
def philox10(ctr, key):
    out = np.zeros(4, np.uint32)
    lib().orc_philox10(np.asarray(ctr, np.uint32), int(key[0]), int(key[1]), out)
    return out


def seed_key(seed: int):
    seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    return seed & 0xFFFFFFFF, seed >> 32


# ------------------------------------------------------------ quantiser
def quant_exponent(n: int) -> int:
    return int(lib().orc_quant_exponent(int(n)))


def quantize(lw32, max_lw) -> np.ndarray:
    lw32 = _f32(lw32)
    q = np.zeros(len(lw32), np.uint64)
    lib().orc_quantize_all(lw32, len(lw32), float(np.float32(max_lw)), q)
    return q


def systematic(lw32, max_lw, u32):
    """Ancestor of every slot and the integer weight total."""
    lw32 = _f32(lw32)
    anc = np.zeros(len(lw32), np.int32)
    w = C.c_uint64(0)
    r = lib().orc_systematic(lw32, len(lw32), float(np.float32(max_lw)), int(u32), anc, C.byref(w))
    if r != 0:
        raise ValueError("all weights quantised to zero")
    return anc, int(w.value)


def systematic_tiled(lw32, u32):
    """The engine's systematic resampler: ancestor of every slot, the integer
    weight total W and the filter maximum, from the tiled integer CDF (each
    128-particle segment quantised against its own maximum and rescaled
    exactly to the tile and filter maxima; pf_oracle.c)."""
    lw32 = _f32(lw32)
    anc = np.zeros(len(lw32), np.int32)
    w = C.c_uint64(0)
    m = C.c_float(0.0)
    r = lib().orc_systematic_tiled(lw32, len(lw32), int(u32), anc, C.byref(w), C.byref(m))
    if r == -2:
        raise MemoryError("oracle allocation")
    return anc, int(w.value)


def det_expf(d: float) -> float:
    return float(lib().orc_det_expf(float(d)))


def quantize_f32(d: float, K: int) -> int:
    return int(lib().orc_quantize_f32(float(d), int(K)))


def megopolis(lw32, iters, seed, epoch, filter_id=0):
    lw32 = _f32(lw32)
    anc = np.zeros(len(lw32), np.int32)
    k0, k1 = seed_key(seed)
    lib().orc_megopolis(lw32, len(lw32), int(iters), k0, k1, int(epoch), int(filter_id), anc)
    return anc


# ----------------------------------------------------- engine semantics
def init_state(n, D, spread_pos, spread_clk, seed, filter_id=0):
    x = np.zeros(D * n, np.float64)
    k0, k1 = seed_key(seed)
    lib().orc_init(n, D, float(np.float32(spread_pos)), float(np.float32(spread_clk)), k0, k1,
                   int(filter_id), x)
    return x.reshape(D, n)


def predict(x_prev, anc, disp, shift, sigma, do_predict, seed, epoch, filter_id=0):
    x_prev = _f64(x_prev)
    D, n = x_prev.shape
    out = np.zeros((D, n), np.float64)
    sh = np.zeros(8)
    sh[:len(shift)] = shift
    sg = np.zeros(8, np.float32)
    sg[:len(sigma)] = sigma
    anc_p = None if anc is None else np.ascontiguousarray(anc, np.int32)
    k0, k1 = seed_key(seed)
    lib().orc_predict(n, D, x_prev, None if anc_p is None else anc_p.ctypes.data, _f64(disp), sh, sg,
                      int(bool(do_predict)), k0, k1, int(epoch), int(filter_id), out)
    return out


def weight(x, anchor, clk_anchor, rot, sats, clk, sigma_pr, mode=0, huber_k=1.5, lw_base=None):
    """sats: (S, 5) rows x, y, z, pr, w."""
    x = _f64(x)
    D, n = x.shape
    sats = _f64(sats).reshape(-1, 5)
    ca = np.zeros(4)
    ca[:len(clk_anchor)] = clk_anchor
    out = np.zeros(n, np.float64)
    base = None if lw_base is None else _f64(lw_base)
    lib().orc_weight(n, D, x, _f64(anchor), ca, _f64(rot).ravel(), len(sats), sats.ravel(),
                     np.ascontiguousarray(clk, np.int32), float(sigma_pr), int(mode), float(huber_k),
                     None if base is None else base.ctypes.data, out)
    return out


def weight_mixture(x, anchor, clk_anchor, rot, sats, sigma_pr, p_nlos, mu, mode, huber_k=1.5):
    """FP64 log-weights of the learned two-component likelihood (the epoch
    kernel's PF_WEIGHT_MIXTURE, one clock state): per satellite with mode 0
    log((1-p) N(r; 0, s2) + p N(r; mu, s2 + mu^2)) without the common
    -log(2 pi)/2, with s2 = sigma_pr^2 / w; mode 1 the Huber term; mode 2
    nothing.  x: (D, n) offsets about `anchor` in the E/N/U frame `rot`;
    sats: (S, 5) rows x, y, z, pr, w."""
    x = _f64(x)
    sats = _f64(sats).reshape(-1, 5)
    pos = _f64(anchor)[None, :] + x[:3].T @ _f64(rot)          # (n, 3) ECEF
    cb = clk_anchor[0] + x[3]
    lw = np.zeros(x.shape[1])
    for s in range(len(sats)):
        rng = np.linalg.norm(sats[s, :3][None, :] - pos, axis=1)
        r = sats[s, 3] - rng - cb
        w = sats[s, 4]
        if mode[s] > 1.5 or w <= 0:
            continue
        if mode[s] > 0.5:
            z = np.abs(r) / sigma_pr
            rho = np.where(z < huber_k, 0.5 * z * z, huber_k * z - 0.5 * huber_k * huber_k)
            lw -= w * rho
            continue
        s2 = sigma_pr * sigma_pr / w
        sn2 = s2 + mu[s] ** 2
        a = np.log1p(-p_nlos[s]) - 0.5 * np.log(s2) - r * r / (2 * s2)
        b = np.log(p_nlos[s]) - 0.5 * np.log(sn2) - (r - mu[s]) ** 2 / (2 * sn2)
        lw += np.logaddexp(a, b)
    return lw


def weight_generic(x, anchor, clk_anchor, rot, sats, sigma_pr, kind="gaussian", nu=0.0, huber_k=1.5,
                   w_los=0.7, mu_nlos=15.0, sigma_nlos=30.0, gate_m=0.0):
    """FP64 log-weights of the device filter's likelihoods, one clock state.

    Per satellite with residual r = pr - |sat - p| - cb and weight w:
      gaussian   -w r^2 / (2 sigma^2)                          pf_device.cu:273-275
      student_t  -(nu + 1)/2 log(1 + w r^2 / (nu sigma^2))      pf_device.cu:265-266
      huber      -w rho_k(|r| / sigma)                         pf_device.cu:19-26,267-268
      gmm        log(w_los/sigma exp(-w r^2/(2 sigma^2))
                     + (1-w_los)/sigma_nlos exp(-w (r-mu)^2/(2 sigma_nlos^2)))
                                                               pf_device.cu:415-428
    gate_m > 0: a particle drops the satellites with |r| > gate_m unless
    fewer than min(n_sat, 4) would remain (pf_device.cu:236-258).
    Satellites of weight <= 0 are skipped.  x: (D, n) offsets about
    `anchor` in the E/N/U frame `rot`; sats: (S, 5) rows x, y, z, pr, w.
    Also returns the (S, n) residuals."""
    x = _f64(x)
    sats = _f64(sats).reshape(-1, 5)
    pos = _f64(anchor)[None, :] + x[:3].T @ _f64(rot)
    cb = clk_anchor[0] + x[3]
    S = len(sats)
    res = np.empty((S, x.shape[1]))
    for s in range(S):
        res[s] = sats[s, 3] - np.linalg.norm(sats[s, :3][None, :] - pos, axis=1) - cb
    use = np.ones_like(res, dtype=bool)
    if gate_m > 0.0:
        inside = np.abs(res) <= gate_m
        gate_on = inside.sum(axis=0) >= min(S, 4)
        use = inside | ~gate_on[None, :]
    lw = np.zeros(x.shape[1])
    for s in range(S):
        r, w = res[s], sats[s, 4]
        if w <= 0.0:
            continue
        if kind == "student_t":
            t = -0.5 * (nu + 1.0) * np.log1p(w * r * r / (nu * sigma_pr * sigma_pr))
        elif kind == "huber":
            z = np.abs(r) / sigma_pr
            t = -w * np.where(z < huber_k, 0.5 * z * z, huber_k * z - 0.5 * huber_k * huber_k)
        elif kind == "gmm":
            a = np.log(w_los) - np.log(sigma_pr) - 0.5 * w * r * r / (sigma_pr * sigma_pr)
            b = np.log(1.0 - w_los) - np.log(sigma_nlos) - 0.5 * w * (r - mu_nlos) ** 2 / (sigma_nlos * sigma_nlos)
            t = np.logaddexp(a, b)
        else:
            t = -0.5 * w * r * r / (sigma_pr * sigma_pr)
        lw += np.where(use[s], t, 0.0)
    return lw, res


OBS_DD_PSEUDORANGE, OBS_CARRIER_AFV, OBS_DD_CARRIER_AFV = 0, 1, 2


def obs_term(x, anchor, clk_anchor, rot, kind, sat_k, obs, weight, sat_ref=None, base_k=None, base_ref=None,
             wavelength=None, sigma=1.0, gate=0.0, huber_k=0.0):
    """FP64 sum over rows of the differenced / carrier-phase terms, per
    particle, in ECEF as the reference computes them:
      DD pseudorange   r = dd - (|p - s_k| - |p - s_ref| - b_k + b_ref)        pf_device.cu:282-368
      carrier AFV      a = afv(cp - (|p - s| + cb) / lambda)                   pf_device.cu:439-494
      DD carrier AFV   a = afv(dd - (|p - s_k| - |p - s_ref| - b_k + b_ref) / lambda)
                                                                               pf_device.cu:496-604
    afv(v) = v - rint(v); cost w r^2 / (2 sigma^2) or the Huber cost
    (huber_k > 0, pf_device.cu:19-26); DD kinds: gate > 0 drops rows with
    |r| > gate unless fewer than min(n, 3) remain.  Returns (-sum of costs,
    residuals (n_rows, n))."""
    x = _f64(x)
    pos = _f64(anchor)[None, :] + x[:3].T @ _f64(rot)
    cb = clk_anchor[0] + x[3]
    sat_k = _f64(sat_k).reshape(-1, 3)
    n_rows = len(sat_k)
    res = np.empty((n_rows, x.shape[1]))
    for i in range(n_rows):
        rk = np.linalg.norm(pos - sat_k[i][None, :], axis=1)
        if kind == OBS_CARRIER_AFV:
            v = obs[i] - (rk + cb) / wavelength[i]
            res[i] = v - np.rint(v)
            continue
        rr = np.linalg.norm(pos - _f64(sat_ref).reshape(-1, 3)[i][None, :], axis=1)
        dd_expected = rk - rr - base_k[i] + base_ref[i]
        if kind == OBS_DD_PSEUDORANGE:
            res[i] = obs[i] - dd_expected
        else:
            v = obs[i] - dd_expected / wavelength[i]
            res[i] = v - np.rint(v)
    use = np.ones_like(res, dtype=bool)
    if gate > 0.0 and kind != OBS_CARRIER_AFV:
        inside = np.abs(res) <= gate
        on = inside.sum(axis=0) >= min(n_rows, 3)
        use = inside | ~on[None, :]
    lw = np.zeros(x.shape[1])
    for i in range(n_rows):
        v = res[i]
        if huber_k > 0.0:
            z = np.abs(v) / sigma
            cost = weight[i] * np.where(z < huber_k, 0.5 * z * z, huber_k * z - 0.5 * huber_k * huber_k)
        else:
            cost = 0.5 * weight[i] * v * v / (sigma * sigma)
        lw -= np.where(use[i], cost, 0.0)
    return lw, res


# ------------------------------------------------ per-particle velocity
TAG_VEL_INIT, TAG_VEL_PREDICT = 0x06000000, 0x07000000


def vel_normals(j, step, tag, seed, filter_id=0):
    """The eight standard normals of particle slot j for a velocity draw:
    Philox4x32-10 blocks (j, step, tag, filter) and (j, step, tag | 1,
    filter), Box-Muller in FP64 (u1 = (a + 1/2) 2^-32, u2 = b 2^-32 - 1/2)."""
    k = seed_key(seed)
    w = np.concatenate([philox10([j, step, tag, filter_id], k), philox10([j, step, tag | 1, filter_id], k)])
    z = np.empty(8)
    for i in range(4):
        u1 = (float(w[2 * i]) + 0.5) * 2.0 ** -32
        u2 = float(w[2 * i + 1]) * 2.0 ** -32 - 0.5
        r = np.sqrt(-2.0 * np.log(u1))
        z[2 * i], z[2 * i + 1] = r * np.cos(2.0 * np.pi * u2), r * np.sin(2.0 * np.pi * u2)
    return z


def vel_predict(pos, v, P, guide, dt, sigma_pos, sigma_vel, alpha, kf, q, step, seed):
    """Velocity predict of pf_device.cu:106-187 with this project's draws:
    v = (1 - a) v + a g (+ sigma_vel z[0:3] unless kf); positions += v dt +
    noise, the noise L z[0:3] with L the Cholesky factor of
    sigma_pos^2 I + dt^2 P (kf; then P += q dt I) or sigma_pos z[k:k+3].
    pos, v: (n, 3) ECEF; P: (n, 9) row-major.  Returns new copies."""
    pos, v, P = np.array(pos, float), np.array(v, float), np.array(P, float)
    a = min(1.0, max(0.0, alpha))
    for j in range(len(pos)):
        z = vel_normals(j, step, TAG_VEL_PREDICT, seed)
        vj = (1.0 - a) * v[j] + a * np.asarray(guide, float)
        zi = 0
        if not kf and sigma_vel > 0.0:
            vj = vj + z[0:3] * sigma_vel
            zi = 3
        v[j] = vj
        if kf:
            Pj = P[j]
            dt2, s2 = dt * dt, sigma_pos * sigma_pos
            a00, a01, a02 = s2 + dt2 * Pj[0], dt2 * Pj[1], dt2 * Pj[2]
            a11, a12, a22 = s2 + dt2 * Pj[4], dt2 * Pj[5], s2 + dt2 * Pj[8]
            l00 = np.sqrt(max(a00, 0.0))
            l10 = a01 / l00 if l00 > 1e-12 else 0.0
            l20 = a02 / l00 if l00 > 1e-12 else 0.0
            l11 = np.sqrt(max(a11 - l10 * l10, 0.0))
            l21 = (a12 - l20 * l10) / l11 if l11 > 1e-12 else 0.0
            l22 = np.sqrt(max(a22 - l20 * l20 - l21 * l21, 0.0))
            nz = np.array([l00 * z[0], l10 * z[0] + l11 * z[1], l20 * z[0] + l21 * z[1] + l22 * z[2]])
            qdt = max(q, 0.0) * max(dt, 0.0)
            P[j, [0, 4, 8]] += qdt
        else:
            nz = z[zi:zi + 3] * sigma_pos
        pos[j] = pos[j] + vj * dt + nz
    return pos, v, P


def _solve4(A):
    A = A.copy()
    for col in range(4):
        mr = col
        for row in range(col + 1, 4):
            if abs(A[row, col]) > abs(A[mr, col]):
                mr = row
        if mr != col:
            A[[col, mr]] = A[[mr, col]]
        if abs(A[col, col]) < 1e-12:
            return None
        for row in range(col + 1, 4):
            f = A[row, col] / A[col, col]
            A[row, col:] -= f * A[col, col:]
    x = np.zeros(4)
    for row in range(3, -1, -1):
        x[row] = (A[row, 4] - A[row, row + 1:4] @ x[row + 1:4]) / A[row, row]
    return x


def doppler(pos, v, P, sat, sat_vel, doppler_hz, weights, wavelength, sigma, gain=0.0, max_update=0.0, kf=False):
    """Per-particle Doppler terms in FP64: pf_device.cu:610-748 (kf False:
    clock drift per particle, Gaussian likelihood, blend toward the WLS
    velocity) and pf_device.cu:750-887 (kf True: sequential velocity KF,
    innovation likelihood).  Returns (log_w (n,), v, P) copies."""
    pos, v, P = np.array(pos, float), np.array(v, float), np.array(P, float)
    n = len(pos)
    lw = np.zeros(n)
    obs = -np.asarray(doppler_hz, float) * wavelength
    w_all = np.maximum(np.asarray(weights, float), 0.0)
    for j in range(n):
        d = sat - pos[j]
        r = np.linalg.norm(d, axis=1)
        ok = r >= 1.0
        los = d / np.where(ok, r, 1.0)[:, None]
        svr = np.sum(sat_vel * los, axis=1)
        if not kf:
            rxr = los @ v[j]
            wsum = float(np.sum(w_all[ok]))
            if wsum <= 0.0:
                continue
            cd = float(np.sum((w_all * (obs - svr + rxr))[ok])) / wsum
            pred = np.sum((sat_vel - v[j]) * los, axis=1) + cd
            res = obs - pred
            lw[j] = float(np.sum((-0.5 * w_all * res * res / (sigma * sigma))[ok]))
            g = min(1.0, max(0.0, gain))
            if g <= 0.0 or len(obs) < 4:
                continue
            A = np.zeros((4, 5))
            for s in np.nonzero(ok)[0]:
                h = np.array([-los[s, 0], -los[s, 1], -los[s, 2], 1.0])
                rhs = obs[s] - svr[s]
                A[:, 4] += h * w_all[s] * rhs
                A[:, :4] += np.outer(h, h) * w_all[s]
            A[range(4), range(4)] += 1e-9
            sol = _solve4(A)
            if sol is None:
                continue
            dv = sol[:3] - v[j]
            nrm = np.linalg.norm(dv)
            if max_update > 0.0 and nrm > max_update:
                dv = dv * (max_update / max(nrm, 1e-9))
            v[j] = v[j] + g * dv
        else:
            use = ok & (w_all > 0.0)
            wsum = float(np.sum(w_all[use]))
            if wsum <= 0.0:
                continue
            hm = np.sum(-los[use] * w_all[use, None], axis=0) / wsum
            ym = float(np.sum(w_all[use] * (obs - svr)[use])) / wsum
            Pj = P[j].reshape(3, 3).copy()
            mu = v[j].copy()
            for s in np.nonzero(use)[0]:
                h = -los[s] - hm
                yc = (obs[s] - svr[s]) - ym
                ph = Pj @ h
                S = float(h @ ph) + sigma * sigma / w_all[s]
                if not (S > 1e-18) or not np.isfinite(S):
                    continue
                innov = yc - float(h @ mu)
                K = ph / S
                mu = mu + K * innov
                Pj = Pj - np.outer(K, h @ Pj)
                for a_, b_ in ((0, 1), (0, 2), (1, 2)):
                    m = 0.5 * (Pj[a_, b_] + Pj[b_, a_])
                    Pj[a_, b_] = Pj[b_, a_] = m if np.isfinite(m) else 0.0
                for a_ in range(3):
                    Pj[a_, a_] = Pj[a_, a_] if (np.isfinite(Pj[a_, a_]) and Pj[a_, a_] > 1e-12) else 1e-12
                lw[j] += -0.5 * (innov * innov / S + np.log(S))
            v[j] = mu
            P[j] = Pj.reshape(9)
    return lw, v, P


# ------------------------------------------------ building-aware likelihood
def los(rx, sat, tris):
    """Line of sight by brute-force FP64 ray casting (weight_3d.cu:14-48):
    rx (R, 3), sat (R, S, 3), tris (T, 3, 3) ECEF -> (R, S) bool."""
    rx = _f64(rx).reshape(-1, 3)
    sat = _f64(sat).reshape(len(rx), -1, 3)
    tri = _f64(tris).reshape(-1, 9)
    out = np.zeros(sat.shape[:2], np.uint8)
    lib().orc_los(rx, sat.reshape(-1), len(rx), sat.shape[1], tri.reshape(-1), len(tri), out.reshape(-1))
    return out.astype(bool)


def weight_3d(pos, cb, sats, tris, sigma_los, sigma_nlos, nlos_bias, p_blocked, p_clear):
    """FP64 log-weights of the building-aware likelihood (weight_3d.cu:86-177)
    and the (n, S) blocked flags.  pos (n, 3) ECEF, cb (n,), sats (S, 5)
    rows x, y, z, pr, w, tris (T, 3, 3)."""
    pos = _f64(pos).reshape(-1, 3)
    n = len(pos)
    sv = _f64(sats).reshape(-1, 5)
    tri = _f64(tris).reshape(-1, 9)
    lw = np.zeros(n)
    blk = np.zeros((n, len(sv)), np.uint8)
    lib().orc_weight_3d(n, pos.reshape(-1), _f64(cb).reshape(-1), len(sv), sv.reshape(-1), tri.reshape(-1), len(tri),
                        float(sigma_los), float(sigma_nlos), float(nlos_bias), float(p_blocked), float(p_clear), lw,
                        blk.ctypes.data)
    return lw, blk.astype(bool)


def stats(x, lw, anchor, clk_anchor, rot):
    x = _f64(x)
    D, n = x.shape
    ca = np.zeros(4)
    ca[:len(clk_anchor)] = clk_anchor
    out = np.zeros(24)
    lib().orc_stats(n, D, x, _f64(lw), _f64(anchor), ca, _f64(rot).ravel(), out)
    return {
        "max_lw": out[0], "sum_w": out[1], "sum_w2": out[2], "ess": out[3],
        "mean": out[4:4 + D].copy(), "est_ecef": out[11:14].copy(),
        "est_clk": out[14:14 + D - 3].copy(), "cov": out[18:24].copy(),
    }


def sys_offset_random(seed, epoch, filter_id=0):
    return int(philox10([0, epoch, TAG_SYS_U, filter_id], seed_key(seed))[0])


# ------------------------------------------- reference host-array semantics
def pf_initialize(init, init_cb, spread_pos, spread_cb, n, seed):
    px, py, pz, pcb = (np.zeros(n) for _ in range(4))
    lib().orc_pf_initialize(px, py, pz, pcb, float(init[0]), float(init[1]), float(init[2]),
                            float(init_cb), float(spread_pos), float(spread_cb), int(n), int(seed))
    return px, py, pz, pcb


def pf_predict(px, py, pz, pcb, v, dt, sp, scb, seed, step):
    px, py, pz, pcb = (_f64(a).copy() for a in (px, py, pz, pcb))
    lib().orc_pf_predict(px, py, pz, pcb, float(v[0]), float(v[1]), float(v[2]), float(dt), float(sp),
                         float(scb), len(px), int(seed), int(step))
    return px, py, pz, pcb


def pf_weight(px, py, pz, pcb, sat, pr, ws, sigma_pr):
    lw = np.zeros(len(px))
    sat = _f64(sat).ravel()
    lib().orc_pf_weight(_f64(px), _f64(py), _f64(pz), _f64(pcb), sat, _f64(pr), _f64(ws), lw, len(px),
                        len(_f64(pr)), float(sigma_pr))
    return lw


def pf_ess(lw):
    lw = _f64(lw)
    return float(lib().orc_pf_ess(lw, len(lw)))


def pf_estimate(px, py, pz, pcb, lw):
    out = np.zeros(4)
    lib().orc_pf_estimate(_f64(px), _f64(py), _f64(pz), _f64(pcb), _f64(lw), out, len(px))
    return out


def pf_systematic_ancestors(lw, seed):
    lw = _f64(lw)
    anc = np.zeros(len(lw), np.int32)
    if lib().orc_pf_systematic_ancestors(lw, len(lw), int(seed), anc) != 0:
        raise ValueError("all weights quantised to zero")
    return anc


def pf_megopolis_ref_ancestors(lw, iters, seed):
    lw = _f64(lw)
    anc = np.zeros(len(lw), np.int32)
    lib().orc_pf_megopolis_ref_ancestors(lw, len(lw), int(iters), int(seed), anc)
    return anc


def num_threads() -> int:
    return int(lib().orc_num_threads())


def set_threads(n: int):
    lib().orc_set_threads(int(n))
