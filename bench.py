#!/usr/bin/env python
"""Benchmark of the GNSS particle-filter step on B200.

One step = one epoch of predict -> weight -> (ESS-conditional) resample ->
estimate for every particle of the workload.  Default workload: the
1,000,000-particle x 32-satellite plain filter with four clock states
(7-D FP32 state about an FP64 anchor), systematic resampling when
ESS < N/2, synthetic seeded observations (cfg "drop-in at scale").

Prints ONE JSON line (rank 0).  Multi-GPU: one process per GPU, each an
independent replica of the workload (the path shards across independent
filters with no exchange), timed on the device, max over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--workload cfg1-systematic|cfg1-megopolis|cfg2-batched|cfg3-learned|
                              cfg4-batched-learned|device-filter|pf3d-city|orbits]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "PF particle-steps/s (1M particles x 32 satellites, predict+weight+resample+estimate)"
UNIT = "particle-steps/s"
L2_FLUSH_BYTES = 512 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="cfg1-systematic",
                    choices=["cfg1-systematic", "cfg1-megopolis", "cfg2-batched", "cfg3-learned",
                             "cfg4-batched-learned", "device-filter", "pf3d-city", "orbits"])
    ap.add_argument("--epochs", type=int, default=0, help="cfg3/cfg4: evaluated epochs (default 600 / 120)")
    ap.add_argument("--n-particles", type=int, default=1_000_000)
    ap.add_argument("--path", default="epoch", choices=["epoch", "chain"],
                    help="epoch: one cooperative kernel per step; chain: one kernel per phase")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--sigma-pr", type=float, default=3.0,
                    help="cfg1: pseudorange sigma of the likelihood (30 gives a wide posterior, ESS ~N/4, for traffic "
                         "profiles; the benchmark is 3)")
    ap.add_argument("--force-resample", action="store_true", help="cfg1: resample every epoch regardless of the ESS")
    ap.add_argument("--no-extras", action="store_true",
                    help="default workload at one GPU: skip the cfg1-megopolis, cfg2 and cfg3 keys")
    return ap.parse_args()


# --------------------------------------------------------------- process set
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def reduce_max(pg, value: float) -> float:
    if pg is None:
        return value
    import torch
    dev = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


# ----------------------------------------------------------------- clocks
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[4], parts[5], parts[6], parts[7], parts[8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        sm = np.array([r[0] for r in rows])
        mx = max(r[1] for r in rows)
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[3:]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        load = sm[sm >= 0.5 * sm.max()] if sm.max() > 0 else sm
        return {"sm_mhz": float(np.median(load)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(rows)}


def host_cpu():
    """Host CPU model, logical CPUs and the CPUs this process may run on."""
    model = ""
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"cpu_model": model, "logical_cpus": os.cpu_count(), "affinity": len(os.sched_getaffinity(0))}


# ------------------------------------------------------------- workloads
def cfg1_inputs(n_epochs: int, seed: int):
    from gnss_gpu_b200 import scenario as S
    return S.config1(n_epochs=n_epochs, seed=seed)


def epoch_record(tr, t, flags):
    return {"disp": tr.disp_enu[t], "sats": tr.sats[t], "pr": tr.pr[t], "clk": tr.clk_idx[t], "flags": flags}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic(kernel: str):
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get(kernel)
    return None


def cpu_baseline_cfg1(n: int, epochs: int, seed: int):
    """The oracle (FP64 C port of the reference's step, OpenMP on all host
    cores) on the same workload: predict, weight, ESS, systematic resample,
    estimate."""
    from oracle import oracle as O
    from gnss_gpu_b200 import scenario as S
    import ctypes as C
    tr = cfg1_inputs(epochs + 1, seed)
    D = 7
    x = O.init_state(n, D, 10.0, 30.0, 4242)
    x = np.ascontiguousarray(x.reshape(-1))
    xt = np.zeros_like(x)
    lw = np.zeros(n)
    lw32 = np.zeros(n, np.float32)
    anc = np.zeros(n, np.int32)
    anchor = np.ascontiguousarray(tr.truth_ecef[0])
    clk = np.ascontiguousarray(tr.truth_clk[0], dtype=np.float64)
    ca = np.zeros(4)
    ca[:4] = clk
    rot = np.ascontiguousarray(tr.rot.ravel())
    sigma = np.array([1, 1, 0.5, 0.5, 0.5, 0.5, 0.5, 0], np.float32)
    stats = np.zeros(24)
    L = O.lib()
    t0 = time.perf_counter()
    for t in range(epochs):
        rows = np.ascontiguousarray(np.column_stack([tr.sats[t], tr.pr[t], np.ones(len(tr.pr[t]))]).ravel())
        ci = np.ascontiguousarray(tr.clk_idx[t], np.int32)
        L.orc_epoch(n, D, x, xt, lw, lw32, anc, anchor, ca, rot, np.ascontiguousarray(tr.disp_enu[t]), sigma,
                    4242, 0, t + 1, len(tr.pr[t]), rows, ci, 3.0, 0.5, stats)
    dt = time.perf_counter() - t0
    return n * epochs / dt, O.num_threads(), dt


# ------------------------------------------------------------ b200 arm
def run_b200(args, world, rank, local, pg):
    import torch
    from gnss_gpu_b200 import _native as N
    from gnss_gpu_b200.engine import Engine, EngineOptions, FilterSpec
    from gnss_gpu_b200 import scenario as S

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    W, K = args.warmup, args.steps
    n = args.n_particles
    resampler = "megopolis" if args.workload == "cfg1-megopolis" else "systematic"
    E = W + K + 1
    tr = cfg1_inputs(E + K + 2, seed=1 + rank)
    opts = EngineOptions(n_clk=4, resampler=resampler, megopolis_iters=32, ess_threshold=0.5,
                         sys_offset="random", max_sats=32, obs_slots=E, covariance=True, recenter=True,
                         kernel_chain=args.path == "chain")
    spec = FilterSpec(n_particles=n, seed=1234 + rank, sigma_pos=(1.0, 1.0, 0.5), sigma_clk=0.5,
                      sigma_pr=args.sigma_pr)
    eng = Engine([spec], opts, device=local)
    eng.initialize(0, tr.truth_ecef[0], tr.truth_clk[0], 10.0, 30.0)
    flags = N.PF_EP_PREDICT | N.PF_EP_WEIGHT | (N.PF_EP_FORCE_RESAMPLE if args.force_resample else 0)
    for t in range(E):  # every input resident in HBM before timing
        fe, sv = eng.pack_epoch([epoch_record(tr, t, flags)])
        eng.upload(t, fe, sv)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    eng.enable_timing(K + W + 4)

    def one_step(t):
        with torch.cuda.stream(eng.stream):
            flush.fill_(t & 0xFF)  # evict the working set from L2 between steps
        eng.step()

    for t in range(W):
        one_step(t)
    eng.read_timing()
    eng.synchronize()
    barrier(pg)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    resampled = []
    errs = []
    for i in range(K):
        one_step(W + i)
        r = eng.results()[0]  # host read between steps (outside the device intervals)
        resampled.append(r["resampled"])
        truth = tr.truth_ecef[W + i]
        errs.append(float(np.linalg.norm((r["est_ecef"] - truth) @ tr.rot[:2].T)))
    torch.cuda.synchronize()
    barrier(pg)
    clk = clocks.stop()
    k_ms, step_ms = eng.read_timing()
    assert len(step_ms) == K, (len(step_ms), K)
    total_s = float(np.sum(step_ms)) / 1e3
    total_s = reduce_max(pg, total_s)
    kern_ms = float(np.mean(k_ms))
    value = n * K * world / total_s
    launches = K * eng.last_launch_count()

    # -------- e2e through the public API, host buffers, per step H2D + D2H
    e2e = None
    if not args.no_e2e:
        eng2 = Engine([spec], EngineOptions(n_clk=4, resampler=resampler, megopolis_iters=32, ess_threshold=0.5,
                                            max_sats=32, obs_slots=1, kernel_chain=args.path == "chain"),
                      device=local)
        eng2.initialize(0, tr.truth_ecef[0], tr.truth_clk[0], 10.0, 30.0)
        # each epoch's inputs as the C-ABI records (pf_filter_epoch_t + pf_sat_t) in host memory
        host_in = [eng2.pack_epoch([epoch_record(tr, i % len(tr.pr), flags)]) for i in range(K + W)]
        h2d = 0
        est = np.zeros((K + W, 3))
        wall = []
        for i in range(K + W):
            fe, sv = host_in[i]
            with torch.cuda.stream(eng2.stream):
                flush.fill_(i & 0xFF)      # evict L2, then let the device go idle: outside the timer
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = eng2.step_io(fe, sv)      # staged pinned H2D + step + D2H of the results + sync
            wall.append(time.perf_counter() - t0)
            est[i] = res[0].est_ecef[:]
            h2d = fe.nbytes + sv.nbytes
        assert np.all(np.isfinite(est))
        e2e_s = float(np.sum(wall[W:]))
        e2e_s = reduce_max(pg, e2e_s)
        e2e = {"value": n * K * world / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(eng2.result_bytes()), "ms_per_step": e2e_s / K * 1e3,
               "api": "gnss_gpu_b200.Engine.step_io per step (pfe_step_io: upload, step, read results)",
               "timing": "host clock around each call, from host inputs to host results; the L2 flush and a "
                         "device synchronize run before each timer starts"}
        eng2.close()

    peak, peak_kind = peaks()
    D = 7
    rs_frac = float(np.mean(resampled))
    # algorithmic bytes per particle-step (the scope table's B_alg = 2 D p + 2 q):
    # state read + write (2*D*4) and log-weight write + read (2*4) = 64 B at
    # D = 7.  Also reported: the same plus the ancestor write and the gather's
    # ancestor read of a resampling step (68 B when every step resamples).
    b_alg = 2 * D * 4 + 2 * 4
    b_alg_anc = 2 * D * 4 + 4 + 4 * rs_frac + 4 * rs_frac
    if args.path == "chain":
        kname = "k_step (fused predict+weight+statistics)"
        alg_k1 = (2 * D * 4 + 4 + 4 * rs_frac) * n
    else:
        kname = "k_epoch (cooperative predict+weight+statistics+resample)"
        alg_k1 = b_alg * n
    achieved = alg_k1 / (kern_ms / 1e3) / 1e9
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": total_s / K * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 state and log-weights / f64 anchor / exact integer CDF", "data": "synthetic",
        "config": {"workload": f"{args.workload}: 1 filter x {n} particles x 32 satellites (4 constellations x 8), "
                               f"D=7 (E,N,U + 4 clocks), sigma_pr {args.sigma_pr:g} m, 25% NLOS Exp(15 m), "
                               + ("every epoch " if args.force_resample else "ESS<N/2 ")
                               + f"{resampler} resampling" + (" (32 iterations)" if resampler == "megopolis" else ""),
                   "particles": n, "satellites": 32, "state_dim": D, "parallelism": f"replicas x{world}",
                   "path": args.path,
                   "l2": "flushed between steps (512 MiB device write outside the per-step event intervals)",
                   "inputs": "all epochs resident in HBM before timing"},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": kname,
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": f"{peak_kind} hbm_gbs", "algorithmic_bytes_per_launch": alg_k1,
                     "kernel_ms": kern_ms, "traffic": committed_traffic(kname.split()[0] + ":" + args.workload),
                     "traffic_wide_posterior": committed_traffic(kname.split()[0] + ":" + args.workload + "-wide"),
                     "traffic_note": "DRAM read + write per launch from one-pass ncu captures of the L2-flushed "
                                     "step (profiles/k_epoch_cfg1_dram.md): the benchmark's peaked posterior and a "
                                     "wide one (sigma_pr 30 m, ESS ~N/4, resampling every epoch)"},
        "step_roofline": {"b_alg_bytes_per_particle_step": b_alg,
                          "achieved_gbs": value / world * b_alg / 1e9,
                          "frac_of_measured_peak": value / world * b_alg / 1e9 / peak,
                          "frac_of_nominal_8tbs": value / world * b_alg / 1e9 / 8000.0,
                          "b_alg_with_ancestors": b_alg_anc,
                          "frac_of_measured_peak_with_ancestors": value / world * b_alg_anc / 1e9 / peak},
        "path": args.path,
        "resampled_fraction": rs_frac,
        "p50_2d_error_m": float(np.median(errs)),
        "clocks": clk,
    }
    if e2e:
        out["e2e"] = e2e
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # bounded sample of the same workload: one epoch to size it, then
        # about 10 s of CPU work on the full particle count
        _, _, dt1 = cpu_baseline_cfg1(n, 1, 7)
        epochs = int(max(2, min(200, 10.0 / max(dt1, 1e-3))))
        v, cores, dt = cpu_baseline_cfg1(n, epochs, 7)
        out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                               "sample": f"oracle FP64 C port (OpenMP), {n} particles x 32 satellites, "
                                         f"{epochs} epochs, {dt:.1f} s", **host_cpu()}
    eng.close()
    return out


# ------------------------------------------------------ cfg2: batched
def run_cfg2(args, world, rank, local, pg):
    """256 independent filters (particle counts log-uniform 1K-100K,
    6-40 satellites per filter and epoch, D = 4), all advanced by one
    cooperative launch per epoch replayed from a CUDA graph, against the
    same engine stepping the filters one launch each."""
    import torch
    from gnss_gpu_b200 import _native as N
    from gnss_gpu_b200.engine import Engine, EngineOptions, FilterSpec
    from gnss_gpu_b200 import scenario as S

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    W, K = args.warmup, args.steps
    E = W + K + 2
    n_part, trajs = S.batched(n_filters=256, n_epochs=E, seed=2 + rank)
    flags = N.PF_EP_PREDICT | N.PF_EP_WEIGHT
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)

    def make():
        specs = [FilterSpec(n_particles=int(nf), seed=100 + k, sigma_pos=(1.0, 1.0, 0.5), sigma_clk=0.5,
                            sigma_pr=3.0) for k, nf in enumerate(n_part)]
        eng = Engine(specs, EngineOptions(n_clk=1, resampler="systematic", ess_threshold=0.5, max_sats=40,
                                          obs_slots=E, covariance=True, recenter=True), device=local)
        for k, tr in enumerate(trajs):
            eng.initialize(k, tr.truth_ecef[0], tr.truth_clk[0], 10.0, 30.0)
        for t in range(E):
            recs = [{"disp": tr.disp_enu[t], "sats": tr.sats[t], "pr": tr.pr[t], "flags": flags} for tr in trajs]
            fe, sv = eng.pack_epoch(recs)
            eng.upload(t, fe, sv)
        return eng

    def timed(eng, fn, launches):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
        with torch.cuda.stream(eng.stream):
            for i in range(W):
                flush.fill_(i & 0xFF)
                fn()
            for i in range(K):
                flush.fill_(i & 0xFF)
                ev[i][0].record(eng.stream)
                fn()
                ev[i][1].record(eng.stream)
        eng.synchronize()
        barrier(pg)
        return reduce_max(pg, sum(a.elapsed_time(b) for a, b in ev) / 1e3)

    total_n = int(np.sum(n_part))
    clocks = ClockSampler(local)
    clocks.start()
    eng = make()
    eng.capture(False)
    t_graph = timed(eng, lambda: eng.replay(1), 1)
    eng.close()
    eng = make()
    t_pf = timed(eng, eng.step_per_filter, len(n_part))
    pf_launches = eng.last_launch_count()
    eng.close()
    eng = make()
    eng.capture(True)
    t_pfg = timed(eng, lambda: eng.replay(1), len(n_part))
    eng.close()
    clk = clocks.stop()
    # e2e: the same epochs from host records to host results through the
    # public one-call API (pfe_step_io: pinned upload, the batched launch,
    # one copy of every filter's results), host clock
    e2e = None
    if not args.no_e2e:
        specs = [FilterSpec(n_particles=int(nf), seed=100 + k, sigma_pos=(1.0, 1.0, 0.5), sigma_clk=0.5,
                            sigma_pr=3.0) for k, nf in enumerate(n_part)]
        eng = Engine(specs, EngineOptions(n_clk=1, resampler="systematic", ess_threshold=0.5, max_sats=40,
                                          obs_slots=1, covariance=True, recenter=True), device=local)
        for k, tr in enumerate(trajs):
            eng.initialize(k, tr.truth_ecef[0], tr.truth_clk[0], 10.0, 30.0)
        host_in = [eng.pack_epoch([{"disp": tr.disp_enu[t], "sats": tr.sats[t], "pr": tr.pr[t], "flags": flags}
                                   for tr in trajs]) for t in range(E)]
        wall, h2d = [], 0
        for t in range(W + K):
            fe, sv = host_in[t]
            with torch.cuda.stream(eng.stream):
                flush.fill_(t & 0xFF)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            eng.step_io(fe, sv)
            wall.append(time.perf_counter() - t0)
            h2d = max(h2d, fe.nbytes + sv.nbytes)
        e2e_s = reduce_max(pg, float(np.sum(wall[W:])))
        e2e = {"value": total_n * K * world / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(eng.result_bytes()), "ms_per_step": e2e_s / K * 1e3,
               "api": "gnss_gpu_b200.Engine.step_io per epoch (all 256 filters)",
               "timing": "host clock around each call; the L2 flush and a device synchronize run before each "
                         "timer starts"}
        eng.close()
    value = total_n * K * world / t_graph
    v_pf = total_n * K * world / t_pf
    peak, peak_kind = peaks()
    D = 4
    b_alg = 2 * D * 4 + 4 + 4 + 4  # state r+w, log-weight, ancestor read + write (resampling each epoch at most)
    achieved = value / world * b_alg / 1e9
    return {
        "metric": "PF particle-steps/s (256 batched uneven filters, 1 launch per epoch from a CUDA graph)",
        "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": t_graph / K * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 state and log-weights / f64 anchor / exact integer CDF", "data": "synthetic",
        "config": {"workload": f"cfg2-batched: 256 filters, particles log-uniform 1K-100K (total {total_n}), "
                               "6-40 satellites per filter and epoch, D=4, ESS<N/2 systematic resampling",
                   "particles": total_n, "filters": 256, "parallelism": f"replicas x{world}",
                   "l2": "flushed between steps (512 MiB device write outside the event intervals)"},
        "gpu_launches": K,
        "per_filter_launches": {"value": v_pf, "unit": UNIT, "ms_per_step": t_pf / K * 1e3,
                                "launches_per_step": pf_launches},
        "per_filter_launches_graph": {"value": total_n * K * world / t_pfg, "unit": UNIT,
                                      "ms_per_step": t_pfg / K * 1e3},
        "batched_over_per_filter": value / v_pf,
        "e2e": e2e,
        "roofline": {"bound": "hbm", "kernel": "k_epoch (cooperative, all filters)", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": f"{peak_kind} hbm_gbs",
                     "algorithmic_bytes_per_launch": b_alg * total_n, "traffic": committed_traffic("k_epoch:cfg2-batched")},
        "clocks": clk,
    }


# --------------------------------------------------- cfg3 / cfg4: learned
def train_network(rank: int):
    """The network of the learned likelihood: 2M satellite-epochs from 128
    drives x 650 epochs in 8 box cities (6-40 of 40 satellites per epoch),
    prior means from the plain robust filter (10K particles) on the GPU,
    3000 Adam steps of 8192 rows on the tensor-core kernels."""
    from gnss_gpu_b200 import learned as LR
    t0 = time.perf_counter()
    trs = LR.make_trajectories(128, 650, seed=100 + rank, n_sat=40, sat_range=(6, 40))
    r = LR.run_filters(trs, 10_000, "huber", seed=1, keep_priors=True)
    X, Y = LR.training_set(trs, r.priors)
    params, losses = LR.train(X, Y, steps=3000, batch=8192, lr=2e-3, seed=rank)
    p, _ = LR.predict(params, X[:200_000])
    acc = float(np.mean((p > 0.5) == (Y[:200_000, 0] > 0.5)))
    return params, {"rows": int(len(X)), "nlos_fraction": float(Y[:, 0].mean()), "adam_steps": 3000,
                    "batch": 8192, "loss_first": losses[0], "loss_last": losses[-1],
                    "nlos_accuracy_train": acc, "seconds": time.perf_counter() - t0}


def run_learned(args, world, rank, local, pg, cfg4: bool):
    import torch
    from gnss_gpu_b200 import learned as LR
    torch.cuda.set_device(local)
    params, training = train_network(rank)
    if cfg4:
        E = args.epochs or 120
        trs = LR.make_trajectories(1024, E, seed=200 + rank, n_sat=40, sat_range=(6, 40))
        rng = np.random.default_rng(7 + rank)
        n = np.exp(rng.uniform(np.log(10_000), np.log(1_000_000), len(trs)))
        n = np.maximum(1000, np.floor(n * min(1.0, 64e6 / n.sum()))).astype(int)  # total capped at 64M
        label = (f"cfg4-batched-learned: 1024 drives in 8 box cities, particles log-uniform 10K-1M scaled to "
                 f"{int(n.sum())} in total, 6-40 satellites per epoch, {E} epochs")
    else:
        E = args.epochs or 600
        trs = LR.make_trajectories(64, E, seed=300 + rank, n_sat=24)
        n = np.full(len(trs), 100_000)
        label = f"cfg3-learned: 64 held-out drives in 8 box cities, 100K particles x 24 satellites, {E} epochs"
    out_runs = {}
    for mode in ("huber", "mixture"):
        t0 = time.perf_counter()
        rr = LR.run_filters(trs, n, mode, params=params, seed=9 + rank)
        wall = time.perf_counter() - t0
        e = rr.err2d[:, 10:]
        out_runs[mode] = {"particle_steps_per_s": rr.steps_per_s, "e2e_particle_steps_per_s": float(n.sum()) * E / wall,
                          "p50_2d_m": float(np.median(e)), "rms_2d_m": float(np.sqrt(np.mean(e ** 2))),
                          "h2d": rr.h2d_bytes, "d2h": rr.d2h_bytes}
    total = int(n.sum())
    # whole-job rate: every rank did the same work, the slowest sets the time
    value = -reduce_max(pg, -out_runs["mixture"]["particle_steps_per_s"])
    peak, peak_kind = peaks()
    b_alg = 2 * 4 * 4 + 4 + 4 + 4
    achieved = value * b_alg / 1e9
    lm, pm = out_runs["mixture"], out_runs["huber"]
    return {
        "metric": "PF particle-steps/s with the learned NLOS mixture likelihood; P50 2D error learned vs plain",
        "value": value * world, "unit": UNIT, "n_gpus": world, "steps": E, "warmup": 0,
        "ms_per_step": total / value * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 state / f64 anchor; network bf16 x bf16 -> f32 on tensor cores", "data": "synthetic (box-city simulator)",
        "config": {"workload": label, "particles": total, "parallelism": f"replicas x{world}",
                   "l2": "working set larger than L2 (no flush)", "path": "epoch"},
        "gpu_launches": E,
        "accuracy": {"p50_2d_plain_m": pm["p50_2d_m"], "p50_2d_learned_m": lm["p50_2d_m"],
                     "rms_2d_plain_m": pm["rms_2d_m"], "rms_2d_learned_m": lm["rms_2d_m"],
                     "plain": "same engine, Huber likelihood (k = 1.5), same particles and seeds",
                     "epochs_scored": "all after the first 10"},
        "plain_particle_steps_per_s": pm["particle_steps_per_s"],
        "e2e": {"value": lm["e2e_particle_steps_per_s"], "unit": UNIT,
                "h2d_bytes_per_step": int(lm["h2d"]), "d2h_bytes_per_step": int(lm["d2h"]),
                "api": "learned.run_filters per epoch: prior geometry with the blocked flags ray-traced on the "
                       "device (pf_city_los), pack_epoch, upload, step, results"},
        "training": training,
        "roofline": {"bound": "hbm", "kernel": "k_epoch<.., mixture, systematic>", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": f"{peak_kind} hbm_gbs",
                     "algorithmic_bytes_per_particle_step": b_alg, "traffic": None},
    }


# --------------------------------------- ParticleFilterDevice drop-in
def cpu_baseline_d4(n: int, epochs: int, seed: int, sats, pr):
    """The oracle's FP64 step (OpenMP) with D = 4 and the given satellites:
    predict, Gaussian weight, ESS, systematic resample, estimate."""
    from oracle import oracle as O
    D = 4
    x = np.ascontiguousarray(O.init_state(n, D, 50.0, 200.0, 4242).reshape(-1))
    xt = np.zeros_like(x)
    lw = np.zeros(n)
    lw32 = np.zeros(n, np.float32)
    anc = np.zeros(n, np.int32)
    anchor = np.zeros(3)
    ca = np.array([100.0, 0.0, 0.0, 0.0])
    rot = np.ascontiguousarray(np.eye(3).ravel())
    sigma = np.array([1, 1, 1, 300, 0, 0, 0, 0], np.float32)
    stats = np.zeros(24)
    rows = np.ascontiguousarray(np.column_stack([sats, pr, np.ones(len(pr))]).ravel())
    ci = np.zeros(len(pr), np.int32)
    L = O.lib()
    t0 = time.perf_counter()
    for t in range(epochs):
        L.orc_epoch(n, D, x, xt, lw, lw32, anc, anchor, ca, rot, np.zeros(3), sigma, 4242, 0, t + 1, len(pr), rows,
                    ci, 5.0, 0.5, stats)
    dt = time.perf_counter() - t0
    return n * epochs / dt, O.num_threads(), dt


def run_device_filter(args, world, rank, local, pg):
    """ParticleFilterDevice, the reference's device-resident filter API:
    the predict + update cycle of its stream benchmark (8 satellites 20,000 km
    from a receiver at the ECEF origin, systematic resampling), at N
    particles, for three likelihoods.  value: device time of the cycles
    (CUDA events on the filter's stream, L2 flushed between cycles); e2e:
    the same cycles plus estimate() to the host, timed around the host calls."""
    import torch
    from gnss_gpu_b200 import ParticleFilterDevice
    torch.cuda.set_device(local)
    W, K = args.warmup, args.steps
    n = args.n_particles
    rng = np.random.RandomState(123)
    d = rng.randn(8, 3)
    sats = d / np.linalg.norm(d, axis=1, keepdims=True) * 20_000_000.0
    pr = np.linalg.norm(sats, axis=1) + 100.0
    pr[[1, 5]] += (30.0, 12.0)  # two NLOS-like delays
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=torch.device("cuda", local))
    variants = {"gaussian": dict(), "student_t_gate": dict(nu=4.0, per_particle_nlos_gate=True,
                                                            per_particle_nlos_undiff_pr_threshold_m=20.0),
                "gmm": dict()}
    res = {}
    clocks = ClockSampler(local)
    clocks.start()
    for name, kw in variants.items():
        pf = ParticleFilterDevice(n_particles=n, sigma_pos=1.0, sigma_cb=300.0, sigma_pr=5.0,
                                  resampling="systematic", seed=42 + rank, **kw)
        pf.initialize(np.zeros(3), clock_bias=100.0, spread_pos=50.0, spread_cb=200.0)
        stream = pf._engine.stream
        upd = (lambda: pf.update_gmm(sats, pr, None)) if name == "gmm" else (lambda: pf.update(sats, pr, None))
        for i in range(W):
            pf.predict(dt=1.0)
            upd()
        pf.sync()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(2 * K)]
        for i in range(K):  # device time of the cycle
            with torch.cuda.stream(stream):
                flush.fill_(i & 0xFF)
                ev[i][0].record(stream)
            pf.predict(dt=1.0)
            upd()
            with torch.cuda.stream(stream):
                ev[i][1].record(stream)
        pf.sync()
        est = []
        for i in range(K):  # e2e: cycle + estimate to the host
            with torch.cuda.stream(stream):
                flush.fill_(i & 0xFF)
                ev[K + i][0].record(stream)
            pf.predict(dt=1.0)
            upd()
            est.append(pf.estimate())
            with torch.cuda.stream(stream):
                ev[K + i][1].record(stream)
        pf.sync()
        dev_s = sum(a.elapsed_time(b) for a, b in ev[:K]) / 1e3
        e2e_s = sum(a.elapsed_time(b) for a, b in ev[K:]) / 1e3
        res[name] = {"value": n * K / reduce_max(pg, dev_s), "ms_per_cycle": dev_s / K * 1e3,
                     "e2e": n * K / reduce_max(pg, e2e_s), "e2e_ms_per_cycle": e2e_s / K * 1e3,
                     "launches_per_cycle": pf._engine.last_launch_count(),
                     "final_error_m": float(np.linalg.norm(est[-1][:3]))}
        pf._engine.close()
    clk = clocks.stop()
    peak, peak_kind = peaks()
    D = 4
    b_alg = 2 * D * 4 + 4 + 4 + 4
    g = res["gaussian"]
    achieved = g["value"] * b_alg / 1e9
    out = {
        "metric": "ParticleFilterDevice particle-steps/s (predict + update cycle, 8 satellites)",
        "value": g["value"] * world, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": g["ms_per_cycle"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 state / f64 anchor", "data": "synthetic (the reference stream benchmark's geometry)",
        "config": {"workload": f"device-filter: ParticleFilterDevice, {n} particles x 8 satellites, D=4, "
                               "sigma_pr 5 m, systematic resampling when ESS<N/2",
                   "particles": n, "satellites": 8, "parallelism": f"replicas x{world}",
                   "l2": "flushed between cycles (outside the event intervals)"},
        "gpu_launches": K * g["launches_per_cycle"],
        "likelihoods": res,
        "e2e": {"value": g["e2e"] * world, "unit": UNIT, "h2d_bytes_per_step": 56 * 8 + 64,
                "d2h_bytes_per_step": 8 * 4, "api": "ParticleFilterDevice.predict/update/estimate per cycle"},
        "roofline": {"bound": "hbm", "kernel": "k_epoch<generic> (+ k_estimate in e2e)", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": f"{peak_kind} hbm_gbs",
                     "algorithmic_bytes_per_launch": b_alg * n, "traffic": None},
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        _, _, dt1 = cpu_baseline_d4(n, 1, 7, sats, pr)
        epochs = int(max(2, min(400, 10.0 / max(dt1, 1e-3))))
        v, cores, dt = cpu_baseline_d4(n, epochs, 7, sats, pr)
        out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                               "sample": f"oracle FP64 C port (OpenMP), Gaussian, {n} particles x 8 satellites, "
                                         f"{epochs} epochs, {dt:.1f} s"}
    return out


# ----------------------------------------- building-aware (3D) filter
def run_pf3d(args, world, rank, local, pg):
    """ParticleFilter3DBVH's update on the device: 1M particles x 16
    satellites, shadow rays through a 2 km box city (about 10K triangles in
    the hierarchy), then the ESS test and resampling.  value: particle-steps/s
    of the whole update (ray-traced likelihood + resample step), device
    events, L2 flushed; rays_per_s of the likelihood kernel alone."""
    import torch
    from gnss_gpu_b200 import BVHAccelerator
    from gnss_gpu_b200 import _native as N
    from gnss_gpu_b200 import citysim as CS
    from gnss_gpu_b200 import scenario as S
    from gnss_gpu_b200.engine import Engine, EngineOptions, FilterSpec
    torch.cuda.set_device(local)
    W, K = args.warmup, args.steps
    n = args.n_particles
    S_ = 16
    city = CS.make_city(11 + rank, size=2000.0, cell=40.0)
    rot = S.enu_rotation_lla(35.63, 139.78)
    anchor = S.lla_to_ecef(35.63, 139.78, 40.0)
    tri = CS.city_triangles(city, anchor, rot)
    bvh = BVHAccelerator(tri)
    rng = np.random.default_rng(5 + rank)
    b = city.box[city.occ]
    while True:
        e_, n_ = rng.uniform(200.0, 1800.0, 2)
        if not np.any((b[:, 0] - 3 <= e_) & (e_ <= b[:, 1] + 3) & (b[:, 2] - 3 <= n_) & (n_ <= b[:, 3] + 3)):
            break
    truth = anchor + np.array([e_, n_, 1.5]) @ rot
    az = rng.uniform(0, 2 * np.pi, S_)
    el = rng.uniform(np.radians(10), np.radians(80), S_)
    sats = truth + 2.2e7 * (np.stack([np.cos(el) * np.sin(az), np.cos(el) * np.cos(az), np.sin(el)], 1) @ rot)
    blocked = ~bvh.check_los(truth, sats)
    pr = np.linalg.norm(sats - truth, axis=1) + 80.0 + np.where(blocked, 25.0, 0.0) + rng.normal(0, 1.0, S_)
    w = np.ones(S_)
    eng = Engine([FilterSpec(n_particles=n, seed=7, sigma_pos=(0.5, 0.5, 0.5), sigma_clk=1.0, sigma_pr=3.0)],
                 EngineOptions(n_clk=1, max_sats=S_, ess_threshold=0.5))
    eng.initialize(0, truth, 80.0, 20.0, 5.0)
    eng.sort_spatially(0)  # as ParticleFilter3DBVH.initialize does
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=torch.device("cuda", local))
    fe, sv = eng.pack_epoch([{"disp": np.zeros(3), "flags": N.PF_EP_PREDICT | N.PF_EP_RESAMPLE_CHECK}])
    eng.upload(0, fe, sv)

    def update():
        eng.add_3d_term(0, bvh.mesh, sats, pr, w, 3.0, 30.0, 20.0, 1.0, 0.0)
        eng.step()   # predict noise of the next epoch folded in, ESS test, resampling

    for _ in range(W):
        update()
    eng.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    clocks = ClockSampler(local)
    clocks.start()
    for i in range(K):
        with torch.cuda.stream(eng.stream):
            flush.fill_(i & 0xFF)
            ev[i][0].record(eng.stream)
        eng.add_3d_term(0, bvh.mesh, sats, pr, w, 3.0, 30.0, 20.0, 1.0, 0.0)
        with torch.cuda.stream(eng.stream):
            ev[i][1].record(eng.stream)
        eng.step()
        with torch.cuda.stream(eng.stream):
            ev[i][2].record(eng.stream)
    eng.synchronize()
    clk = clocks.stop()
    t_term = reduce_max(pg, sum(a.elapsed_time(b_) for a, b_, _ in ev) / 1e3)
    t_all = reduce_max(pg, sum(a.elapsed_time(c) for a, _, c in ev) / 1e3)
    est = eng.estimate(0)
    out = {
        "metric": "ParticleFilter3DBVH update particle-steps/s (1M particles x 16 satellites, ray-traced city)",
        "value": n * K * world / t_all, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": t_all / K * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "rays f32 in the mesh frame, ranges and likelihood f64", "data": "synthetic (box city)",
        "config": {"workload": f"pf3d-city: {n} particles x {S_} satellites, 2 km box city, {len(tri)} triangles, "
                               f"{bvh.n_nodes} hierarchy nodes, systematic resampling when ESS<N/2",
                   "particles": n, "satellites": S_, "triangles": int(len(tri)), "parallelism": f"replicas x{world}",
                   "l2": "flushed between steps (outside the event intervals)"},
        "gpu_launches": 2 * K,
        "likelihood_kernel": {"ms_per_step": t_term / K * 1e3, "rays_per_s": n * S_ * K * world / t_term},
        "blocked_satellites_at_truth": int(blocked.sum()),
        "estimate_error_m": float(np.linalg.norm(est[:3] - truth)),
        "roofline": None,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        m = 50_000
        t0 = time.perf_counter()
        pts = truth + rng.normal(0, 20.0, (m, 3))
        O.weight_3d(pts, np.full(m, 80.0), np.column_stack([sats, pr, w]), tri, 3.0, 30.0, 20.0, 1.0, 0.0)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": m / dt, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
                               "sample": f"oracle FP64 brute-force ray casting (the reference's ParticleFilter3D "
                                         f"kernel restated), {m} particles x {S_} satellites x {len(tri)} triangles, "
                                         f"{dt:.1f} s"}
    eng.close()
    return out


def run_orbits(args, world, rank, local, pg):
    """Input formation on the device: broadcast orbits and clocks of one day
    at 1 Hz (86,400 epochs) x 64 satellites (40 Kepler records of G/E/J/C
    re-selected every 2 h, 24 GLONASS states re-selected every 30 min and
    integrated by RK4 from their toe), one pf_broadcast_orbits call per
    step (three kernels: GLONASS steps needed, shared GLONASS states, the
    orbits).  value: satellite-epochs/s, inputs resident; e2e: the public
    broadcast_orbits call with host arrays (records, index and times up,
    positions and clocks down)."""
    import ctypes as C
    import torch
    from gnss_gpu_b200 import _native as N
    from gnss_gpu_b200.ephemeris import broadcast_orbits
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    W, K = args.warmup, args.steps
    n_epoch = args.epochs or 86_400
    rng = np.random.default_rng(21 + rank)
    n_kep, n_glo = 40, 24
    kep_sets, glo_sets = 12, 48
    n_rec = n_kep * kep_sets + n_glo * glo_sets
    recs = np.zeros(n_rec, N.BROADCAST_DTYPE)
    sys_k = np.array([ord(c) for c in "G" * 16 + "E" * 12 + "J" * 4 + "C" * 8])
    for s in range(n_kep):
        for j in range(kep_sets):
            r = s * kep_sets + j
            recs["system"][r] = sys_k[s]
            k = recs["kepler"][r:r + 1]
            k["sqrt_a"] = 5153.6 if sys_k[s] != ord("C") else 5282.6
            k["e"] = rng.uniform(0.001, 0.02)
            k["i0"], k["omega0"], k["omega"] = rng.uniform(0.9, 1.0), rng.uniform(-3, 3), rng.uniform(-3, 3)
            k["M0"], k["delta_n"], k["omega_dot"] = rng.uniform(-3, 3), 4.5e-9, -8e-9
            k["crc"], k["crs"], k["cuc"], k["cus"] = 220.0, -14.0, -3e-6, 7e-6
            k["toe"] = k["toc"] = 7200.0 * j + 3600.0
            k["af0"], k["af1"], k["tgd"] = rng.uniform(-1e-4, 1e-4), -1e-12, -1e-8
    base = n_kep * kep_sets
    for s in range(n_glo):
        ang = 2 * np.pi * s / n_glo
        for j in range(glo_sets):
            r = base + s * glo_sets + j
            recs["system"][r] = ord("R")
            g = recs["glonass"][r:r + 1]
            g["toe"] = 1800.0 * j + 900.0
            g["pos"] = (2.55e7 * np.cos(ang), 2.55e7 * np.sin(ang), 0.0)
            v = np.sqrt(3.9860044e14 / 2.55e7)
            g["vel"] = (-v * np.sin(ang) * 0.5, v * np.cos(ang) * 0.5, v * 0.86)
            g["tau_n"], g["gamma_n"] = 1e-5, 1e-12
    t = np.arange(n_epoch, dtype=np.float64) + 18.0
    idx = np.empty((n_epoch, n_kep + n_glo), np.int32)
    kj = np.clip(np.floor((t - 3600.0) / 7200.0 + 0.5), 0, kep_sets - 1).astype(np.int32)
    gj = np.clip(np.floor((t - 18.0 - 900.0) / 1800.0 + 0.5), 0, glo_sets - 1).astype(np.int32)
    for s in range(n_kep):
        idx[:, s] = s * kep_sets + kj
    for s in range(n_glo):
        idx[:, n_kep + s] = base + s * glo_sets + gj
    S_ = n_kep + n_glo
    d_rec = torch.from_numpy(recs.view(np.uint8).copy()).to(dev)
    d_idx = torch.from_numpy(idx).to(dev)
    d_t = torch.from_numpy(t).to(dev)
    d_pos = torch.empty((n_epoch, S_, 3), dtype=torch.float64, device=dev)
    d_clk = torch.empty((n_epoch, S_), dtype=torch.float64, device=dev)
    st = torch.cuda.Stream(dev)
    L = N.load()
    ptr = lambda x: C.c_void_p(x.data_ptr())  # noqa: E731
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)

    def launch():
        N.check(L.pf_broadcast_orbits(ptr(d_rec), n_rec, ptr(d_idx), ptr(d_t), n_epoch, S_, 60.0, ptr(d_pos),
                                      ptr(d_clk), C.c_void_p(st.cuda_stream)))

    for _ in range(W):
        launch()
    st.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    clocks = ClockSampler(local)
    clocks.start()
    for i in range(K):
        with torch.cuda.stream(st):
            flush.fill_(i & 0xFF)
            ev[i][0].record(st)
        launch()
        with torch.cuda.stream(st):
            ev[i][1].record(st)
    st.synchronize()
    clk = clocks.stop()
    t_dev = reduce_max(pg, sum(a.elapsed_time(b_) for a, b_ in ev) / 1e3)
    units = n_epoch * S_
    out_bytes = units * 32 + units * 4 + n_epoch * 8
    ms = t_dev / K * 1e3
    peak, peak_kind = peaks()
    out = {
        "metric": "broadcast orbit satellite-epochs/s (positions + clocks, multi-GNSS)",
        "value": units * K * world / t_dev, "unit": "satellite-epochs/s", "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic broadcast records",
        "config": {"workload": f"orbits: {n_epoch} epochs x {S_} satellites ({n_kep} Kepler G/E/J/C re-selected "
                               f"every 2 h, {n_glo} GLONASS RK4 from toe re-selected every 30 min), "
                               f"{n_rec} records",
                   "epochs": n_epoch, "satellites": S_, "parallelism": f"replicas x{world}",
                   "l2": "flushed between steps (outside the event intervals)"},
        "gpu_launches": 3 * K,  # k_glo_need, k_glo_table, k_broadcast_orbits
        "roofline": {"bound": "hbm", "achieved": out_bytes / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": out_bytes / (ms / 1e3) / 1e9 / peak, "peak_kind": f"{peak_kind} hbm_gbs",
                     "traffic": None,
                     "note": "FP64 math (Kepler iterations, sin/cos/atan2, RK4) bounds this kernel, "
                             "not HBM: 36 B moved per satellite-epoch"},
        "clocks": clk,
    }
    if not args.no_e2e:
        ts = []
        for i in range(max(3, min(K, 5))):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            pos, clk_h = broadcast_orbits(recs, t, idx)
            ts.append(time.perf_counter() - t0)
        e2e_t = float(np.median(ts))
        out["e2e"] = {"value": units * world / e2e_t, "unit": "satellite-epochs/s",
                      "h2d_bytes_per_step": int(recs.nbytes + idx.nbytes + t.nbytes),
                      "d2h_bytes_per_step": int(units * 32), "timing": "host clock, median of calls"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import orbit as OO
        m = 600
        t0 = time.perf_counter()
        for s in range(S_):
            for r in np.unique(idx[:m, s]):
                e_ = np.nonzero(idx[:m, s] == r)[0]
                if recs["system"][r] == ord("R"):
                    g = recs["glonass"][r]
                    st_ = {"toe": float(g["toe"]), "pos": g["pos"], "vel": g["vel"], "acc": g["acc"],
                           "tau_n": float(g["tau_n"]), "gamma_n": float(g["gamma_n"])}
                    for e in e_:
                        OO.glonass(st_, float(t[e]))
                else:
                    rec = {f: float(recs["kepler"][f][r]) for f in N.EPHEMERIS_FIELDS}
                    OO.kepler(rec, chr(recs["system"][r]), t[e_])
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": m * S_ / dt, "unit": "satellite-epochs/s", "cores": 1, "kind": "port",
                               "sample": f"oracle FP64 (numpy Kepler per record, Python RK4 per GLONASS "
                                         f"epoch), first {m} epochs x {S_} satellites, {dt:.1f} s"}
    return out


# ------------------------------------- the rest of the metric, one GPU
def run_extras(args, world, rank, local, pg):
    """The other halves of the headline metric, bounded to a few minutes, as
    extra keys of the default line: cfg1 with 32 Megopolis iterations, the
    256 batched filters against per-filter launches, and the learned
    likelihood against the plain robust filter (P50 / RMS 2D error)."""
    import copy
    out = {}
    a = copy.copy(args)
    a.workload, a.no_e2e, a.no_cpu_baseline = "cfg1-megopolis", True, True
    m = run_b200(a, world, rank, local, pg)
    out["cfg1_megopolis"] = {"value": m["value"], "unit": UNIT, "ms_per_step": m["ms_per_step"],
                             "steps": m["steps"], "resampled_fraction": m["resampled_fraction"],
                             "roofline_frac_64B": m["value"] * 64 / 1e9 / m["roofline"]["peak"],
                             "roofline": m["roofline"], "clocks": m["clocks"],
                             "workload": m["config"]["workload"]}
    a = copy.copy(args)
    a.workload, a.no_e2e = "cfg2-batched", False
    c2 = run_cfg2(a, world, rank, local, pg)
    out["cfg2"] = {"value": c2["value"], "unit": UNIT, "ms_per_step": c2["ms_per_step"], "steps": c2["steps"],
                   "per_filter_launches": c2["per_filter_launches"],
                   "per_filter_launches_graph": c2["per_filter_launches_graph"],
                   "batched_over_per_filter": c2["batched_over_per_filter"],
                   "e2e": c2["e2e"], "roofline": c2["roofline"], "clocks": c2["clocks"],
                   "workload": c2["config"]["workload"]}
    a = copy.copy(args)
    a.workload = "cfg3-learned"
    c3 = run_learned(a, world, rank, local, pg, False)
    out["cfg3"] = {"value": c3["value"], "unit": UNIT, "plain_particle_steps_per_s": c3["plain_particle_steps_per_s"],
                   "accuracy": c3["accuracy"], "e2e": c3["e2e"], "training": c3["training"],
                   "workload": c3["config"]["workload"]}
    return out


# ------------------------------------------------------- reference arm
def reference_gpu_cfg1(n: int, steps: int):
    """The reference's own GPU path on this GPU: its stock ParticleFilter
    class (python/gnss_gpu/particle_filter.py) over its _gnss_gpu_pf module,
    as installed unmodified into baseline/_ref (CUDA built for sm_100a).  A
    step is predict + update (weight, ESS, systematic resampling when
    ESS < N/2) + estimate, as in the reference's benchmarks/
    bench_particle_filter.py:53-145.  Every call moves the full FP64 particle
    arrays between host and device, which is the reference's design.  It has
    one clock state, so the four constellations' clocks are one state here."""
    import torch
    ref = ROOT / "baseline" / "_ref"
    if not (ref / "gnss_gpu" / "particle_filter.py").exists():
        return {"unavailable": "baseline/_ref holds no reference install"}
    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}
    sys.path.insert(0, str(ref))
    try:
        from gnss_gpu.particle_filter import ParticleFilter as RefPF
    finally:
        sys.path.remove(str(ref))
    tr = cfg1_inputs(steps + 4, 21)
    pf = RefPF(n_particles=n, sigma_pos=1.0, sigma_cb=0.5, sigma_pr=3.0, resampling="systematic",
               ess_threshold=0.5, seed=42)
    pf.initialize(tr.truth_ecef[0], clock_bias=float(tr.truth_clk[0][0]), spread_pos=10.0, spread_cb=30.0)

    def step(t):
        vel = tr.disp_enu[t] @ tr.rot  # ENU displacement per 1 s epoch -> ECEF velocity
        pf.predict(velocity=vel, dt=1.0)
        pf.update(tr.sats[t], tr.pr[t])
        return pf.estimate()

    for t in range(2):
        step(t)
    t0 = time.perf_counter()
    k = 0
    while k < steps and (k < 3 or time.perf_counter() - t0 < 20.0):
        step(2 + k)
        k += 1
    dt = time.perf_counter() - t0
    return {"value": n * k / dt, "unit": UNIT, "ms_per_step": dt / k * 1e3, "steps": k,
            "api": "gnss_gpu.ParticleFilter predict + update + estimate (reference, baseline/_ref)",
            "timing": "host clock; every reference call synchronises the device and copies to the host",
            "config": f"{n} particles x 32 satellites, one clock state, systematic resampling when ESS<N/2"}


def run_reference(args, world, rank):
    if rank != 0:
        return None
    W, K = args.warmup, args.steps
    n = args.n_particles
    from oracle import oracle as O
    # bounded sample: the full workload, at most a few seconds per step
    t0 = time.perf_counter()
    v_w, cores, _ = cpu_baseline_cfg1(n, max(1, min(W, 1)), 11)
    per_step = (time.perf_counter() - t0)
    k_eff = max(1, min(K, int(60.0 / max(per_step, 1e-3))))
    v, cores, dt = cpu_baseline_cfg1(n, k_eff, 12)
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": k_eff,
        "warmup": 1, "ms_per_step": dt / k_eff * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.workload}: 1 filter x {n} particles x 32 satellites, D=7, "
                               "systematic resampling when ESS<N/2 (CPU restatement of the reference step)",
                   "parallelism": "host cores (OpenMP)"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{n} particles x {k_eff} epochs, {dt:.1f} s", **host_cpu()},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    if args.workload == "cfg1-systematic":
        try:
            out["reference_gpu"] = reference_gpu_cfg1(n, max(3, K))
        except Exception as exc:  # a stated extra, never the arm itself
            out["reference_gpu"] = {"unavailable": f"{type(exc).__name__}: {exc}"[:200]}
    return out


def main():
    args = parse()
    world, rank, local, pg = dist_setup(args)
    if args.impl == "reference":
        out = run_reference(args, world, rank)
    elif args.workload == "cfg2-batched":
        out = run_cfg2(args, world, rank, local, pg)
    elif args.workload == "device-filter":
        out = run_device_filter(args, world, rank, local, pg)
    elif args.workload == "pf3d-city":
        out = run_pf3d(args, world, rank, local, pg)
    elif args.workload == "orbits":
        out = run_orbits(args, world, rank, local, pg)
    elif args.workload in ("cfg3-learned", "cfg4-batched-learned"):
        out = run_learned(args, world, rank, local, pg, args.workload == "cfg4-batched-learned")
    else:
        out = run_b200(args, world, rank, local, pg)
        if args.workload == "cfg1-systematic" and world == 1 and not args.no_extras:
            out.update(run_extras(args, world, rank, local, pg))
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
