#!/usr/bin/env python
"""Benchmark: Langevin sweeps/s of quenched SU(3) NSPT on B200.

Workload (default): 32^4 lattice, 24 perturbative orders, FP64 complex 3x3
series links (~14.5 GB per field), twisted boundary conditions in y and z,
Euler dt = 0.005, plain Jacobi Langevin sweep (no gauge fixing in the timed
step), noise from the device Philox generator, field resident in HBM.

One step = one full sweep over all 4 V links.  `value` is whole-job sweeps/s
(sum over replicas: every rank runs its own independent lattice, so scaling is
weak, "replicas only").  `e2e` is the same metric through the public C ABI
with the configuration on the host: upload, K sweeps each reading the
plaquette / norm / trU back, download -- host<->device copies inside the
timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Langevin sweeps/s at 32^4 x 24 orders (FP64, twisted y,z)"
GF_ALPHA = -0.05


def canonical_flops_per_link(N: int) -> float:
    """14 series products + 1 series exp per link update; a 3x3 complex
    multiply-accumulate is 216 flops; a truncated product of N-order series
    is N(N-1)/2 of them, the pruned exp C(N+1,3)."""
    P = N * (N - 1) // 2
    E = (N - 1) * N * (N + 1) // 6
    return (14 * P + E) * 216.0


def algorithmic_bytes_per_sweep(V: int, N: int) -> float:
    """Read U and write U' once (order-0 flags not counted)."""
    return 2.0 * 4 * V * 9 * N * 16


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    mx = max(mx, float(p[2]))
                except ValueError:
                    continue
                for n, v in zip(names, p[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        except OSError:
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "samples": len(sm), "reasons": sorted(reasons)}


def barrier(world: int):
    import torch
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def dist_setup():
    from prlgt2020_b200.replicas import world_info
    return world_info()


def read_profile_value(key: str, path: str = "profiles/sweep_32x4_n24_traffic.txt"):
    """A per-launch figure of the sweep kernel from a committed ncu summary
    (`key: value` lines)."""
    try:
        for line in open(os.path.join(ROOT, path)):
            if line.startswith(key + ":"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def read_profile_traffic():
    """DRAM bytes (read + write) of one 32^4 x 24 sweep-kernel launch, from
    the committed ncu summary (a 16^4 capture scaled by the link count)."""
    return read_profile_value("traffic_bytes_per_launch")


def executed_fraction(N: int, V: int, kernel_ms: float, peak: float):
    """The FP64 rate the sweep kernel executes (not the canonical count):
    DFMA thread instructions per link from the committed ncu summary of the
    benchmark kernel (profiles/k_sweep_16x16x16x8_n24_full.md, key
    dfma_thread_inst_per_link) x 2 flops x the 4V links of this sweep, over
    the kernel time measured here.  Only for the 24-order benchmark shape."""
    per_link = read_profile_value("dfma_thread_inst_per_link",
                                  "profiles/k_sweep_16x16x16x8_n24_full.md")
    if per_link is None or N != 24:
        return None
    tflops = per_link * 2.0 * 4 * V / (kernel_ms * 1e-3) / 1e12
    return {"achieved": tflops, "frac": tflops / peak, "unit": "TFLOP/s",
            "source": "DFMA thread instructions per link: ncu smsp__sass_thread_inst_executed_"
                      "op_dfma_pred_on.sum of one launch at 16x16x16x8 x 24 orders "
                      "(profiles/k_sweep_16x16x16x8_n24_full.md)"}


def host_cpu() -> dict:
    """The host's CPU model and logical core count (/proc/cpuinfo)."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "nproc": os.cpu_count()}


def cpu_reference_sample(N: int, L_sample, sweeps: int, warmup: int = 1,
                         threads_cap: int | None = None):
    """Time the reference's own code (oracle/_ref) on a bounded sample: the
    same plain Jacobi sweep the GPU arm times (gauge_wilson, Umu = Fmu,
    twist_boundary; no gauge fixing), twisted y,z, with the largest OpenMP
    grid the sample and the host allow.  `warmup` untimed sweeps, then
    `sweeps` timed ones in the same process.  Returns (seconds of each timed
    sweep, threads, kind, binary)."""
    from oracle import oracle as O
    ncpu = os.cpu_count() or 1
    if threads_cap:
        ncpu = min(ncpu, threads_cap)
    grids = [(1, 1, 1), (2, 1, 1), (2, 2, 1), (2, 2, 2), (4, 2, 2), (4, 4, 2), (4, 4, 4)]
    best = (1, 1, 1)
    for gr in grids:
        n = gr[0] * gr[1] * gr[2]
        if n <= ncpu and all(L_sample[d + 1] // gr[d] >= 2 for d in range(3)):
            best = gr
    binary = O.ref_binary(N, "tw", "local", best)
    if not os.path.exists(binary):
        try:
            binary = O.build_reference(N, "tw", "local", best)
        except Exception:
            binary = None
    if binary and os.path.exists(binary):
        with tempfile.TemporaryDirectory() as d:
            r = O.run_reference(binary, L_sample, warmup + sweeps, 0.005, 0.0, 1, d, noise=False,
                                timing=True, sweep_only=True)
        return r["step_seconds"][warmup:], best[0] * best[1] * best[2], "reference", binary
    # the reference binary cannot be built here: time the oracle port
    o = O.Oracle(L_sample, N, twist_mask=6)
    rng = O.Rand55(1)
    per = []
    for s in range(warmup + sweeps):
        nz = rng.gauss(o.V * 32)
        t0 = time.perf_counter()
        o.sweep(0.005, nz)
        if s >= warmup:
            per.append(time.perf_counter() - t0)
    return per, 1, "port", "oracle/liboracle.so"


# The CPU sample of the benchmark workload: the same 24-order twisted sweep on
# 16^4 (1/16 of the 32^4 volume; the cost is exactly linear in V at fixed N).
CPU_SAMPLE_L = (16, 16, 16, 16)


def cpu_baseline_line(N: int, V: int, sweeps: int, warmup: int) -> dict:
    """cpu_baseline of the workload: median, min and max over `sweeps` timed
    16^4 sweeps (after `warmup`), scaled by V to the full lattice."""
    per, threads, kind, _b = cpu_reference_sample(N, CPU_SAMPLE_L, sweeps, warmup)
    Vs = 1
    for x in CPU_SAMPLE_L:
        Vs *= x
    scale = V / Vs
    med = statistics.median(per)
    return {"value": 1.0 / (med * scale), "unit": "sweeps/s", "cores": threads, "kind": kind,
            "min": 1.0 / (max(per) * scale), "max": 1.0 / (min(per) * scale),
            "sample": "%d sweeps of 16^4 x %d orders (twisted y,z; gauge_wilson + Umu = Fmu + "
                      "twist_boundary, the GPU arm's timed work) after %d untimed, median "
                      "scaled by V to 32^4" % (len(per), N, warmup),
            "seconds_per_sample_sweep": per}


def run_reference_arm(args, world, rank):
    L = tuple(args.L)
    V = 1
    for x in L:
        V *= x
    if rank != 0:
        return
    sweeps = max(3, min(args.steps, 8))
    cpu = cpu_baseline_line(args.N, V, sweeps, min(args.warmup, 1))
    value = cpu["value"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "sweeps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (cold start)",
        "config": {"workload": "sweep_32^4_N24_twisted_yz", "L": list(L), "N": args.N,
                   "dt": 0.005, "bc": "twisted y,z", "update": "Jacobi",
                   "gauge_fixing": "none in the timed sweep"},
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": "sweeps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "host": host_cpu(),
    }
    print(json.dumps(line), flush=True)


def eng_grid(L):
    """The engine's default thread grid: blocks of 2 sites along even extents."""
    return tuple(l // 2 if l % 2 == 0 else 1 for l in L)


def e2e_leg(args, eng, lib, _lib, P, N, V, world, field_bytes):
    """Upload from pinned host memory, K x (sweep + observables read-back),
    download -- all through the C ABI, wall-clocked on the host."""
    import numpy as np
    import torch

    from prlgt2020_b200.replicas import max_over_ranks, whole_job_rate
    host = torch.empty((V * 4 * P.series_len(N),), dtype=torch.float64, pin_memory=True)
    eng.cold_start()
    obs_p = np.zeros((N + 1, 2))
    obs_n = np.zeros(N)
    obs_t = np.zeros((4, N, 2))
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    host_ptr = host.data_ptr()
    h = eng._h
    barrier(world)
    t0 = time.perf_counter()
    _lib.check(lib.nspt_download_links(h, ctypes.c_void_p(host_ptr), N), "download")
    t1 = time.perf_counter()
    e2e_steps = args.steps
    _lib.check(lib.nspt_upload_links(h, ctypes.c_void_p(host_ptr), N), "upload")
    for _ in range(e2e_steps):
        _lib.check(lib.nspt_step(h, args.dt, 1, 0), "step")
        _lib.check(lib.nspt_observables(h, dp(obs_p), dp(obs_n), dp(obs_t)), "observables")
    _lib.check(lib.nspt_download_links(h, ctypes.c_void_p(host_ptr), N), "download")
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    e2e_value = whole_job_rate(e2e_steps, world, max_over_ranks(t2 - t1))
    obs_bytes = obs_p.nbytes + obs_n.nbytes + obs_t.nbytes

    return {"value": e2e_value, "unit": "sweeps/s",
            "h2d_bytes_per_step": field_bytes / e2e_steps,
            "d2h_bytes_per_step": field_bytes / e2e_steps + obs_bytes,
            "note": "upload + %d x (sweep + observables read-back) + download" % e2e_steps}


def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    import prlgt2020_b200 as P
    from prlgt2020_b200 import _lib
    from prlgt2020_b200.replicas import max_over_ranks, replica_seed, whole_job_rate

    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device")
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    L = tuple(args.L)
    N = args.N
    V = int(np.prod(L))
    lib = _lib.load()
    peak = P.fp64_peak_tflops()

    # local gauge fixing (the reference's default with twisted boundaries) is
    # enabled for the secondary "with_gf" figure; the headline sweeps skip it
    eng = P.NsptEngine(L, N, twist="yz", local_gf=True, alpha=GF_ALPHA, update=args.update)
    eng.seed(replica_seed(1000, rank), 0)
    eng.cold_start()

    # warm-up sweeps (also move the field away from the cold start)
    eng.NsptEvolve(args.dt, args.warmup, 0)
    barrier(world)
    with ClockSampler(local) as clk:
        eng.NsptEvolve(args.dt, args.steps, 0)
        ms = eng.last_step_ms()
        kernel_ms = eng.last_kernel_ms()
    barrier(world)
    clocks = clk.summary()
    ms_max = max_over_ranks(ms)
    ms_step = ms_max / args.steps
    value = whole_job_rate(args.steps, world, ms_max * 1e-3)

    # roofline of the dominant kernel (the sweep): canonical flops / the
    # average duration of one sweep-kernel launch (CUDA events on its stream)
    flops = canonical_flops_per_link(N) * 4 * V
    kernel_ms = max_over_ranks(kernel_ms)
    achieved = flops / (kernel_ms * 1e-3) / 1e12

    # the workload's full step: local gauge fixing every 10 sweeps
    if args.no_gf:
        with_gf = None
    else:
        barrier(world)
        eng.NsptEvolve(args.dt, 10, 10)
        gf_ms = max_over_ranks(eng.last_step_ms())
        eng.stochastic_gauge_fixing()
        pass_ms = max_over_ranks(eng.last_step_ms())
        with_gf = {"value": whole_job_rate(10, world, gf_ms * 1e-3), "unit": "sweeps/s",
                   "gf_every": 10, "gf": "local stochastic (nspt.cc:660-862), finest thread grid",
                   "alpha": GF_ALPHA, "ms_per_10_steps": gf_ms, "gf_pass_ms": pass_ms}

    # end to end through the C ABI with the configuration on the host
    field_bytes = V * 4 * P.series_len(N) * 8
    if args.no_e2e:
        e2e = None
    else:
        e2e = e2e_leg(args, eng, lib, _lib, P, N, V, world, field_bytes)
    cpu = None
    if rank == 0 and not args.no_cpu:
        cpu = cpu_baseline_line(N, V, 3, 1)
        per1, _t1, kind1, _b1 = cpu_reference_sample(N, (4, 4, 4, 4), 1, 0, threads_cap=1)
        cpu["single_thread"] = {"value": 1.0 / (per1[0] * V / 4 ** 4), "unit": "sweeps/s",
                                "cores": 1, "kind": kind1,
                                "sample": "1 sweep of 4^4 x %d orders, scaled by V to 32^4" % N}
        cpu["host"] = host_cpu()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "sweeps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (cold start, device Philox noise)",
            "config": {"workload": "sweep_32^4_N24_twisted_yz", "L": list(L), "N": N,
                       "dt": args.dt, "bc": "twisted y,z",
                       "update": "Jacobi" if args.update == "jacobi" else
                                 "on the fly, thread grid %s" % (list(eng_grid(L)),),
                       "gauge_fixing": "none in the timed sweep",
                       "l2": "inputs larger than L2 (field %.1f GB)" % (field_bytes / 1e9),
                       "parallelism": "replicas" if world > 1 else "single"},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": read_profile_traffic(),
                         "traffic_source": "profiles/sweep_32x4_n24_traffic.txt: ncu dram__bytes_read.sum "
                                           "+ dram__bytes_write.sum of one k_sweep launch at 16^4 x 24, "
                                           "scaled x16 (links) to 32^4; not measured in this run",
                         "kernel": "k_sweep", "kernel_ms": kernel_ms,
                         "peak_source": "FP64 FMA microbenchmark on this GPU "
                                        "(nspt_measure_fp64_peak); MEASURED_PEAKS.json has no FP64 entry",
                         "flops_per_sweep": flops,
                         "executed": executed_fraction(N, V, kernel_ms, peak),
                         "algorithmic_bytes_per_sweep": algorithmic_bytes_per_sweep(V, N),
                         "hbm_gbs_equiv": algorithmic_bytes_per_sweep(V, N) / (ms_step * 1e-3) / 1e9},
            "clocks": clocks,
            "e2e": e2e,
            "with_gf": with_gf,
            # per sweep: k_sweep, three k_rowsum reductions, k_inc (the
            # Philox step counter) -- the launch list in profiles/
            "gpu_launches": 5 * args.steps,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def run_c2(args, world, rank, local):
    """16^4 x 20 orders, periodic, every step: sweep (with the per-link log
    the zero modes need), zero-mode subtraction, FA gauge fixing.  Each pass
    is timed on the device and set against its own roofline: canonical
    FP64 work for the series passes (the per-link log is in the sweep, one
    exp per link in the zero modes, a log, 1/4 exp and 2 products per link
    plus the FFTs in FA), HBM bytes for the FFT-dominated FA pass."""
    import numpy as np
    import torch

    import prlgt2020_b200 as P
    from prlgt2020_b200.replicas import max_over_ranks, replica_seed, whole_job_rate
    torch.cuda.set_device(local)
    # FA with alpha > 0: its step multiplies by -alpha/p^2 (nspt.cc:888-892); the
    # negative alpha of the reference's Quench.cfg makes FA grow exponentially
    L, N, alpha, dt = (16, 16, 16, 16), 20, 0.05, 0.01
    V = int(np.prod(L))
    peak = P.fp64_peak_tflops()
    eng = P.NsptEngine(L, N, zero_modes=True, fa=True, alpha=alpha)
    eng.seed(replica_seed(2000, rank), 0)
    eng.NsptEvolve(dt, args.warmup, 1)
    sweep = zm = fa = kern = 0.0
    for _ in range(args.steps):
        eng.gauge_wilson(dt)
        sweep += eng.last_step_ms()
        kern += eng.last_kernel_ms()
        eng.zero_modes_subtraction()
        zm += eng.last_step_ms()
        eng.FAstochastic_gauge_fixing(alpha)
        fa += eng.last_step_ms()
    eng.NsptEvolve(dt, args.steps, 1)
    step_ms = max_over_ranks(eng.last_step_ms()) / args.steps
    K = args.steps
    sweep, zm, fa, kern = (max_over_ranks(x) / K for x in (sweep, zm, fa, kern))
    Pn = N * (N - 1) // 2
    E = (N - 1) * N * (N + 1) // 6
    f_sweep = (14 * Pn + 2 * E) * 216.0 * 4 * V          # + the per-link log
    f_zm = E * 216.0 * 4 * V
    f_fa = (E + 0.25 * E + 2 * Pn) * 216.0 * 4 * V
    fft_flops = 2 * (9 * N + 1) * 5 * V * np.log2(V)
    fft_bytes = 2 * 4 * (9 * N + 1) * 16 * V              # 2 FFTs x 4 axis passes, read + write
    if rank == 0:
        tf = lambda f, ms: f / (ms * 1e-3) / 1e12
        line = {
            "metric": "Langevin steps/s at 16^4 x 20 orders (FP64, ZM + FA every step)",
            "value": whole_job_rate(1, world, step_ms * 1e-3), "unit": "steps/s",
            "n_gpus": world, "steps": K, "warmup": args.warmup, "ms_per_step": step_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (cold start + warm-up sweeps, device Philox noise)",
            "config": {"workload": "c2_16^4_N20_zm_fa", "L": list(L), "N": N, "dt": dt,
                       "alpha": alpha, "bc": "periodic"},
            "passes": {
                "sweep": {"ms": sweep, "kernel_ms": kern, "tflops": tf(f_sweep, kern),
                          "frac_fp64": tf(f_sweep, kern) / peak},
                "zero_modes": {"ms": zm, "tflops": tf(f_zm, zm), "frac_fp64": tf(f_zm, zm) / peak},
                "fa_gauge_fixing": {"ms": fa, "tflops": tf(f_fa + fft_flops, fa),
                                    "frac_fp64": tf(f_fa + fft_flops, fa) / peak,
                                    "fft_hbm_gbs_equiv": fft_bytes / (fa * 1e-3) / 1e9},
            },
            "fp64_peak_tflops": peak,
        }
        print(json.dumps(line), flush=True)
    eng.close()


def dt_extrapolation(rep_means, L, dts, orders=(2,)):
    """dt -> 0 of the plaquette coefficients: rep_means[r, k] is replica r's
    time-averaged order-k plaquette; replicas are grouped by volume and dt,
    and per volume P_k(dt) = P0 + c dt is fitted by weighted least squares
    (weights 1 / standard error^2 of each dt's replica mean)."""
    import numpy as np
    out = {}
    vols = sorted(set(tuple(l) for l in L))
    for vol in vols:
        key = "x".join(str(v) for v in vol)
        res = {}
        for k in orders:
            xs, ys, es = [], [], []
            for dt in sorted(set(dts)):
                idx = [r for r in range(len(L)) if tuple(L[r]) == vol and dts[r] == dt]
                v = rep_means[idx, k]
                xs.append(dt)
                ys.append(float(v.mean()))
                es.append(float(v.std(ddof=1) / np.sqrt(len(v))) if len(v) > 1 else float("nan"))
            x, y, e = np.array(xs), np.array(ys), np.array(es)
            w = 1.0 / np.maximum(e, 1e-300) ** 2
            A = np.stack([np.ones_like(x), x], axis=1)
            cov = np.linalg.inv(A.T @ (A * w[:, None]))
            p0, c = cov @ (A.T @ (w * y))
            chi2 = float(np.sum(w * (y - (p0 + c * x)) ** 2))
            res["order_%d" % k] = {"P0": float(p0), "P0_err": float(np.sqrt(cov[0, 0])),
                                   "slope": float(c), "chi2": chi2, "dof": len(x) - 2,
                                   "per_dt": {str(a): [b, d] for a, b, d in zip(xs, ys, es)}}
        out["L=" + key] = res
    return out


def run_c4(args, world, rank, local):
    """64 independent replicas, 12 orders, periodic, zero modes + FA gauge
    fixing every step: replica r has L = {6,8,10}[r mod 3]^4, dt =
    {0.005,0.01,0.02}[(r/3) mod 3], seed = 3000 + r.  Batched: all replicas
    in one CUDA graph per 2 steps (nspt_batch_step), sweep shape picked by
    the autotuner.  Plain: the same replicas advanced one after the other
    with nspt_step, as one process per lattice would.  The unit is replica
    steps per second; the plaquette series are averaged per dt for the
    dt -> 0 extrapolation."""
    import numpy as np
    import torch

    import prlgt2020_b200 as P
    from prlgt2020_b200.replicas import max_over_ranks, replica_seed, whole_job_rate
    torch.cuda.set_device(local)
    nrep, N, alpha = 64, 12, 0.05  # FA damps for alpha > 0 (nspt.cc:888-892)
    Ls = [(v,) * 4 for v in (6, 8, 10) for _ in range(1)]
    L = [Ls[r % 3] for r in range(nrep)]
    dts = [(0.005, 0.01, 0.02)[(r // 3) % 3] for r in range(nrep)]
    seeds = [replica_seed(3000 + r, rank) for r in range(nrep)]
    K = max(2, args.steps - args.steps % 2)
    kw = dict(zero_modes=True, fa=True, alpha=alpha)
    # plain: one replica after another, each its own launches and syncs
    plain = [P.NsptEngine(l, N, **kw) for l in L]
    for e, sd, dt in zip(plain, seeds, dts):
        e.seed(sd, 0)
        e.NsptEvolve(dt, args.warmup, 1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for e, dt in zip(plain, dts):
        e.NsptEvolve(dt, K, 1)
    torch.cuda.synchronize()
    plain_s = max_over_ranks(time.perf_counter() - t0)
    for e in plain:
        e.close()
    # batched
    b = P.NsptBatch(L, N, dts, seeds, **kw)
    warps, shape_mo, tune_ms = b.tune_shape(1)
    b.step(max(2, args.warmup - args.warmup % 2), 1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b.step(K, 1)
    torch.cuda.synchronize()
    batch_s = max_over_ranks(time.perf_counter() - t0)
    batch_dev_ms = max_over_ranks(b.last_step_ms())
    b.close()
    # dt -> 0: a fresh batch, thermalised, then the plaquette series of every
    # replica averaged over the measured steps (read every 2 steps)
    b = P.NsptBatch(L, N, dts, seeds, **kw)
    b.tune_shape(1)
    therm, meas = args.c4_therm - args.c4_therm % 2, max(2, args.c4_meas - args.c4_meas % 2)
    t_phys = time.perf_counter()
    if therm:
        b.step(therm, 1)
    acc = np.zeros((nrep, N + 1))
    for _ in range(meas // 2):
        b.step(2, 1)
        acc += b.plaquettes()[:, :, 0]
    t_phys = time.perf_counter() - t_phys
    b.close()
    rep_means = acc / (meas // 2)
    Pn = N * (N - 1) // 2
    E = (N - 1) * N * (N + 1) // 6
    links = sum(4 * int(np.prod(l)) for l in L)
    flops = (14 * Pn + 2 * E + E + 1.25 * E + 2 * Pn) * 216.0 * links * K
    peak = P.fp64_peak_tflops()
    if rank == 0:
        series = {}
        for dt in (0.005, 0.01, 0.02):
            idx = [r for r in range(nrep) if dts[r] == dt]
            series[str(dt)] = rep_means[idx].mean(axis=0).tolist()
        extrap = dt_extrapolation(rep_means, L, dts, orders=(2, 4))
        extrap["how"] = ("per replica the plaquette series averaged over %d measured steps (every "
                         "2nd) after %d thermalisation steps; per (L, dt) the mean over replicas "
                         "and its standard error; per L a weighted least-squares fit "
                         "P(dt) = P0 + c dt (the Euler update's O(dt) error), P0 +- its error"
                         % (meas, therm))
        extrap["seconds"] = t_phys
        line = {
            "metric": "replica Langevin steps/s, 64 replicas of 6^4/8^4/10^4 x 12 orders "
                      "(FP64, ZM + FA every step)",
            "value": whole_job_rate(nrep * K, world, batch_s), "unit": "replica steps/s",
            "n_gpus": world, "steps": K, "warmup": args.warmup,
            "ms_per_step": batch_s * 1e3 / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (cold start + warm-up, device Philox noise per replica)",
            "config": {"workload": "c4_batch_64x{6,8,10}^4_N12", "nrep": nrep, "N": N,
                       "dt": [0.005, 0.01, 0.02], "alpha": alpha, "gf_every": 1},
            "plain": {"value": whole_job_rate(nrep * K, world, plain_s), "unit": "replica steps/s",
                      "how": "replicas one after another, nspt_step each"},
            "batched_over_plain": plain_s / batch_s,
            "batched_device_ms": batch_dev_ms,
            "tuned": {"warps_per_cta": warps, "orders_per_lane": shape_mo,
                      "run_length": shape_mo // 2,
                      "ms_per_2_steps": {"orders_per_lane_8": tune_ms[0].tolist(),
                                         "orders_per_lane_4": tune_ms[1].tolist()}},
            "roofline": {"bound": "fp64", "achieved": flops / batch_s / 1e12, "peak": peak,
                         "unit": "TFLOP/s", "frac": flops / batch_s / 1e12 / peak},
            "plaquette_per_dt": series,
            "dt_to_0": extrap,
        }
        print(json.dumps(line), flush=True)


def run_c5(args, world, rank, local):
    """Float-float Cauchy products against the plain FP64 path, periodic,
    zero modes + FA gauge fixing every step, same seed on both.  FA runs
    with alpha = +0.05: the reference's FA step multiplies by -alpha/p^2
    (nspt.cc:888-892), and with the negative alpha of its Quench.cfg (meant for
    the local gauge fixing) the reference's own FA path grows exponentially
    in Langevin time at every order.
    Speed at 24^4 x 40 orders: the sweep kernel and the whole step, each
    engine alone.  Accuracy at 8^4 x 40 (so that 1000 steps take about a
    minute): from a common field (20 FP64 steps from a cold start) the
    float-float and the FP64 engine run on with the same noise, and the
    per-order relative difference max|ff - fp64| / max|fp64| over each
    order's coefficients is taken after 1, 100 and 1000 steps.  Beside it,
    the same figure for a second FP64 run whose dt is larger by one part in
    2^52: the growth of a rounding-level difference that FP64 itself
    cannot avoid, i.e. the accuracy an FP64 run has at that order."""
    import numpy as np
    import torch

    import prlgt2020_b200 as P
    from prlgt2020_b200.replicas import max_over_ranks, replica_seed
    torch.cuda.set_device(local)
    N, alpha, dt = 40, 0.05, 0.01
    kw = dict(zero_modes=True, fa=True, alpha=alpha)
    seed = replica_seed(5000, rank)
    K = args.steps
    Pn = N * (N - 1) // 2
    E = (N - 1) * N * (N + 1) // 6
    speed = {}
    L = (24, 24, 24, 24)
    V = int(np.prod(L))
    for prec in ("fp64", "ff"):
        eng = P.NsptEngine(L, N, precision=prec, **kw)
        eng.seed(seed, 0)
        eng.NsptEvolve(dt, args.warmup, 1)
        kern = 0.0
        for _ in range(K):
            eng.gauge_wilson(dt)
            kern += eng.last_kernel_ms()
            eng.zero_modes_subtraction()
            eng.FAstochastic_gauge_fixing(alpha)
        eng.NsptEvolve(dt, K, 1)
        step_ms = max_over_ranks(eng.last_step_ms()) / K
        kern = max_over_ranks(kern) / K
        f = (14 * Pn + 2 * E) * 216.0 * 4 * V
        speed[prec] = {"step_ms": step_ms, "sweep_kernel_ms": kern,
                       "sweep_canonical_tflops": f / (kern * 1e-3) / 1e12}
        if prec == "ff":
            speed[prec]["scale_exponent"] = eng.ff_scale()
        eng.close()
    # accuracy: float-float vs FP64 from a common field, same noise
    La, warm = (8, 8, 8, 8), 20
    base = P.NsptEngine(La, N, **kw)
    base.seed(seed, 0)
    base.NsptEvolve(dt, warm, 1)
    start = base.download()
    base.close()
    ff = P.NsptEngine(La, N, precision="ff", **kw)
    ref = P.NsptEngine(La, N, **kw)
    pert = P.NsptEngine(La, N, **kw)
    for e in (ff, ref, pert):
        e.upload(start)
        e.seed(seed, warm)
    dt_pert = dt * (1.0 + 2.0 ** -52)

    def rel_per_order(a, b):
        a = a.reshape(-1, 2 + 18 * N)
        b = b.reshape(-1, 2 + 18 * N)
        out = []
        for k in range(1, N + 1):
            sl = slice(2 + 18 * (k - 1), 2 + 18 * k)
            den = np.abs(b[:, sl]).max()
            out.append(float(np.abs(a[:, sl] - b[:, sl]).max() / den))
        return out

    err, done = {}, 0
    for m in (1, 100, 1000):
        ff.NsptEvolve(dt, m - done, 1)
        ref.NsptEvolve(dt, m - done, 1)
        pert.NsptEvolve(dt_pert, m - done, 1)
        done = m
        r = ref.download()
        e_ff = rel_per_order(ff.download(), r)
        e_64 = rel_per_order(pert.download(), r)
        err[str(m)] = {"ff_vs_fp64": e_ff, "fp64_ulp_dt_vs_fp64": e_64,
                       "ff_max": max(e_ff), "fp64_ulp_dt_max": max(e_64),
                       "finite": bool(np.isfinite(r).all())}
    for e in (ff, ref, pert):
        e.close()
    if rank == 0:
        line = {
            "metric": "Langevin steps/s at 24^4 x 40 orders, float-float Cauchy products "
                      "(ZM + FA every step)",
            "value": 1e3 / speed["ff"]["step_ms"] * world, "unit": "steps/s",
            "n_gpus": world, "steps": K, "warmup": args.warmup,
            "ms_per_step": speed["ff"]["step_ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32x2 products, f64 elsewhere",
            "data": "synthetic (cold start + warm-up, device Philox noise, same seed both paths)",
            "config": {"workload": "c5_24^4_N40_ff_vs_fp64", "L": list(L), "N": N, "dt": dt,
                       "alpha": alpha, "accuracy_lattice": list(La),
                       "accuracy_start": "%d FP64 steps from a cold start" % warm},
            "fp64": speed["fp64"], "ff": speed["ff"],
            "ff_over_fp64_speed": speed["fp64"]["step_ms"] / speed["ff"]["step_ms"],
            "ff_over_fp64_sweep_kernel": speed["fp64"]["sweep_kernel_ms"]
                                         / speed["ff"]["sweep_kernel_ms"],
            "per_order_rel_error_after_steps": err,
        }
        print(json.dumps(line), flush=True)


def run_imp(args, world, rank, local):
    """Improved action (tree-level Symanzik) sweep at 16^4 x 20, periodic,
    no zero modes or gauge fixing: the force kernel with the six 2x1
    rectangle staples per plane (staple2x1, QCDenvNODEpt_test.h:579-611).
    Canonical work per link, as the reference multiplies: 12 plaquette-staple
    products, 72 rectangle products (6 rectangles x 3 planes x 4), U W and
    U W2, exp, exp U: (87 P(N) + E(N)) x 216 flop."""
    import numpy as np
    import torch

    import prlgt2020_b200 as P
    from prlgt2020_b200.replicas import max_over_ranks, replica_seed, whole_job_rate
    torch.cuda.set_device(local)
    L, N, dt = (16, 16, 16, 16), 20, 0.01
    V = int(np.prod(L))
    peak = P.fp64_peak_tflops()
    eng = P.NsptEngine(L, N, action="tlsym")
    eng.seed(replica_seed(6000, rank), 0)
    eng.NsptEvolve(dt, args.warmup, 1)
    eng.NsptEvolve(dt, args.steps, 1)
    step_ms = max_over_ranks(eng.last_step_ms()) / args.steps
    kern = max_over_ranks(eng.last_kernel_ms())
    Pn = N * (N - 1) // 2
    E = (N - 1) * N * (N + 1) // 6
    flops = (87 * Pn + E) * 216.0 * 4 * V
    if rank == 0:
        ach = flops / (kern * 1e-3) / 1e12
        line = {
            "metric": "Langevin sweeps/s at 16^4 x 20 orders, tree-level Symanzik action (FP64)",
            "value": whole_job_rate(1, world, step_ms * 1e-3), "unit": "sweeps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (cold start + warm-up, device Philox noise)",
            "config": {"workload": "imp_16^4_N20_tlsym", "L": list(L), "N": N, "dt": dt,
                       "action": "tlsym", "bc": "periodic"},
            "roofline": {"bound": "fp64", "achieved": ach, "peak": peak, "unit": "TFLOP/s",
                         "frac": ach / peak, "kernel": "k_sweep_imp", "kernel_ms": kern,
                         "flops_per_sweep": flops},
        }
        print(json.dumps(line), flush=True)
    eng.close()


def run_loops(args, world, rank, local):
    """Wilson loops (ComputeLoops, nspt.cc:1148-1312) of a 16^4 x 20 periodic
    field: the 1x2, 2x2, 2x4 and 4x4 loops of every plane and site, traced
    per order.  Canonical work as the reference multiplies: per (plane,
    site) 28 path products and 6 closing products W += P Q^dag, 34 P(N) x
    216 flop; the engine replaces each closing product by a trace (a sixth
    of its flops)."""
    import numpy as np
    import torch

    import prlgt2020_b200 as P
    from prlgt2020_b200.replicas import max_over_ranks, replica_seed, whole_job_rate
    torch.cuda.set_device(local)
    L, N, dt = (16, 16, 16, 16), 20, 0.01
    V = int(np.prod(L))
    peak = P.fp64_peak_tflops()
    eng = P.NsptEngine(L, N, zero_modes=True)
    eng.seed(replica_seed(7000, rank), 0)
    eng.NsptEvolve(dt, 3, 1)
    for _ in range(args.warmup):
        eng.ComputeLoops()
    ms = 0.0
    for _ in range(args.steps):
        eng.ComputeLoops()
        ms += eng.last_step_ms()
    ms = max_over_ranks(ms) / args.steps
    Pn = N * (N - 1) // 2
    flops = 34 * Pn * 216.0 * 6 * V
    if rank == 0:
        ach = flops / (ms * 1e-3) / 1e12
        line = {
            "metric": "ComputeLoops calls/s at 16^4 x 20 orders (FP64)",
            "value": whole_job_rate(1, world, ms * 1e-3), "unit": "calls/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (cold start + 3 sweeps, device Philox noise)",
            "config": {"workload": "loops_16^4_N20", "L": list(L), "N": N, "bc": "periodic"},
            "roofline": {"bound": "fp64", "achieved": ach, "peak": peak, "unit": "TFLOP/s",
                         "frac": ach / peak, "kernel": "k_loops", "flops_per_call": flops},
        }
        print(json.dumps(line), flush=True)
    eng.close()


def run_qcfg(args, world, rank, local):
    """The reference's shipped Quench.cfg run: 12^4, PTORD 8, tau_g 0.005,
    alpha -0.05, periodic, Wilson action, zero-mode subtraction and local
    stochastic gauge fixing every step (NsptEvolve, nspt.cc:953-1039).  The
    reference's default build updates on the fly (UPDATE_ONTHEFLY,
    choices.h:61), so that is the line's value; the Jacobi update of the same
    run is reported beside it.  Steps/s of the whole step."""
    import numpy as np
    import torch

    import prlgt2020_b200 as P
    from prlgt2020_b200.replicas import max_over_ranks, replica_seed, whole_job_rate
    torch.cuda.set_device(local)
    L, N, dt, alpha = (12, 12, 12, 12), 8, 0.005, -0.05

    def timed(update):
        eng = P.NsptEngine(L, N, zero_modes=True, local_gf=True, alpha=alpha, update=update)
        eng.set_local_gf_form(args.lgf_form)
        eng.seed(replica_seed(8000, rank), 0)
        eng.NsptEvolve(dt, args.warmup, 1)
        eng.NsptEvolve(dt, args.steps, 1)
        ms = max_over_ranks(eng.last_step_ms()) / args.steps
        eng.close()
        return ms

    step_ms = timed("onthefly")
    jac_ms = timed("jacobi")
    if rank == 0:
        line = {
            "metric": "Langevin steps/s, the reference's Quench.cfg run (12^4 x 8 orders, ZM + "
                      "local gauge fixing every step, on-the-fly update)",
            "value": whole_job_rate(1, world, step_ms * 1e-3), "unit": "steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (cold start + warm-up, device Philox noise)",
            "config": {"workload": "qcfg_12^4_N8_zm_localgf", "L": list(L), "N": N, "dt": dt,
                       "alpha": alpha, "bc": "periodic", "gf_every": 1,
                       "local_gf_form": args.lgf_form, "update": "on the fly",
                       "thread_grid": list(eng_grid(L))},
            "jacobi": {"value": whole_job_rate(1, world, jac_ms * 1e-3), "unit": "steps/s",
                       "ms_per_step": jac_ms},
        }
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--L", type=int, nargs=4, default=[32, 32, 32, 32])
    ap.add_argument("--N", type=int, default=24)
    ap.add_argument("--dt", type=float, default=0.005)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    ap.add_argument("--no-gf", action="store_true", help="skip the gauge-fixing figure")
    ap.add_argument("--update", default="jacobi", choices=["jacobi", "onthefly"],
                    help="gauge_wilson update of the sweep workload: Jacobi, or the reference's "
                         "default in-place update in thread-grid order (qcfg reports both)")
    ap.add_argument("--lgf-form", default="auto", choices=["auto", "group", "team"],
                    help="local gauge fixing kernel of the qcfg workload")
    ap.add_argument("--c4-therm", type=int, default=600,
                    help="c4: thermalisation steps before the dt -> 0 measurement")
    ap.add_argument("--c4-meas", type=int, default=600,
                    help="c4: measured steps (plaquette read every 2nd) for dt -> 0")
    ap.add_argument("--workload", default="sweep", choices=["sweep", "c2", "c4", "c5", "imp", "loops", "qcfg"],
                    help="sweep: 32^4 x 24 twisted (the headline); c2: 16^4 x 20 periodic "
                         "with zero modes and FA gauge fixing every step, per pass; c4: 64 "
                         "replicas of 6^4..10^4 x 12, batched in one CUDA graph vs plain; "
                         "c5: 24^4 x 40 float-float products vs FP64, speed and per-order "
                         "error after 1/100/1000 steps; imp: 16^4 x 20 tree-level "
                         "Symanzik sweep; loops: Wilson loops of a 16^4 x 20 field; qcfg: the "
                         "reference's shipped Quench.cfg run, 12^4 x 8 with ZM and local GF")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        return
    if args.workload == "c2":
        run_c2(args, world, rank, local)
        return
    if args.workload == "c4":
        run_c4(args, world, rank, local)
        return
    if args.workload == "c5":
        run_c5(args, world, rank, local)
        return
    if args.workload == "imp":
        run_imp(args, world, rank, local)
        return
    if args.workload == "loops":
        run_loops(args, world, rank, local)
        return
    if args.workload == "qcfg":
        run_qcfg(args, world, rank, local)
        return
    run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
