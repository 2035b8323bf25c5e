"""Benchmark of the explicit Euler step on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K (2000)] [--warmup W (5; at least 32 are run)] [--impl ours|reference]
                    [--config 2|3|0|1|4]

Workload (default, --config 2): batching, 256 independent instances on one grid of two
species (electron, photon) of 32 log p bins x 8 u bins = 256 states each, sharing one gain
tensor 2 x 256 x 65,536 stored as BF16 hi+lo with per-row scales (134 MB, streamed every step,
larger than L2), loss, emission and flux as in the config recipe (dtb/synth.py); per-instance
f0 and dt. A step is one batched Euler step of all instances (the autotuned tcgen05 gain GEMM
and the epilogue kernel). --config 3: three species, 64 instances, 4.59 GB of G per step.
--config 1: the plain single instance (FP32 G 8.6 GB); --config 0: the FP64 N_s = 128 case
(L2-resident, launch-bound); --config 4: serving (Poisson request stream, p50/p99).

value: instance-steps/s over the timed steps, inputs resident in HBM, device-timed with CUDA
events on the library's stream (a captured graph replayed); N GPUs run independent batch
replicas (weak scaling) and the whole-job value is the sum over ranks (total instance-steps /
max time over ranks).
e2e: the same steps through the public API with host buffers: every step uploads the whole
batch's f (FP64) from pinned host memory, steps, and reads it back (dtb_batch_run_io, one
call and one wait per step).
roofline: the gain GEMM (dominant), algorithmic FLOPs = 3 MMAs x 2 x M x K x instances per
step (tensor-bound; config 3: operator bytes, HBM-bound), duration from CUDA events around
every GEMM launch over a second run of the same steps.
cpu_baseline / --impl reference: the FP64 oracle port timed on the host cores with OpenMP on
one instance for a few steps, scaled to instance-steps/s.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "diplodocustransport.jl_b200"))

METRIC = "steps/s & p99 latency, batched BF16-split vs plain FP64, at ≤1e-5 rel err"
GRAPH_WARMUP = 32  # two captured graphs of 16 steps


def _env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _profile_traffic(name: str):
    """dram bytes per launch recorded from an ncu capture in profiles/<name> (or None)."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        txt = open(path).read()
    except OSError:
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", txt)
    return float(m.group(1)) if m else None


def _smi_id(local: int) -> str:
    """nvidia-smi id of the torch device (UUID when torch exposes it, else the index)."""
    try:
        import torch
        u = str(torch.cuda.get_device_properties(local).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return str(local)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: str):
        self.gpu = gpu
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.p is not None:
            time.sleep(0.25)
            self.p.terminate()
            try:
                out, _ = self.p.communicate(timeout=5)
            except Exception:
                self.p.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            parts = [x.strip() for x in l.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_workload(config: int, device: str, host_sample_rows=None, grid=None):
    from dtb import synth
    if config == 1 and grid:  # same recipe on another grid, e.g. "32x16" (small profiling case)
        p, u = (int(x) for x in grid.split("x"))
        return synth.two_species(p, 1e-3, 1e3, u, seed=1, gain_on_device=True, device=device), "f32"
    if config == 1:
        if host_sample_rows:
            return synth.config1(seed=1, gain_on_device=False, gain_rows=host_sample_rows), "f32"
        return synth.config1(seed=1, gain_on_device=True, device=device), "f32"
    if config == 0:
        return synth.config0(seed=0), "f64"
    raise SystemExit(f"unknown --config {config}")


def cpu_sample(w, dtype: str, budget_s: float = 15.0):
    """Oracle port on the host cores: time a sample of gain rows (FP64) plus the O(N^2) rest,
    scale the rows to the full count; returns (steps/s, cores, sample description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle
    ps = w.ps
    ns_list = ps.species_sizes
    n_rows_total = sum(ns_list[g.out_sp] for g in w.binm.gains)
    off = ps.momentum_species_offset
    f0 = np.asarray(w.f0, dtype=np.float64)
    # rows of the first gain block as FP64 host arrays
    g0 = w.binm.gains[0]
    n1, n2 = ns_list[g0.in1_sp], ns_list[g0.in2_sp]
    row_bytes = n1 * n2 * 8
    n_sample = int(max(1, min(np.asarray(g0.G).shape[0] if not hasattr(g0.G, "is_cuda") else ns_list[g0.out_sp],
                              (2 << 30) // row_bytes)))
    G = g0.G
    if hasattr(G, "is_cuda"):
        Gs = G[:n_sample].double().cpu().numpy()
    else:
        Gs = np.ascontiguousarray(np.asarray(G)[:n_sample], dtype=np.float64)
    f1, f2 = f0[off[g0.in1_sp]:off[g0.in1_sp] + n1], f0[off[g0.in2_sp]:off[g0.in2_sp] + n2]
    oracle.gain_rows(Gs, 0, 1, f1, f2)  # warm
    t0 = time.perf_counter()
    reps = 0
    while True:
        oracle.gain_rows(Gs, 0, n_sample, f1, f2)
        reps += 1
        if time.perf_counter() - t0 > budget_s * 0.8 or reps >= 50:
            break
    t_rows = (time.perf_counter() - t0) / reps / n_sample
    # the rest of a step (flux, emission, loss, update) with the gain rows removed
    from dtb.structs import LossBlock  # noqa: F401
    ops = oracle.BlockedOperands(ns_list, ps.n_space, [], w.binm.losses, w.emim.blocks, w.fluxm.F_Flux,
                                 1.0 / np.asarray(w.fluxm.Ap_Flux), w.fluxm.Vol, w.inj)
    t1 = time.perf_counter()
    k = 0
    while time.perf_counter() - t1 < budget_s * 0.2 and k < 200:
        ops.step(f0, 1.0, 1)
        k += 1
    t_rest = (time.perf_counter() - t1) / k
    t_step = t_rows * n_rows_total + t_rest
    desc = (f"FP64 oracle (C, OpenMP): {n_sample} of {n_rows_total} gain rows x {reps} reps scaled to all rows, "
            f"plus {k} full steps without gain")
    return 1.0 / t_step, oracle.num_threads(), desc


def build_batched(config: int, device: str, host: bool = False):
    from dtb import synth
    if config == 2:
        return synth.config2(seed=2, gain_on_device=not host, device=device)
    if config == 3:
        return synth.config3(seed=3, batch=64, gain_on_device=not host, device=device)
    raise SystemExit(f"unknown batched config {config}")


def cpu_sample_batched(w, budget_s: float = 15.0):
    """FP64 oracle port of one instance on the host cores (OpenMP), a few steps; instance-steps/s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle
    gains = [type(g)(g.out_sp, g.in1_sp, g.in2_sp,
                     g.G.double().cpu().numpy() if hasattr(g.G, "is_cuda") else np.asarray(g.G, dtype=np.float64))
             for g in w.binm.gains]
    ops = oracle.BlockedOperands(w.ps.species_sizes, 1, gains, w.binm.losses, w.emim.blocks, w.fluxm.F_Flux,
                                 1.0 / np.asarray(w.fluxm.Ap_Flux), w.fluxm.Vol, w.inj)
    f = np.array(w.f0[0])
    ops.step(f, float(w.dt[0]), 1)
    t0 = time.perf_counter()
    k = 0
    while time.perf_counter() - t0 < budget_s and k < 200:
        f, _, _ = ops.step(f, float(w.dt[0]), 1)
        k += 1
    dt = (time.perf_counter() - t0) / k
    return 1.0 / dt, oracle.num_threads(), f"FP64 oracle (C, OpenMP), one instance, {k} full steps"


def run_reference(args):
    rank, local, world = _env_rank()
    if rank != 0:
        return 0
    if args.config in (2, 3):
        w = build_batched(args.config, "cpu", host=True)
        v, cores, desc = cpu_sample_batched(w, budget_s=20.0)
        value = v
        line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "instance-steps/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / value,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": _config_dict(args.config, w),
                "cpu_baseline": {"value": value, "unit": "instance-steps/s", "cores": cores, "kind": "port",
                                 "sample": desc},
                "e2e": {"value": value, "unit": "instance-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0
    # host-only workload: a sample of gain rows is all the timing needs
    w, dtype = build_workload(args.config, "cpu", host_sample_rows=256)
    v, cores, desc = cpu_sample(w, dtype, budget_s=20.0)
    value = v
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": _config_dict(args.config, w),
            "cpu_baseline": {"value": value, "unit": "steps/s", "cores": cores, "kind": "port", "sample": desc},
            "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def _has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def _config_dict(config: int, w):
    sizes = w.ps.species_sizes
    if config == 2:
        return {"workload": "batching (config 2): 256 independent instances, 2 species x 256 states "
                            "(32 log p x 8 u), shared G 2 x 256 x 65536 as BF16 hi+lo, per-instance f0 and dt",
                "species_states": sizes, "batch": 256, "precision": "BF16x3 gain GEMM, FP32 f, FP64 update",
                "l2": "G hi+lo 134 MB per step, larger than L2"}
    if config == 3:
        return {"workload": "mixed precision (config 3): 64 instances, e-, e+, gamma x 576 states "
                            "(48 log p x 12 u), 6 gain tensors 576 x 331776 as BF16 hi+lo, synchrotron-like emission",
                "species_states": sizes, "batch": 64, "precision": "BF16x3 gain GEMM, FP32 f, FP64 update",
                "l2": "G hi+lo 4.6 GB per step, larger than L2"}
    if config == 1 and sizes != [1024, 1024]:
        return {"workload": f"config-1 recipe on a smaller grid: 2 species x {sizes[0]} states, FP32",
                "species_states": sizes, "precision": "FP32"}
    if config == 1:
        return {"workload": "plain single instance (config 1): 2 species x 1024 states (64 log p x 16 u), "
                            "FP32 gain 2 x 1024 x 1048576, 2000-step run shape",
                "species_states": sizes, "precision": "FP32", "l2": "inputs larger than L2 (8.6 GB gain)"}
    return {"workload": "plain single instance (config 0): 2 species x 128 states (16 log p x 8 u), FP64",
            "species_states": sizes, "precision": "FP64",
            "l2": "operators (34 MB) fit in L2; no flush between steps (launch/L2-bound case)"}


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    from dtb import _lib
    from dtb.stepping import ForwardEulerStruct
    rank, local, world = _env_rank()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    w, dtype = build_workload(args.config, f"cuda:{local}", grid=args.grid)
    stream = torch.cuda.Stream()
    m = ForwardEulerStruct(w.ps, w.f0, w.inj, w.binm, w.emim, w.fluxm,
                           Precision=np.float32 if dtype == "f32" else np.float64, device=local,
                           stream=stream.cuda_stream)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_sample(w, dtype, budget_s=15.0)
    # the library holds its own copy of G
    w.binm.gains = [type(g)(g.out_sp, g.in1_sp, g.in2_sp, None) for g in w.binm.gains]
    torch.cuda.empty_cache()
    L = m.L
    # warm-up: at least two graphs' worth of steps, so the 16-step graph is captured and
    # instantiated before the timed region
    K, W = args.steps, max(args.warmup, GRAPH_WARMUP)
    scales = np.ones(K)
    m.run(np.ones(W))
    lps = _lib.ctypes.c_int32()
    L.dtb_launches_per_step(m.ctx, _lib.ctypes.byref(lps))
    # ---- timed region: device resident, gain kernel timed per launch
    use_profile = args.config == 1
    L.dtb_set_profiling(m.ctx, 1 if use_profile else 0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(_smi_id(local)) as cs:
        e0.record(stream)
        m.run(scales)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    avg_ms = _lib.ctypes.c_double()
    bpl = _lib.ctypes.c_double()
    L.dtb_gain_kernel_stats(m.ctx, _lib.ctypes.byref(avg_ms), _lib.ctypes.byref(bpl))
    L.dtb_set_profiling(m.ctx, 0)
    # ---- e2e: host buffers through the public API every step
    n = w.ps.n_state
    f_host = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    f_host[:] = m.f
    K2 = K
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_wall0 = time.perf_counter()
    e2.record(stream)
    for _ in range(K2):
        m.f = f_host
        m(0.0, 1e30, m.dt0, 0)
        f_host[:] = m.f
    e3.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e2.elapsed_time(e3)
    t_wall = time.perf_counter() - t_wall0
    ms_e2e = max(ms_e2e, 0.0)
    if world > 1:
        t = torch.tensor([ms, ms_e2e], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_e2e = float(t[0]), float(t[1])
    value = world * K / (ms / 1e3)
    e2e_value = world * K2 / (ms_e2e / 1e3)
    esz = 4 if dtype == "f32" else 8
    peak, peak_kind = _peaks()
    achieved = bpl.value / (avg_ms.value / 1e3) / 1e9 if avg_ms.value > 0 else None
    traffic = _profile_traffic("gain_stream_f32_config1.md") if args.config == 1 else None
    line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": dtype, "data": "synthetic (seeded; no collision data files)",
            "config": dict(_config_dict(args.config, w), parallelism=f"replicas x{world}"),
            "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": n * esz,
                    "d2h_bytes_per_step": n * esz, "wall_s": t_wall},
            "gpu_launches": int(lps.value) * K,
            "roofline": {"bound": "hbm", "kernel": "gain_stream", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None,
                         "traffic": traffic, "algorithmic_bytes_per_launch": bpl.value,
                         "avg_launch_ms": avg_ms.value},
            "clocks": cs.summary()}
    if cpu is not None:
        v, cores, desc = cpu
        line["cpu_baseline"] = {"value": v, "unit": "steps/s", "cores": cores, "kind": "port", "sample": desc}
    m.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_batched(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from dtb.batch import BatchedEuler, set_tune_cache
    from dtb.stepping import ForwardEulerStruct
    rank, local, world = _env_rank()
    torch.cuda.set_device(local)
    if args.tune_cache:
        set_tune_cache(args.tune_cache)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    dev = f"cuda:{local}"
    w = build_batched(args.config, dev)
    B = w.f0.shape[0]
    n = w.ps.n_state
    # warm-up: at least two graphs' worth of steps (the 16-step graph is captured and instantiated
    # before the timed region)
    K, W = args.steps, max(args.warmup, GRAPH_WARMUP)
    stream = torch.cuda.Stream()
    m = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B, device=local, stream=stream.cuda_stream)
    for i in range(B):
        m.admit(i, w.f0[i], float(w.dt[i]), 1 << 40)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_sample_batched(w, budget_s=15.0)
    # accuracy against the FP64 oracle: W warm-up steps of two instances
    acc = None
    if rank == 0 and not args.no_check:
        import oracle
        gains = [type(g)(g.out_sp, g.in1_sp, g.in2_sp, g.G.double().cpu().numpy()) for g in w.binm.gains]
        ops = oracle.BlockedOperands(w.ps.species_sizes, 1, gains, w.binm.losses, w.emim.blocks, w.fluxm.F_Flux,
                                     1.0 / np.asarray(w.fluxm.Ap_Flux), w.fluxm.Vol, w.inj)
    # plain FP64 path on the same grid (one instance), for the batched-vs-plain comparison
    gains64 = [type(g)(g.out_sp, g.in1_sp, g.in2_sp, g.G.double()) for g in w.binm.gains]
    from dtb.structs import BinaryMatrices
    binm64 = BinaryMatrices(gains=gains64, losses=w.binm.losses)
    plain = ForwardEulerStruct(w.ps, w.f0[0], w.inj, binm64, w.emim, w.fluxm, Precision=np.float64, device=local,
                               stream=stream.cuda_stream)
    del gains64, binm64
    w.binm.gains = [type(g)(g.out_sp, g.in1_sp, g.in2_sp, None) for g in w.binm.gains]
    torch.cuda.empty_cache()
    m.run(W)  # warm-up (captures and instantiates the graphs)
    if rank == 0 and not args.no_check:
        errs = []
        for i in (0, B - 1):
            f = np.array(w.f0[i])
            for _ in range(W):
                f, _, _ = ops.step(f, float(w.dt[i]), 0)
            g = m.get_f(i)
            errs.append(float(np.max(np.abs(g - f)) / np.max(np.abs(f))))
        acc = {"rel_linf_vs_fp64_oracle": max(errs), "steps": W, "instances": [0, B - 1]}
        del ops
    # ---- timed region: graph replay, device resident
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(_smi_id(local)) as cs:
        e0.record(stream)
        m.run(K)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    # ---- the same K steps with CUDA events around every gain-GEMM launch (direct launches)
    m.set_profiling(True)
    e4, e5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e4.record(stream)
    m.run(K)
    e5.record(stream)
    torch.cuda.synchronize()
    ms_prof = e4.elapsed_time(e5)
    st = m.gemm_stats()
    plans = []
    while (pl := m.gemm_plan(len(plans))) is not None:
        plans.append(pl)
    m.set_profiling(False)
    # ---- e2e: the whole batch state from pinned host memory in and out every step
    Fh = torch.empty((B, n), dtype=torch.float64).pin_memory().numpy()
    m.get_f_all(Fh)
    K2 = max(1, K // 4)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(K2):
        m.run_io(Fh, 1, Fh)  # upload, one batched step, download: one call, one wait
    e3.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e2.elapsed_time(e3)
    # ---- plain FP64 single instance on the same grid
    K3 = max(16, K // 4)
    plain.run(np.ones(4))
    e6, e7 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e6.record(stream)
    plain.run(np.full(K3, float(w.dt[0])))
    e7.record(stream)
    torch.cuda.synchronize()
    ms_plain = e6.elapsed_time(e7)
    plain.close()
    if world > 1:
        t = torch.tensor([ms, ms_e2e, ms_plain], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_e2e, ms_plain = float(t[0]), float(t[1]), float(t[2])
    value = world * B * K / (ms / 1e3)
    plain_sps = world * K3 / (ms_plain / 1e3)
    pj = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak = float(pj.get("bf16_tflops", 1590.0))
    peak_s = float(pj.get("bf16_tflops_sustained", 1400.0))
    achieved = st["flops_per_step"] / (st["avg_ms"] / 1e3) / 1e12 if st["avg_ms"] > 0 else None
    traffic = _profile_traffic(f"gain_gemm_config{args.config}.md")
    # 256-column tiles over an even number of 128-row m tiles run on SM pairs (cta_group::2)
    GEMM_LABEL = ("gain_gemm_pair (tcgen05.mma.cta_group::2, BF16 hi+lo x3)" if all(p["pair"] for p in plans)
                  else "gain_gemm (tcgen05, BF16 hi+lo x3)")
    # the GEMM's bound: the slower of its tensor time and its operator-streaming time
    hbm = float(pj.get("hbm_gbs", 6650.0))
    hbm_bound = st["bytes_per_step"] / (hbm * 1e9) > st["flops_per_step"] / (peak * 1e12)
    if hbm_bound:
        gbs = st["bytes_per_step"] / (st["avg_ms"] / 1e3) / 1e9 if st["avg_ms"] > 0 else None
        roof = {"bound": "hbm", "kernel": GEMM_LABEL, "achieved": gbs, "peak": hbm,
                "peak_kind": "measured" if pj else "fallback", "unit": "GB/s", "frac": gbs / hbm if gbs else None,
                "tensor_tflops": achieved}
    else:
        roof = {"bound": "tensor", "kernel": GEMM_LABEL, "achieved": achieved,
                "peak": peak, "peak_kind": "measured burst" if pj else "fallback", "unit": "TFLOP/s",
                "frac": achieved / peak if achieved else None,
                "frac_of_sustained": achieved / peak_s if achieved else None}
    roof.update({"gemm_plans": [dict(p, tuned_us=round(p["tuned_us"], 2)) for p in plans], "traffic": traffic, "algorithmic_flops_per_step": st["flops_per_step"],
                 "operator_bytes_per_step": st["bytes_per_step"], "avg_gemm_ms_per_step": st["avg_ms"],
                 "profiled_ms_per_step": ms_prof / K})
    line = {"metric": METRIC, "value": value, "unit": "instance-steps/s", "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16x3 (gain GEMM), f32 state, f64 update", "data": "synthetic (seeded; no collision data files)",
            "config": dict(_config_dict(args.config, w), parallelism=f"batch replicas x{world}"),
            "e2e": {"value": world * B * K2 / (ms_e2e / 1e3), "unit": "instance-steps/s",
                    "h2d_bytes_per_step": B * n * 8, "d2h_bytes_per_step": B * n * 8},
            "gpu_launches": int(st["launches_per_step"]) * K + (K + 15) // 16,  # + one step-counter advance per graph
            "roofline": roof,
            "plain_fp64": {"value": plain_sps, "unit": "steps/s", "workload": "same grid, one instance, FP64"},
            "speedup_vs_plain_fp64": value / plain_sps,
            "clocks": cs.summary()}
    if acc is not None:
        line["accuracy"] = acc
    if cpu is not None:
        v, cores, desc = cpu
        line["cpu_baseline"] = {"value": v, "unit": "instance-steps/s", "cores": cores, "kind": "port",
                                "sample": desc}
    m.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


SERVE_GRIDS = [(16, 8), (32, 8), (32, 16), (64, 16)]


def run_serving(args):
    """Config 4: a Poisson stream of solve requests over four grids, served with continuous
    batching; p50/p99 time-to-solution and aggregate instance-steps/s, beside the same stream
    one at a time on the plain FP64 path (FIFO single server with per-grid FP64 step times
    measured here)."""
    import numpy as np
    import torch
    from dtb import synth
    from dtb.batch import BatchedEuler
    from dtb.serve import Server
    from dtb.stepping import ForwardEulerStruct
    from dtb.structs import BinaryMatrices
    rank, local, world = _env_rank()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    if args.tune_cache:
        from dtb.batch import set_tune_cache
        set_tune_cache(args.tune_cache)
    rng = np.random.default_rng(44)
    n_req = args.requests
    rate = args.rate
    grids, batched, step_ms_fp64 = [], [], []
    srv = Server(hbm_budget_bytes=150 * 10**9)
    gids = []
    for g, (p, u) in enumerate(SERVE_GRIDS):
        w = synth.two_species(p, 1e-2, 1e2, u, seed=100 + g, gain_on_device=True, device=f"cuda:{local}")
        b = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, args.capacity, device=local)
        gids.append(srv.add_grid(b))
        # plain FP64 step time of this grid (one instance), for the one-at-a-time comparison
        gains64 = [type(x)(x.out_sp, x.in1_sp, x.in2_sp, x.G.double()) for x in w.binm.gains]
        ps_stream = torch.cuda.Stream()
        pl = ForwardEulerStruct(w.ps, w.f0, w.inj, BinaryMatrices(gains=gains64, losses=w.binm.losses), w.emim,
                                w.fluxm, Precision=np.float64, device=local, stream=ps_stream.cuda_stream)
        del gains64
        pl.run(np.ones(8))
        K = 200 if p * u <= 256 else 50
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(ps_stream)
        pl.run(np.ones(K))
        t1.record(ps_stream)
        torch.cuda.synchronize()
        step_ms_fp64.append(t0.elapsed_time(t1) / K)
        pl.close()
        w.binm.gains = []
        torch.cuda.empty_cache()
        grids.append(w)
        batched.append(b)
    # the request stream
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_req))
    gsel = rng.integers(0, len(SERVE_GRIDS), size=n_req)
    steps = rng.integers(500, 20001, size=n_req)
    mus = rng.uniform(-1, 1, size=n_req)
    dts = rng.uniform(0.5, 1.0, size=n_req)
    f0s = [synth.lognormal_f0(grids[g].ps, [mu, mu], 1.0) for g, mu in zip(gsel, mus)]
    srv.start()
    t_start = time.perf_counter()
    rids = []
    for k in range(n_req):
        delay = arrivals[k] - (time.perf_counter() - t_start)
        if delay > 0:
            time.sleep(delay)
        rids.append(srv.submit(gids[gsel[k]], f0s[k], float(dts[k]), int(steps[k])))
    infos = [srv.wait(r, timeout_s=3600, with_f=False)[1] for r in rids]
    st = srv.stats()
    srv.close()
    for b in batched:
        b.close()
    tts = np.array([i["t_done"] - i["t_submit"] for i in infos])
    t_first = min(i["t_submit"] for i in infos)
    t_last = max(i["t_done"] for i in infos)
    total = int(steps.sum())
    agg = total / (t_last - t_first)
    # one at a time on the plain FP64 path: FIFO single server over the same arrivals
    svc = np.array([steps[k] * step_ms_fp64[gsel[k]] / 1e3 for k in range(n_req)])
    free_at, tts_plain, done_plain = 0.0, [], []
    for k in range(n_req):
        start = max(free_at, arrivals[k])
        free_at = start + svc[k]
        tts_plain.append(free_at - arrivals[k])
    agg_plain = total / (free_at - arrivals[0])
    line = {"metric": METRIC, "value": agg, "unit": "instance-steps/s", "n_gpus": 1, "steps": total,
            "warmup": 0, "ms_per_step": 1e3 / agg, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16x3 (gain GEMM), f32 state, f64 update",
            "data": "synthetic (seeded Poisson stream, seeded operators and spectra)",
            "config": {"workload": f"serving (config 4): {n_req} requests, Poisson rate {rate}/s, grids "
                                   "p16xu8, p32xu8, p32xu16, p64xu16 (2 species), 500-20000 steps each",
                       "capacity_per_grid": args.capacity, "hbm_budget_bytes": 150 * 10**9,
                       "device_bytes": st["device_bytes"]},
            "tts_p50_s": float(np.percentile(tts, 50)), "tts_p99_s": float(np.percentile(tts, 99)),
            "plain_fp64_one_at_a_time": {"value": agg_plain, "unit": "instance-steps/s",
                                         "tts_p50_s": float(np.percentile(tts_plain, 50)),
                                         "tts_p99_s": float(np.percentile(tts_plain, 99)),
                                         "step_ms_per_grid": step_ms_fp64,
                                         "method": "FIFO single server over the same arrivals, service time = "
                                                   "steps x FP64 step time measured per grid"},
            "speedup_vs_plain_fp64": agg / agg_plain,
            "serve_stats": st}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grid", default=None, help="p_bins x u_bins override of the config-1 grid, e.g. 32x16")
    ap.add_argument("--no-check", action="store_true", help="skip the FP64 accuracy check of the batched run")
    ap.add_argument("--tune-cache", default=None,
                    help="gain-GEMM plan cache file: plans recorded there are reused, new ones are measured and "
                         "appended (a profiling run can replay the plan a plain run chose)")
    ap.add_argument("--requests", type=int, default=2000, help="serving stream length (--config 4)")
    ap.add_argument("--rate", type=float, default=20.0, help="mean request arrival rate per second (--config 4)")
    ap.add_argument("--capacity", type=int, default=256, help="slots per grid (--config 4)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        return run_reference(args)
    if args.config in (2, 3):
        return run_batched(args)
    if args.config == 4:
        return run_serving(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
