"""Benchmark of the explicit Euler step on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K (2000)] [--warmup W (5)] [--impl ours|reference]
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
plain_fp64: one instance of the same grid on the plain FP64 path (graphs prepared, the same
W warm-up and K timed steps), with its gain kernel's HBM roofline.
accuracy: every instance re-run over the configuration's run length (10,000 steps for config
2, 5,000 for config 3); three instances compared with the plain FP64 path over the same steps,
with FP64 number and energy moments (drift of both paths, and the mixed path's error against
FP64); also a W-step comparison with the FP64 oracle itself.
serving (default run): 200 requests per GPU of config 4's grids and request mix at 0.7 of the
full-occupancy capacity, routed across GPUs; p50/p99 time to solution (tts_p50_s, tts_p99_s).
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
    """nvidia-smi clocks and throttle reasons sampled every 100 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: str):
        self.gpu = gpu
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            time.sleep(0.4)  # the sampler is up before the timed region starts
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


def build_batched(config: int, device: str, host: bool = False, grid=None):
    from dtb import synth
    if config == 3 and grid:  # the config-3 recipe on another grid, e.g. "24x12" (small profiling case)
        p, u = (int(x) for x in grid.split("x"))
        w = synth.three_species(p, 1e-3, 1e3, u, 64, seed=3, gain_on_device=not host, device=device)
        w.n_steps = 5000
        return w
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
                "data": "synthetic (seeded; no collision data files)", "config": _config_dict(args.config, w, world),
                "precision": "FP64 oracle port (C, OpenMP): FP64 operators and state",
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
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded; no collision data files)",
            "config": _config_dict(args.config, w, world),
            "precision": "FP64 oracle port (C, OpenMP): FP64 operators and state",
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


def _config_dict(config: int, w, world: int = 1):
    """The workload description; both arms (--impl ours / reference) print the same object."""
    sizes = w.ps.species_sizes
    if config == 2:
        return {"workload": "batching (config 2): 256 independent instances, 2 species x 256 states "
                            "(32 log p x 8 u), shared G 2 x 256 x 65536, per-instance f0 and dt",
                "species_states": sizes, "batch": 256, "run_length_steps": 10000,
                "l2": "G hi+lo 134 MB per step, larger than L2", "parallelism": f"batch replicas x{world}"}
    if config == 3 and sizes != [576, 576, 576]:
        return {"workload": f"config-3 recipe on a smaller grid: 64 instances, 3 species x {sizes[0]} states",
                "species_states": sizes, "batch": 64, "parallelism": f"batch replicas x{world}"}
    if config == 3:
        return {"workload": "mixed precision (config 3): 64 instances, e-, e+, gamma x 576 states "
                            "(48 log p x 12 u), 6 gain tensors 576 x 331776, synchrotron-like emission",
                "species_states": sizes, "batch": 64, "run_length_steps": 5000,
                "l2": "G hi+lo 4.6 GB per step, larger than L2", "parallelism": f"batch replicas x{world}"}
    if config == 1 and sizes != [1024, 1024]:
        return {"workload": f"config-1 recipe on a smaller grid: 2 species x {sizes[0]} states",
                "species_states": sizes, "parallelism": f"replicas x{world}"}
    if config == 1:
        return {"workload": "plain single instance (config 1): 2 species x 1024 states (64 log p x 16 u), "
                            "gain 2 x 1024 x 1048576, 2000-step run shape",
                "species_states": sizes, "l2": "inputs larger than L2 (8.6 GB gain)",
                "parallelism": f"replicas x{world}"}
    return {"workload": "plain single instance (config 0): 2 species x 128 states (16 log p x 8 u)",
            "species_states": sizes,
            "l2": "operators (34 MB) fit in L2; no flush between steps (launch/L2-bound case)",
            "parallelism": f"replicas x{world}"}


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
    # graphs captured and uploaded first, then exactly W warm-up steps
    K, W = args.steps, args.warmup
    scales = np.ones(K)
    m.prepare()
    m.run(np.ones(W))
    nl0, nl1 = _lib.ctypes.c_int64(), _lib.ctypes.c_int64()
    L.dtb_launch_count(m.ctx, _lib.ctypes.byref(nl0))
    # ---- timed region: device resident, graph replay
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
    L.dtb_launch_count(m.ctx, _lib.ctypes.byref(nl1))
    # ---- CUDA events around every gain-kernel launch (direct launches): 8 discarded, then
    # max(K, 400) timed
    L.dtb_set_profiling(m.ctx, 1)
    m.run(scales[:PROF_WARM] if len(scales) >= PROF_WARM else np.full(PROF_WARM, scales[0]))
    L.dtb_set_profiling(m.ctx, 1)
    m.run(np.resize(scales, max(len(scales), PROF_MIN)))
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
        m.step_io(f_host, 0.0, 1e30, m.dt0, 0, out=f_host)  # upload, step, download: one wait
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
    traffic = _profile_traffic("gain_stream_f32_config1.md") if args.config == 1 and not args.grid else None
    line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": dtype, "data": "synthetic (seeded; no collision data files)",
            "config": _config_dict(args.config, w, world),
            "precision": "FP32 operators and state" if dtype == "f32" else "FP64 operators and state",
            "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": n * esz,
                    "d2h_bytes_per_step": n * esz, "wall_s": t_wall},
            "gpu_launches": int(nl1.value - nl0.value),
            "roofline": {"bound": "hbm", "kernel": "gain_stream", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None,
                         "traffic": traffic, "algorithmic_bytes_per_launch": bpl.value,
                         "avg_launch_ms": avg_ms.value,
                         "step_frac": bpl.value / (ms / K / 1e3) / 1e9 / peak,
                         "l2_resident": bpl.value < 100e6},
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


PROF_WARM = 8    # discarded direct launches before a kernel's per-launch timing
PROF_MIN = 400   # at least this many timed launches


def _plain_leg(plain, stream, dt: float, K: int, W: int, hbm: float):
    """Plain FP64 single instance on the batched grid: graphs prepared, W warm-up steps, K timed
    steps (CUDA events on the library's stream), then the gain kernel timed per launch for its
    HBM roofline (8 discarded launches, then max(K, 400)). Returns the plain leg's JSON object."""
    import numpy as np
    import torch
    from dtb import _lib
    plain.prepare()
    plain.run(np.full(W, dt))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    plain.run(np.full(K, dt))
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    L = plain.L
    L.dtb_set_profiling(plain.ctx, 1)
    plain.run(np.full(PROF_WARM, dt))  # discarded
    L.dtb_set_profiling(plain.ctx, 1)  # restarts the average
    plain.run(np.full(max(K, PROF_MIN), dt))
    avg_ms, bpl = _lib.ctypes.c_double(), _lib.ctypes.c_double()
    L.dtb_gain_kernel_stats(plain.ctx, _lib.ctypes.byref(avg_ms), _lib.ctypes.byref(bpl))
    L.dtb_set_profiling(plain.ctx, 0)
    step_ms = ms / K
    gbs_kernel = bpl.value / (avg_ms.value / 1e3) / 1e9 if avg_ms.value > 0 else None
    gbs_step = bpl.value / (step_ms / 1e3) / 1e9
    return {"value": 1e3 / step_ms, "unit": "steps/s", "ms_per_step": step_ms, "steps": K, "warmup": W,
            "workload": "same grid, one instance, FP64 (gain_stream + euler_rows per step)",
            "roofline": {"bound": "hbm", "kernel": "gain_stream<double>", "unit": "GB/s",
                         "algorithmic_bytes_per_step": bpl.value, "avg_launch_ms": avg_ms.value,
                         "achieved": gbs_kernel, "frac": gbs_kernel / hbm if gbs_kernel else None,
                         "step_achieved": gbs_step, "step_frac": gbs_step / hbm, "peak": hbm}}


def _accuracy_leg(m, w, plain, n_steps: int, inst, oracle_ops=None):
    """Full-length accuracy of the batched mixed path: every slot re-admitted with its f0 and
    run n_steps; the instances `inst` compared with the plain FP64 GPU path over the same steps
    (relative L-inf), and FP64 device moments (number, energy per species) before and after for
    both, giving each path's drift |S(T) - S(0)| / S(0) and the mixed path's error in them
    |S_mixed(T) - S_fp64(T)| / max(|S_fp64(T)|, S(0)) (a species the run depletes is measured
    against its initial amount). With oracle_ops, instance inst[0] is also run on the
    FP64 oracle (host) over the same steps."""
    import numpy as np
    from dtb.structs import energy_weights
    B = w.f0.shape[0]
    for i in range(B):
        m.admit(i, w.f0[i], float(w.dt[i]), n_steps)
    wts = energy_weights(w.ps)
    num0, en0 = m.moments(wts)
    m.run(n_steps)
    num1, en1 = m.moments(wts)
    errs, drift = {}, []
    for i in inst:
        plain.f = w.f0[i]
        plain.run(np.full(n_steps, float(w.dt[i])))
        ref = plain.f
        got = m.get_f(i)
        errs[str(i)] = float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))
        pn, pe = plain.moments(wts)
        pn, pe = np.asarray(pn)[0], np.asarray(pe)[0]
        drift.append({
            "instance": i,
            "number_drift_mixed": (np.abs(num1[i] - num0[i]) / num0[i]).tolist(),
            "number_drift_fp64": (np.abs(pn - num0[i]) / num0[i]).tolist(),
            "energy_drift_mixed": (np.abs(en1[i] - en0[i]) / en0[i]).tolist(),
            "energy_drift_fp64": (np.abs(pe - en0[i]) / en0[i]).tolist(),
            "number_error_mixed_vs_fp64": (np.abs(num1[i] - pn) / np.maximum(np.abs(pn), num0[i])).tolist(),
            "energy_error_mixed_vs_fp64": (np.abs(en1[i] - pe) / np.maximum(np.abs(pe), en0[i])).tolist()})
    out = {"steps": n_steps, "instances": list(inst), "rel_linf_vs_fp64": max(errs.values()),
           "rel_linf_per_instance": errs,
           "reference": "plain FP64 GPU path, same f0 and dt (FP64 oracle parity <= 1e-12 in tests)",
           "tolerance": 1e-5, "moments": drift,
           "max_number_error_mixed_vs_fp64": max(max(d["number_error_mixed_vs_fp64"]) for d in drift),
           "max_energy_error_mixed_vs_fp64": max(max(d["energy_error_mixed_vs_fp64"]) for d in drift)}
    if oracle_ops is not None:
        i = inst[0]
        f = np.array(w.f0[i])
        for _ in range(n_steps):
            f, _, _ = oracle_ops.step(f, float(w.dt[i]), 0)
        got = m.get_f(i)
        out["oracle"] = {"instance": i, "steps": n_steps,
                         "rel_linf_mixed_vs_oracle": float(np.max(np.abs(got - f)) / np.max(np.abs(f)))}
    return out


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
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    dev = f"cuda:{local}"
    w = build_batched(args.config, dev, grid=args.grid)
    if args.shard and world > 1:
        # strong scaling: the configuration's instances partitioned across the ranks
        from dtb.shard import shard_range
        lo, hi = shard_range(w.f0.shape[0], rank, world)
        w.f0, w.dt = w.f0[lo:hi], w.dt[lo:hi]
    B = w.f0.shape[0]
    n = w.ps.n_state
    K, W = args.steps, args.warmup
    stream = torch.cuda.Stream()
    m = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B, device=local, stream=stream.cuda_stream)
    for i in range(B):
        m.admit(i, w.f0[i], float(w.dt[i]), 1 << 40)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_sample_batched(w, budget_s=15.0)
    ops = None
    if rank == 0 and not args.no_check:
        import oracle
        gains = [type(g)(g.out_sp, g.in1_sp, g.in2_sp, g.G.double().cpu().numpy()) for g in w.binm.gains]
        ops = oracle.BlockedOperands(w.ps.species_sizes, 1, gains, w.binm.losses, w.emim.blocks, w.fluxm.F_Flux,
                                     1.0 / np.asarray(w.fluxm.Ap_Flux), w.fluxm.Vol, w.inj)
        del gains
    # plain FP64 path on the same grid (one instance), for the batched-vs-plain comparison
    gains64 = [type(g)(g.out_sp, g.in1_sp, g.in2_sp, g.G.double()) for g in w.binm.gains]
    from dtb.structs import BinaryMatrices
    binm64 = BinaryMatrices(gains=gains64, losses=w.binm.losses)
    plain = ForwardEulerStruct(w.ps, w.f0[0], w.inj, binm64, w.emim, w.fluxm, Precision=np.float64, device=local,
                               stream=stream.cuda_stream)
    del gains64, binm64
    w.binm.gains = [type(g)(g.out_sp, g.in1_sp, g.in2_sp, None) for g in w.binm.gains]
    torch.cuda.empty_cache()
    # graphs captured and uploaded before any step, then exactly W warm-up steps
    m.prepare()
    m.run(W)
    acc_short = None
    if ops is not None:
        errs = []
        for i in (0, B - 1):
            f = np.array(w.f0[i])
            for _ in range(W):
                f, _, _ = ops.step(f, float(w.dt[i]), 0)
            g = m.get_f(i)
            errs.append(float(np.max(np.abs(g - f)) / np.max(np.abs(f))))
        acc_short = {"rel_linf_vs_fp64_oracle": max(errs), "steps": W, "instances": [0, B - 1]}
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
    # ---- CUDA events around every gain-GEMM launch (direct launches): a few launches to warm the
    # direct-launch path (discarded), then max(K, 400) timed launches, so a short timed region
    # (20 steps) still gives a steady per-launch average
    m.set_profiling(True)
    m.run(PROF_WARM)
    m.set_profiling(True)  # restarts the averages
    K_prof = max(K, PROF_MIN)
    e4, e5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e4.record(stream)
    m.run(K_prof)
    e5.record(stream)
    torch.cuda.synchronize()
    ms_prof = e4.elapsed_time(e5) * K / K_prof
    st = m.gemm_stats()
    plans = []
    while (pl := m.gemm_plan(len(plans))) is not None:
        plans.append(pl)
    m.set_profiling(False)
    # ---- e2e: the whole batch state from pinned host memory in and out every step, K steps
    Fh = torch.empty((B, n), dtype=torch.float64).pin_memory().numpy()
    m.get_f_all(Fh)
    m.run_io(Fh, 1, Fh)  # the 1-step graphs of both state buffers are warm
    m.run_io(Fh, 1, Fh)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(K):
        m.run_io(Fh, 1, Fh)  # upload, one batched step, download: one call, one wait
    e3.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e2.elapsed_time(e3)
    pj = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm = float(pj.get("hbm_gbs", 6650.0))
    # ---- plain FP64 single instance on the same grid
    plain_line = _plain_leg(plain, stream, float(w.dt[0]), K, W, hbm)
    ms_plain = plain_line["ms_per_step"] * K
    # ---- accuracy and drift over the configuration's full run length
    acc = None
    if rank == 0 and not args.no_check:
        L_run = args.check_steps if args.check_steps is not None else int(w.n_steps)
        acc = _accuracy_leg(m, w, plain, L_run, [0, B // 2, B - 1], ops if args.oracle_long else None)
        acc["short_run_vs_oracle"] = acc_short
    plain.close()
    if world > 1:
        t = torch.tensor([ms, ms_e2e, ms_plain], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_e2e, ms_plain = float(t[0]), float(t[1]), float(t[2])
    # every rank steps B instances (its share when sharded); the whole job is the sum
    B_all = sum(_gather_ints([B])) if world > 1 else B
    value = B_all * K / (ms / 1e3)
    plain_sps = world * K / (ms_plain / 1e3)
    plain_line["value"] = plain_sps
    peak = float(pj.get("bf16_tflops", 1590.0))
    peak_s = float(pj.get("bf16_tflops_sustained", 1400.0))
    achieved = st["flops_per_step"] / (st["avg_ms"] / 1e3) / 1e12 if st["avg_ms"] > 0 else None
    # per step of the configuration's own grid (a --grid case has other operator bytes)
    traffic = _profile_traffic(f"gain_gemm_config{args.config}.md") if not args.grid else None
    # 256-column tiles over an even number of 128-row m tiles run on SM pairs (cta_group::2)
    GEMM_LABEL = ("gain_gemm_pair (tcgen05.mma.cta_group::2, BF16 hi+lo x3)" if all(p["pair"] for p in plans)
                  else "gain_gemm (tcgen05, BF16 hi+lo x3)")
    # the GEMM's bound: the slower of its tensor time and its operator-streaming time
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
    cfg = _config_dict(args.config, w, world)
    if args.shard and world > 1:
        cfg["parallelism"] = f"instances sharded over {world} GPUs"
    line = {"metric": METRIC, "value": value, "unit": "instance-steps/s", "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True,
            "scaling": "strong" if (args.shard and world > 1) else "weak", "vs_baseline": None,
            "dtype": "bf16x3 (gain GEMM), f32 state, f64 update", "data": "synthetic (seeded; no collision data files)",
            "config": cfg,
            "precision": "BF16 hi+lo gain (3 MMAs, FP32 accumulation), FP32 f, FP64 compensated update",
            "e2e": {"value": B_all * K / (ms_e2e / 1e3), "unit": "instance-steps/s",
                    "h2d_bytes_per_step": B * n * 8, "d2h_bytes_per_step": B * n * 8, "steps": K},
            "gpu_launches": int(st["launches_per_step"]) * K + (K + 15) // 16,  # + one step-counter advance per graph
            "roofline": roof,
            "plain_fp64": plain_line,
            "speedup_vs_plain_fp64": value / plain_sps,
            "clocks": cs.summary()}
    if acc is not None:
        line["accuracy"] = acc
    if cpu is not None:
        v, cores, desc = cpu
        line["cpu_baseline"] = {"value": v, "unit": "instance-steps/s", "cores": cores, "kind": "port",
                                "sample": desc}
    m.close()
    torch.cuda.empty_cache()
    if args.config == 2 and args.serve_requests > 0:
        # the metric's p99: a served stream (config 4's grids and request mix) at 0.7 of capacity
        setup = _serving_grids(local, args.capacity)
        sv = _serving_leg(rank, world, local, args.serve_requests, 0.7, args.capacity, 45, setup)
        for b in setup[1]:
            b.close()
        line["tts_p50_s"], line["tts_p99_s"] = sv["tts_p50_s"], sv["tts_p99_s"]
        line["serving"] = sv
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


SERVE_GRIDS = [(16, 8), (32, 8), (32, 16), (64, 16)]


def _gather_ints(vals):
    """Every rank's list of ints, concatenated in rank order (torch.distributed)."""
    import torch.distributed as dist
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, list(vals))
    return [v for part in out for v in part]


def _serving_grids(local: int, capacity: int):
    """The four served grids (2 species each, seeded operators): one batched context per grid
    with `capacity` slots, the batched step time of each grid with every slot running, and the
    plain FP64 step time of one instance (the one-at-a-time comparison)."""
    import numpy as np
    import torch
    from dtb import synth
    from dtb.batch import BatchedEuler
    from dtb.stepping import ForwardEulerStruct
    from dtb.structs import BinaryMatrices
    grids, batched, t_full_ms, step_ms_fp64 = [], [], [], []
    for g, (p, u) in enumerate(SERVE_GRIDS):
        w = synth.two_species(p, 1e-2, 1e2, u, seed=100 + g, gain_on_device=True, device=f"cuda:{local}")
        stream = torch.cuda.Stream()
        gains64 = [type(x)(x.out_sp, x.in1_sp, x.in2_sp, x.G.double()) for x in w.binm.gains]
        pl = ForwardEulerStruct(w.ps, w.f0, w.inj, BinaryMatrices(gains=gains64, losses=w.binm.losses), w.emim,
                                w.fluxm, Precision=np.float64, device=local, stream=stream.cuda_stream)
        del gains64
        pl.prepare()
        pl.run(np.ones(4))
        K = 200 if p * u <= 256 else 48
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        pl.run(np.ones(K))
        t1.record(stream)
        torch.cuda.synchronize()
        step_ms_fp64.append(t0.elapsed_time(t1) / K)
        pl.close()
        torch.cuda.empty_cache()
        b = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, capacity, device=local, stream=stream.cuda_stream)
        w.binm.gains = []
        torch.cuda.empty_cache()
        # full occupancy: every slot running
        for sl in range(capacity):
            b.admit(sl, w.f0, 1.0, 1 << 40)
        b.prepare()
        b.run(3)
        Kb = 48 if p * u >= 1024 else 160
        t0.record(stream)
        b.run(Kb)
        t1.record(stream)
        torch.cuda.synchronize()
        t_full_ms.append(t0.elapsed_time(t1) / Kb)
        for sl in range(capacity):
            b.release(sl)
        grids.append(w)
        batched.append(b)
    return grids, batched, t_full_ms, step_ms_fp64


def _request_stream(n: int, rate: float, seed: int, rng_grids: int):
    import numpy as np
    rng = np.random.default_rng(seed)
    return {"arrivals": np.cumsum(rng.exponential(1.0 / rate, size=n)),
            "grid": rng.integers(0, rng_grids, size=n), "steps": rng.integers(500, 20001, size=n),
            "mu": rng.uniform(-1, 1, size=n), "dt": rng.uniform(0.5, 1.0, size=n)}


def _serve_share(batched, grids, stream, mine, budget):
    """Serves the requests `mine` (global indices into `stream`) on this GPU with continuous
    batching, submitting each at its arrival time; one record per request."""
    import numpy as np
    from dtb import synth
    from dtb.serve import Server
    srv = Server(hbm_budget_bytes=budget)
    gids = [srv.add_grid(b) for b in batched]
    f0s = {k: synth.lognormal_f0(grids[stream["grid"][k]].ps, [stream["mu"][k]] * 2, 1.0) for k in mine}
    srv.start()
    t_start = time.perf_counter()
    rids = []
    for k in mine:
        delay = stream["arrivals"][k] - (time.perf_counter() - t_start)
        if delay > 0:
            time.sleep(delay)
        rids.append(srv.submit(gids[stream["grid"][k]], f0s[k], float(stream["dt"][k]), int(stream["steps"][k])))
    infos = [srv.wait(r, timeout_s=3600, with_f=False)[1] for r in rids]
    st = srv.stats()
    srv.close()
    recs = [{"tts": i["t_done"] - i["t_submit"], "t_submit": i["t_submit"], "t_done": i["t_done"],
             "queue_s": i["t_admit"] - i["t_submit"], "steps": int(i["steps"]), "finite": bool(i["finite"])}
            for i in infos]
    if recs:
        recs[0]["serve_stats"] = st
    return recs


def _serving_leg(rank: int, world: int, local: int, n_req: int, load: float, capacity: int, seed: int,
                 setup=None, rate=None):
    """One served stream: n_req requests per GPU (weak scaling), Poisson arrivals at `load` times
    the capacity of the four grids at full occupancy (or at `rate` requests/s per GPU), routed
    across ranks; p50/p99 time to solution and aggregate instance-steps/s, beside the same requests
    served one at a time on the plain FP64 path (FIFO per GPU)."""
    import numpy as np
    from dtb.shard import route, serve_sharded
    grids, batched, t_full_ms, step_ms_fp64 = setup
    mean_steps = (500 + 20000) / 2.0
    # at full occupancy every grid is stepping; one step of every grid moves 4 x capacity instances
    lam_max = len(SERVE_GRIDS) * capacity / (mean_steps * sum(t_full_ms) / 1e3)
    lam = rate if rate is not None else load * lam_max
    stream = _request_stream(n_req * world, lam * world, seed, len(SERVE_GRIDS))
    budget = 150 * 10**9
    recs = serve_sharded([float(x) for x in stream["steps"]], rank, world,
                         lambda mine: _serve_share(batched, grids, stream, mine, budget))
    tts = np.array([r["tts"] for r in recs])
    total = int(stream["steps"].sum())
    span = max(max(r["t_done"] for r in recs if r["rank"] == q) - min(r["t_submit"] for r in recs if r["rank"] == q)
               for q in set(r["rank"] for r in recs))
    # one at a time on the plain FP64 path: a FIFO single server per GPU over the same arrivals
    ranks = route([float(x) for x in stream["steps"]], world)
    tts_plain, span_plain = [], 0.0
    for q in range(world):
        free_at, first = 0.0, None
        for k in (k for k in range(len(ranks)) if ranks[k] == q):
            a = float(stream["arrivals"][k])
            first = a if first is None else first
            free_at = max(free_at, a) + stream["steps"][k] * step_ms_fp64[stream["grid"][k]] / 1e3
            tts_plain.append(free_at - a)
        if first is not None:
            span_plain = max(span_plain, free_at - first)
    stats = [r["serve_stats"] for r in recs if "serve_stats" in r]
    return {"requests": n_req * world, "load": None if rate is not None else load,
            "rate_per_s": lam * world, "capacity_rate_per_s": lam_max * world,
            "tts_p50_s": float(np.percentile(tts, 50)), "tts_p99_s": float(np.percentile(tts, 99)),
            "queue_p99_s": float(np.percentile([r["queue_s"] for r in recs], 99)),
            "instance_steps_per_s": total / span, "all_finite": all(r["finite"] for r in recs),
            "full_occupancy_step_ms": t_full_ms, "capacity_per_grid": capacity,
            "plain_fp64_one_at_a_time": {"instance_steps_per_s": total / span_plain,
                                         "tts_p50_s": float(np.percentile(tts_plain, 50)),
                                         "tts_p99_s": float(np.percentile(tts_plain, 99)),
                                         "step_ms_per_grid": step_ms_fp64,
                                         "method": "FIFO single server per GPU over the same arrivals, service "
                                                   "time = steps x FP64 step time measured per grid"},
            "device_bytes": sum(s["device_bytes"] for s in stats) // max(1, len(stats)),
            "busy_s": max((s["busy_s"] for s in stats), default=None)}


def run_serving(args):
    """Config 4: Poisson streams of solve requests over four grids served with continuous
    batching at each requested load (fraction of the full-occupancy capacity), or one stream at
    --rate; p50/p99 time to solution and aggregate instance-steps/s, beside the same stream one
    at a time on the plain FP64 path."""
    import torch
    import torch.distributed as dist
    rank, local, world = _env_rank()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    if args.tune_cache:
        from dtb.batch import set_tune_cache
        set_tune_cache(args.tune_cache)
    setup = _serving_grids(local, args.capacity)
    points = []
    if args.rate is not None:
        points.append(_serving_leg(rank, world, local, args.requests, 0.0, args.capacity, 44, setup, rate=args.rate))
    else:
        for ld in args.loads:
            points.append(_serving_leg(rank, world, local, args.requests, ld, args.capacity, 44, setup))
    for b in setup[1]:
        b.close()
    head = points[0]
    line = {"metric": METRIC, "value": head["instance_steps_per_s"], "unit": "instance-steps/s", "n_gpus": world,
            "steps": int(args.requests * world), "warmup": 0, "ms_per_step": 1e3 / head["instance_steps_per_s"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16x3 (gain GEMM), f32 state, f64 update",
            "data": "synthetic (seeded Poisson stream, seeded operators and spectra)",
            "config": {"workload": f"serving (config 4): {args.requests} requests per GPU, grids p16xu8, p32xu8, "
                                   "p32xu16, p64xu16 (2 species), 500-20000 steps each",
                       "capacity_per_grid": args.capacity, "hbm_budget_bytes": 150 * 10**9,
                       "parallelism": f"requests routed over {world} GPU(s)"},
            "tts_p50_s": head["tts_p50_s"], "tts_p99_s": head["tts_p99_s"], "serving": points}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grid", default=None,
                    help="p_bins x u_bins override of the config-1 or config-3 grid, e.g. 32x16 (profiling cases)")
    ap.add_argument("--no-check", action="store_true", help="skip the FP64 accuracy checks of the batched run")
    ap.add_argument("--check-steps", type=int, default=None,
                    help="length of the batched accuracy run (default: the configuration's run length, "
                         "10000 steps for --config 2, 5000 for --config 3)")
    ap.add_argument("--oracle-long", action="store_true",
                    help="also run one instance of the accuracy run on the FP64 oracle (host cores)")
    ap.add_argument("--tune-cache", default=None,
                    help="gain-GEMM plan cache file: plans recorded there are reused, new ones are measured and "
                         "appended (a profiling run can replay the plan a plain run chose)")
    ap.add_argument("--requests", type=int, default=200, help="serving stream length per GPU (--config 4)")
    ap.add_argument("--rate", type=float, default=None,
                    help="mean request arrival rate per second per GPU (--config 4; default: --loads)")
    ap.add_argument("--loads", type=lambda x: [float(v) for v in x.split(",")], default=[0.5, 0.7, 0.9],
                    help="serving loads as fractions of the four grids' full-occupancy capacity (--config 4)")
    ap.add_argument("--shard", action="store_true",
                    help="batched configs under torchrun: partition the instances across the GPUs (strong "
                         "scaling) instead of a full batch per GPU (weak scaling)")
    ap.add_argument("--serve-requests", type=int, default=200,
                    help="requests per GPU of the default run's serving leg (0: skip it)")
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
