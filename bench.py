#!/usr/bin/env python
"""Benchmark of the step engine on the headline workload.

Workload (the reference's Hohenberg-Halperin compressible configuration):
1024x1024 active grid (3/2 rule -> 1536^2 compute grid), Lx = Ly = 2048 (grid
spacing 2, which keeps -M k^2 (a + b k^2) dt of every active mode inside the
SRK3 stability interval at dt = 0.01; at spacing 1 the highest modes grow),
N = 2 order parameters with phi4 free energy (mu_a = -psi_a + psi_a^3 -
lap psi_a), M_a = 1, rho0 = 1, eta = zeta = 1, linear EOS cT = 1, advection of
psi and j, conservative noise kBT = 1e-3, psi initial state equilibrium
Gaussian (seed 7, real-space std ~0.1), SRK3 with dt = 0.01.  Synthetic
inputs of that shape (no dataset is involved).

One "step" = one SRK3 step of one trajectory.  `value` = trajectory steps/s
over all ranks (each rank advances its own replica: the single-grid path has
no data-path collective), timed on the device with CUDA events on the
engine's stream, max over ranks.  `e2e` = the same metric through the C ABI
with host buffers: every step uploads the host State (reference layout,
pinned), steps, and downloads the host State, as a drop-in
FluidSolver::step(State&) must.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "spectral-hohenberg-halperin-dynamics-2d_b200")
sys.path.insert(0, PKG)

METRIC = "SRK3 steps/s (1024^2, N=2)"
UNIT = "steps/s"
L2_BYTES = 126 * 1024 * 1024

WORKLOAD = """dimension 2
boundary p p
grid 1024 1024
length 2048 2048
dealias 3/2
order_parameters 2
timestep 0.01
time_evolution srk3/compressible
model thermo linear_eos cT 1
model free_energy phi4 a[0] -1 b[0] 1 u[0] 1 a[1] -1 b[1] 1 u[1] 1
model transport constant eta 1 zeta 1 M[0,0] 1 M[1,1] 1
fix 1 all nonlinear on
fix 2 all noise on seed 7 kBT 1e-3
set density uniform value 1.0
set order_parameter all equilibrium/gaussian seed 7 kBT 0.0400782395901117 k0 1 k2 0
run 10000
"""

# ensemble configuration: 256 members, 256^2 (3/2 -> 384^2), quiescent phi4 quench; grid spacing 2
# (length 512) keeps -M k^2 (a + b k^2) dt inside the SRK3 stability interval at dt = 0.02
ENSEMBLE = """dimension 2
grid 256 256
length 512 512
dealias 3/2
order_parameters 1
timestep 0.02
time_evolution srk3/quiescent
model free_energy phi4 a[0] -1 b[0] 1 u[0] 1
model transport constant eta 0 zeta 0 M[0,0] 1
fix 1 order_parameter noise on seed 0 kBT 0.05
set density uniform value 1.0
set order_parameter all equilibrium/gaussian seed 0 kBT 0.040314340638216074 k0 1 k2 0
run 5000
"""

CONFIG = {
    "workload": "HH compressible 1024^2 (3/2 -> 1536^2), N=2 phi4, advection + noise, SRK3 dt=0.01",
    "grid": [1024, 1024],
    "length": [2048, 2048],
    "compute_grid": [1536, 1536],
    "order_parameters": 2,
    "mode": "srk3/compressible",
    "l2": "no flush: per-step working set (3 states + 16 transform planes) exceeds the 126 MB L2",
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
# process group (one rank per GPU)
# ---------------------------------------------------------------------------
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def launch_plan(gpus: int, env) -> str:
    """How `bench.py --gpus N` runs: "run" (this process is one of the N ranks, or N = 1),
    "spawn" (N > 1 and no launcher: re-execute under torch.distributed.run with N ranks).
    A launcher whose world size differs from --gpus is an error, so an N-GPU number is never
    a silent 1-GPU run."""
    if gpus < 1:
        raise SystemExit(f"bench.py: --gpus must be >= 1 (got {gpus})")
    if "WORLD_SIZE" in env:
        world = int(env["WORLD_SIZE"])
        if world != gpus:
            raise SystemExit(f"bench.py: --gpus {gpus} but the launcher started {world} ranks (WORLD_SIZE)")
        return "run"
    return "spawn" if gpus > 1 else "run"


def spawn_command(argv, gpus: int, port: int):
    """torch.distributed.run command line that starts `gpus` ranks of this script on this node."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}", "--master-addr=127.0.0.1",
            f"--master-port={port}", os.path.abspath(__file__)] + list(argv)


def init_group(world, local, backend):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    if world > 1:
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=120))
    return dist


def max_over_ranks(x: float, world: int) -> float:
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str):
        self.uuid = uuid
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="shhd_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.2)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            if self.uuid and parts[0] != self.uuid:
                continue
            rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[i] for r in rows for i in range(4) if r[4 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ---------------------------------------------------------------------------
# CPU baselines (the reference's own code; the numpy port if that is absent)
# ---------------------------------------------------------------------------
def reference_lib():
    path = os.path.join(ROOT, "oracle", "_ref", "libshhd_ref.so")
    if not os.path.exists(path):
        return None
    lib = ctypes.CDLL(path)
    lib.shref_create.restype = ctypes.c_void_p
    lib.shref_last_error.restype = ctypes.c_char_p
    lib.shref_time_steps.restype = ctypes.c_double
    lib.shref_threads.restype = ctypes.c_int
    return lib


def time_reference(nsteps_max: int, budget_s: float):
    """Time the reference's own step on the workload; returns (steps/s, steps, cores, kind, note)."""
    lib = reference_lib()
    if lib is not None:
        h = ctypes.c_void_p(lib.shref_create(WORKLOAD.encode()))
        if not h.value:
            raise RuntimeError(lib.shref_last_error().decode())
        first = lib.shref_time_steps(h, 1)
        n = max(1, min(nsteps_max, int(budget_s / max(first, 1e-3))))
        t = lib.shref_time_steps(h, n)
        cores = lib.shref_threads()
        lib.shref_destroy(h)
        return n / t, n, cores, "reference", "reference src .cc files (unmodified) on single-rank MPI/heFFTe shims, threaded shim FFT"
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import shhd_oracle as so
    import shhd_b200 as sb
    from shhd_b200.initial import initial_state
    cfg = so.parse_script(WORKLOAD)
    o = so.Oracle(cfg)
    u = initial_state(sb.config_from_script(WORKLOAD), WORKLOAD)
    t0 = time.perf_counter()
    u = o.step(u, "philox")
    t = time.perf_counter() - t0
    return 1.0 / t, 1, 1, "port", "numpy FP64 restatement (reference checker not built)"


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------
def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return
    budget = float(os.environ.get("SHHD_REF_BUDGET_S", "120"))
    # warm-up steps (untimed), then the timed steps, capped to a bounded sample
    lib = reference_lib()
    if lib is None:
        sps, n, cores, kind, note = time_reference(args.steps, budget)
    else:
        h = ctypes.c_void_p(lib.shref_create(WORKLOAD.encode()))
        if not h.value:
            print(json.dumps({"impl": "reference", "unavailable": lib.shref_last_error().decode()}))
            return
        first = lib.shref_time_steps(h, 1)
        wsteps = max(0, min(args.warmup - 1, int(0.25 * budget / max(first, 1e-3))))
        if wsteps:
            lib.shref_time_steps(h, wsteps)
        n = max(1, min(args.steps, int(budget / max(first, 1e-3))))
        t = lib.shref_time_steps(h, n)
        cores = lib.shref_threads()
        lib.shref_destroy(h)
        sps, kind = n / t, "reference"
        note = "reference src .cc files (unmodified) on single-rank MPI/heFFTe shims, threaded shim FFT"
    sample = f"{n} SRK3 steps of the 1024^2 N=2 workload ({note})"
    line = {
        "metric": METRIC, "value": sps, "unit": UNIT, "impl": "reference", "n_gpus": world, "steps": n, "warmup": args.warmup,
        "ms_per_step": 1e3 / sps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": CONFIG,
        "cpu_baseline": {"value": sps, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": sps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def dram_traffic_from_profiles(workload: str):
    """Per-launch DRAM bytes of each kernel on `workload` from the committed ncu summary (lines
    'kernel workload bytes'), if present."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    out = {}
    if os.path.exists(path):
        for line in open(path):
            t = line.split("#", 1)[0].split()
            if len(t) == 3 and t[1] == workload:
                try:
                    out[t[0]] = float(t[2])
                except ValueError:
                    pass
    return out


def measured_peak_gbs():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        try:
            return float(json.load(open(path))["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def run_b200(args):
    import numpy as np
    import torch

    world, rank, local = dist_setup()
    dist = init_group(world, local, "nccl")
    torch.cuda.set_device(local)
    import shhd_b200 as sb
    from shhd_b200.initial import initial_state

    cfg = sb.config_from_script(WORKLOAD)
    cfg.precision = sb.FP32 if args.precision == "fp32" else sb.FP64
    cfg.member_offset = rank
    u0 = initial_state(cfg, WORKLOAD)
    eng = sb.Engine(cfg)
    eng.set_state(u0)
    stream = torch.cuda.ExternalStream(eng.stream)
    # kernel family and graph replay chosen by timing them on this state (state restored), or the
    # family given on the command line (profiling one family); trials of 10 steps, the graph chunk
    # a long run would replay
    if args.family is None:
        tuning = eng.autotune(10)
    else:
        eng.set_family(args.family)
        tuning = {"family": sb.FAMILY_NAMES[eng.family], "graph_chunk": 0, "forced": True}

    # warm-up
    eng.step(args.warmup)

    props = torch.cuda.get_device_properties(local)
    uuid = "GPU-" + str(getattr(props, "uuid", "")) if getattr(props, "uuid", None) else ""
    clocks = ClockSampler(uuid)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    eng.reset_stats()
    ev0.record(stream)
    eng.step_async(args.steps)
    ev1.record(stream)
    eng.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    stats = eng.kernel_stats()
    launches = int(sum(v[1] for v in stats.values()))
    ms_max = max_over_ranks(ms, world)
    value = world * args.steps / (ms_max / 1e3)

    # per-kernel device time (CUDA events around each launch on the engine stream)
    kprof_steps = max(10, min(args.steps, 100))
    eng.reset_stats()
    eng.set_profiling(True)
    eng.step(kprof_steps)
    eng.set_profiling(False)
    kst = eng.kernel_stats()
    dom = max(("row_pass", "col_forward"), key=lambda k: kst[k][0])
    t_ms, n_l, by = kst[dom]
    achieved = (by / n_l) / (t_ms / n_l * 1e-3) / 1e9
    peak, peak_kind = measured_peak_gbs()
    # the summary holds the pair-line kernels' capture; another family has no captured traffic
    # the committed capture covers the FP32 engine with the family it timed (hh1024_fp32_f<family>)
    traffic = dram_traffic_from_profiles(f"hh1024_fp32_f{eng.family}").get(dom) if args.precision == "fp32" else None
    step_bytes = sum(v[2] for v in kst.values()) / kprof_steps
    step_ms_profiled = sum(v[0] for v in kst.values()) / kprof_steps
    kernels = {k: {"ms_per_launch": (v[0] / v[1]) if v[1] else None, "launches_per_step": v[1] / kprof_steps,
                   "GBps": ((v[2] / v[1]) / (v[0] / v[1] * 1e-3) / 1e9) if v[1] and v[0] > 0 else None} for k, v in kst.items() if v[1]}

    # e2e: host State (pinned) -> device, one step, device -> host State, every step
    e2e_steps = max(3, min(args.steps, 20))
    shape = eng.shape
    nbytes = int(np.prod(shape)) * 16
    hin_t = torch.empty(nbytes // 8, dtype=torch.float64, pin_memory=True)
    hout_t = torch.empty(nbytes // 8, dtype=torch.float64, pin_memory=True)
    hin = hin_t.numpy().view(np.complex128).reshape(shape)
    hout = hout_t.numpy().view(np.complex128).reshape(shape)
    eng.get_state(out=hin)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        eng.set_state(hin)
        eng.step(1)
        eng.get_state(out=hout)
        hin, hout = hout, hin
    t_e2e = time.perf_counter() - t0
    t_e2e = max_over_ranks(t_e2e, world)
    e2e_value = world * e2e_steps / t_e2e
    # resident variant: state stays on the device, one host call for many steps
    t0 = time.perf_counter()
    eng.set_state(hin)
    eng.step(args.steps)
    eng.get_state(out=hout)
    t_res = max_over_ranks(time.perf_counter() - t0, world)
    resident_value = world * args.steps / t_res
    eng.close()

    extras = {}
    if not args.no_extras:
        extras = run_extras(args, world, rank, local, sb, initial_state, torch)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sps, n, cores, kind, note = time_reference(5, float(os.environ.get("SHHD_CPU_BASELINE_S", "20")))
        cpu = {"value": sps, "unit": UNIT, "cores": cores, "kind": kind,
               "sample": f"{n} SRK3 steps of the same 1024^2 N=2 workload ({note})"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "fp32" else "f64", "data": "synthetic", "config": dict(CONFIG, parallelism=f"replicas x{world}"),
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "traffic_source": "profiles/dram_traffic.txt (ncu dram__bytes_read.sum + dram__bytes_write.sum, mean per launch)",
                         "algorithmic_bytes_per_launch": by / n_l, "step_GBps": step_bytes / (step_ms_profiled * 1e-3) / 1e9},
            "kernels": kernels,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                    "what": "set_state(host pinned) + step(1) + get_state(host) through the C ABI every step"},
            "e2e_resident": {"value": resident_value, "unit": UNIT, "what": f"set_state + step({args.steps}) + get_state, one host call"},
            "gpu_launches": launches,
            "warnings": ([] if peak_kind == "measured" else
                         [f"MEASURED_PEAKS.json absent: roofline.peak is the fallback {peak:.0f} GB/s, not a measured peak"]),
            "clocks": clk,
            "autotune": tuning,
        }
        line.update(extras)
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def run_measures(sb, torch, world):
    """The device measures on the headline workload (1024^2, N = 2, FP32): wall time of one call
    (launches, FP64 reduction, read-back), and the step rate with the per-stage flux taps on."""
    import time as _time
    from shhd_b200.initial import initial_state_device
    cfg = sb.config_from_script(WORKLOAD)
    cfg.precision = sb.FP32
    eng = sb.Engine(cfg)
    initial_state_device(eng, WORKLOAD)
    eng.step(2)

    def wall_ms(fn, reps=5):
        fn()
        t0 = _time.perf_counter()
        for _ in range(reps):
            fn()
        return (_time.perf_counter() - t0) / reps * 1e3

    def rate(n=30):
        stream = torch.cuda.ExternalStream(eng.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        eng.step(3)
        eng.synchronize()
        e0.record(stream)
        eng.step_async(n)
        e1.record(stream)
        eng.synchronize()
        return world * n / (max_over_ranks(e0.elapsed_time(e1), world) / 1e3)

    out = {"energies_ms": wall_ms(eng.time_series_energies), "l2_ms": wall_ms(eng.time_series_l2),
           "profile_line_ms": wall_ms(lambda: eng.profile_line(0, 1)), "profile_velocity_x_ms": wall_ms(lambda: eng.profile_velocity(0, 0)),
           "steps_per_s_plain": rate()}
    eng.flux0_enable()
    out["steps_per_s_with_k0_flux_tap"] = rate()
    eng.flux_line_enable(1)
    out["steps_per_s_with_k0_and_flux_line_y_taps"] = rate()
    out["flux_line_read_ms"] = wall_ms(lambda: eng.flux_line(1))
    eng.flux_tap_schedule(0, 10, 0)
    eng.flux_tap_schedule(2, 10, 0)
    out["steps_per_s_with_both_taps_every_10_steps"] = rate()
    out["what"] = ("1024^2 (3/2 -> 1536^2), N = 2, FP32 engine: wall time per measure call (E_T..E_C with the physical-space "
                   "transforms; L2 columns; one spectral profile line; the compressible vx profile over x); step rate "
                   "without taps, with the k = 0 flux tap, with the kx = 0 flux-line tap added (1535 modes, every flux), and with both "
                   "taps recording every 10th step (a measure sampling every 10 steps)")
    eng.close()
    return out


def run_extras(args, world, rank, local, sb, initial_state, torch):
    out = {}
    # the plain one-job-at-a-time FP64 path on the same workload
    cfg = sb.config_from_script(WORKLOAD)
    cfg.precision = sb.FP64
    cfg.member_offset = rank
    eng = sb.Engine(cfg)
    eng.set_state(initial_state(cfg, WORKLOAD))
    eng.step(2)
    n64 = max(3, min(args.steps, 50))
    stream = torch.cuda.ExternalStream(eng.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    eng.step_async(n64)
    e1.record(stream)
    eng.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    out["fp64_plain"] = {"value": world * n64 / (ms / 1e3), "unit": UNIT, "steps": n64}
    eng.close()

    out["measures"] = run_measures(sb, torch, world)

    # batched ensemble: 256 members advanced together
    cfg = sb.config_from_script(ENSEMBLE)
    cfg.precision = sb.FP32
    cfg.batch = 256
    cfg.member_offset = rank * 256
    eng = sb.Engine(cfg)
    from shhd_b200.initial import initial_state_device
    for m in range(cfg.batch):
        # member m: seed m (the ensemble draws psi0 per member seed), generated on the device
        initial_state_device(eng, ENSEMBLE.replace("all equilibrium/gaussian seed 0 ", f"all equilibrium/gaussian seed {m} "), member=m)
    # kernel family, graph chunk and launch shapes timed on the ensemble itself (state restored)
    ens_tuning = eng.autotune(10)
    eng.step(2)
    nb = max(3, min(args.steps, 50))
    stream = torch.cuda.ExternalStream(eng.stream)
    e0.record(stream)
    eng.step_async(nb)
    e1.record(stream)
    eng.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    gbs, frac, kind = roofline_fraction(eng, nb / (ms / 1e3))
    out["batched"] = {"value": world * nb * cfg.batch / (ms / 1e3), "unit": "member-steps/s", "members": cfg.batch * world,
                      "ensemble_steps_per_s": world * nb / (ms / 1e3) / world, "workload": "256 x 256^2 (3/2), quiescent N=1 phi4, SRK3, FP32",
                      "algorithmic_GBps": gbs, "frac_of_hbm": frac, "peak_kind": kind, "autotune": ens_tuning}
    # the plain path for the same members: one member at a time, FP64, each its own engine (batch 1)
    c1 = sb.config_from_script(ENSEMBLE)
    c1.precision = sb.FP64
    c1.member_offset = rank * 256
    n_plain_members, n1 = 8, max(3, min(args.steps, 50))
    t_plain = 0.0
    for m in range(n_plain_members):
        with sb.Engine(c1) as one:
            initial_state_device(one, ENSEMBLE.replace("all equilibrium/gaussian seed 0 ", f"all equilibrium/gaussian seed {m} "))
            one.step(2)
            s1 = torch.cuda.ExternalStream(one.stream)
            a1, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a1.record(s1)
            one.step_async(n1)
            b1.record(s1)
            one.synchronize()
            t_plain += a1.elapsed_time(b1) / 1e3
    plain = n_plain_members * n1 / t_plain
    out["batched"]["plain_fp64_member_steps_per_s"] = plain
    out["batched"]["over_plain_fp64"] = out["batched"]["value"] / (world * plain)
    out["batched"]["plain_what"] = (f"{n_plain_members} of the members one at a time through the plain FP64 path (batch-1 engine each, "
                                    f"{n1} SRK3 steps, device time per member summed)")
    # structure factor of psi over the members (FP64 on the device), summed over ranks by one all-reduce
    from shhd_b200.ensemble import reduce_structure_factor
    for _ in range(4):
        eng.step(5)
        eng.sk_accumulate(1)
    sk_sum, nsamp = eng.sk_read()
    sk_mean, total_members = reduce_structure_factor(sk_sum, nsamp, cfg.batch, device="cuda" if world > 1 else None)
    out["batched"]["structure_factor"] = {"members": total_members, "samples": nsamp, "mean_over_modes": float(sk_mean.mean()),
                                          "what": "S(k) = V <|psi_k|^2> / Np^4, FP64 member mean per rank, FP64 all-reduce over ranks"}
    eng.close()

    out["served"] = run_served(sb, initial_state, torch)
    out["other_configs"] = run_other_configs(sb, initial_state, torch, world)

    # cuFFT beside it: the same transforms per stage (5 C2R + 11 R2C at 1536^2, FP32)
    x = torch.randn(11, 1536, 1536, device="cuda", dtype=torch.float32)
    X = torch.fft.rfft2(x[:5])
    for _ in range(3):
        torch.fft.irfft2(X, s=(1536, 1536))
        torch.fft.rfft2(x)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(10):
        torch.fft.irfft2(X, s=(1536, 1536))
        torch.fft.rfft2(x)
    e1.record()
    torch.cuda.synchronize()
    ms_stage = e0.elapsed_time(e1) / 10
    out["cufft_reference"] = {"ms_per_stage": ms_stage, "steps_per_s_transforms_only": 1e3 / (3 * ms_stage),
                              "what": "torch.fft (cuFFT) 5 irfft2 + 11 rfft2 at 1536^2 FP32 per stage, unfused, no products or RHS"}
    return out


# ---------------------------------------------------------------------------
# the other single-trajectory configurations, timed as reference points
# ---------------------------------------------------------------------------
PLAIN_128 = """dimension 2
grid 128 128
length 128 128
dealias 3/2
order_parameters 0
timestep 0.05
time_evolution srk3/compressible
model thermo linear_eos cT 1
model transport constant eta 1 zeta 1
fix 1 all nonlinear on
fix 2 all noise on seed 1 kBT 1e-4
set density equilibrium/gaussian kBT 1e-4 rho0 1 cT 1 seed 1
set momentum all equilibrium/gaussian/compressible kBT 1e-4 seed 1
run 2000
"""

TURB_4096 = """dimension 2
grid 4096 4096
length 4096 4096
dealias 3/2
order_parameters 0
timestep 0.001
time_evolution srk3/incompressible
model transport constant eta 1e-4 zeta 0
fix 1 momentum nonlinear on
fix 2 all noise on seed 11 kBT 1e-6
set density uniform value 1.0
set momentum all random_vorticity n0 8 sigma 2 urms 1 seed 11
run 2000
"""


def roofline_fraction(eng, steps_per_s):
    """Algorithmic HBM bytes per step (the engine's per-stage count x stages) x steps/s against the
    measured copy bandwidth: (GB/s, fraction, the peak's kind)."""
    info = eng.get_info()
    stages = 3 if eng.cfg.integrator == 1 else 1
    gbs = info.bytes_per_stage * stages * steps_per_s / 1e9
    peak, kind = measured_peak_gbs()
    return gbs, gbs / peak, kind


def run_other_configs(sb, initial_state, torch, world):
    out = {}
    for name, text, prec, nsteps, what in (
            ("plain_128_fp64", PLAIN_128, sb.FP64, 200,
             "128^2 (3/2 -> 192^2), N=0 compressible, linear EOS, eta = zeta = 1, kBT 1e-4, equilibrium ICs seed 1, SRK3 dt 0.05, FP64"),
            ("turbulence_4096_fp32", TURB_4096, sb.FP32, 5,
             "4096^2 (3/2 -> 6144^2), N=0 incompressible, eta 1e-4, advection, kBT 1e-6, SRK3 dt 1e-3, FP32; random-vorticity "
             "initial momentum (n0 8, sigma 2, urms 1, seed 11) generated on the device")):
        from shhd_b200.initial import initial_state_device
        cfg = sb.config_from_script(text)
        cfg.precision = prec
        eng = sb.Engine(cfg)
        initial_state_device(eng, text)
        tuning = eng.autotune(10) if nsteps > 50 else None
        eng.step(3)
        stream = torch.cuda.ExternalStream(eng.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.step_async(nsteps)
        e1.record(stream)
        eng.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), world)
        rate = world * nsteps / (ms / 1e3)
        gbs, frac, kind = roofline_fraction(eng, rate / world)
        out[name] = {"value": rate, "unit": "steps/s", "steps": nsteps, "what": what, "autotune": tuning,
                     "algorithmic_GBps": gbs, "frac_of_hbm": frac, "peak_kind": kind}
        eng.close()
    return out


# ---------------------------------------------------------------------------
# served stream: Poisson arrivals of mixed trajectory jobs
# ---------------------------------------------------------------------------
SERVED = {"jobs": 24, "rate_per_s": 20.0, "grids": (128, 256, 512, 1024), "steps": (25, 500), "seed": 5, "green_kubo": (10, 100),
          "what": "Poisson arrivals (20 jobs/s, seed 5) of trajectory jobs drawn uniformly from grids {128,256,512,1024}^2 "
                  "(3/2 rule, spacing 2; the configured 2048^2 is left out because the plain FP64 path's 3072-point row pass "
                  "holds every input line in shared memory and cannot run compressible jobs with order parameters there), "
                  "N in {0..3}, mode in {compressible, incompressible, quiescent}, kBT in [1e-4, 1e-2]; "
                  "the served configuration's distributions with each job's 10^3-2x10^4 SRK3 steps scaled by 1/40 (25-500 steps) so "
                  "the stream finishes in seconds; every non-quiescent job accumulates the Yokota-Green-Kubo stress measure "
                  "(diagonal modes, every 10 steps, blocks of 100) in FP64, in the server and in the serial FP64 baseline alike; "
                  "one server serves a warm-up pass (untimed; it creates the bucket engines, as the baseline's engine creation "
                  "is untimed), then the capacity run and the Poisson run"}


def served_job_scripts():
    """(arrival time, script, steps) of the seeded served-stream sample."""
    import numpy as np
    rng = np.random.default_rng(SERVED["seed"])
    t = 0.0
    out = []
    for _ in range(SERVED["jobs"]):
        t += rng.exponential(1.0 / SERVED["rate_per_s"])
        na = int(rng.choice(SERVED["grids"]))
        mode = str(rng.choice(["compressible", "incompressible", "quiescent"]))
        nop = int(rng.integers(0, 4))
        if mode == "quiescent" and nop == 0:
            nop = 1
        kbt = float(rng.uniform(1e-4, 1e-2))
        nsteps = int(rng.integers(SERVED["steps"][0], SERVED["steps"][1] + 1))
        lines = ["dimension 2", f"grid {na} {na}", f"length {2 * na} {2 * na}", "dealias 3/2", f"order_parameters {nop}", "timestep 0.01",
                 f"time_evolution srk3/{mode}"]
        if mode == "compressible":
            lines.append("model thermo linear_eos cT 1")
        if nop:
            lines.append("model free_energy phi4 " + " ".join(f"a[{a}] -1 b[{a}] 1 u[{a}] 1" for a in range(nop)))
        eta = {"compressible": 1.0, "incompressible": 0.1, "quiescent": 0.0}[mode]
        zeta = 1.0 if mode == "compressible" else 0.0
        lines.append(f"model transport constant eta {eta} zeta {zeta} " + " ".join(f"M[{a},{a}] 1" for a in range(nop)))
        if mode != "quiescent":
            lines.append("fix 1 all nonlinear on")
        lines.append(f"fix 2 all noise on seed 1 kBT {kbt}")
        lines.append("set density uniform value 1.0")
        if nop:
            lines.append("set order_parameter all equilibrium/gaussian seed 3 kBT 0.0001 k0 1 k2 0")
        lines.append(f"run {nsteps}")
        out.append((t, "\n".join(lines) + "\n", nsteps, mode != "quiescent"))
    return out


def run_served(sb, initial_state, torch):
    from shhd_b200 import serve
    specs = served_job_scripts()
    jobs = []
    for k, (t, text, n, gk) in enumerate(specs):
        cfg = sb.config_from_script(text)
        jobs.append(serve.Job(key=100 + k, config=cfg, state=initial_state(cfg, text), nsteps=n, arrival=t,
                              green_kubo=SERVED["green_kubo"] if gk else None))
    total_steps = sum(j.nsteps for j in jobs)
    # one server kept warm across the runs, as a serving process is: the untimed warm-up (every job
    # configuration once, 50 steps) creates its bucket engines and captures their graphs, as the
    # FP64 baseline below creates its engines and warms up untimed
    warm = [serve.Job(key=j.key, config=j.config, state=j.state, nsteps=50, arrival=0.0, green_kubo=j.green_kubo) for j in jobs]
    srv = serve.Server(precision=sb.FP32, seed=77, max_slots=8, chunk=25)
    srv.run(warm)
    # capacity: the jobs all present at t = 0
    sat_jobs = [serve.Job(key=j.key, config=j.config, state=j.state, nsteps=j.nsteps, arrival=0.0, green_kubo=j.green_kubo) for j in jobs]
    sat = srv.run(sat_jobs)
    # latency under Poisson arrivals (its throughput is bounded by the arrivals)
    stats = srv.run(jobs)
    srv.close()
    # the same jobs one at a time through the plain FP64 path (engine creation not timed), after an
    # untimed warm-up of every job configuration
    seen = set()
    for j in jobs:
        key = serve.bucket_key(j.config, j.green_kubo)
        if key in seen:
            continue
        seen.add(key)
        c = j.config.copy()
        c.precision = sb.FP64
        with sb.Engine(c) as eng:
            if j.green_kubo is not None:
                eng.gk_enable(*j.green_kubo)
            eng.set_state(j.state)
            eng.step(3)
    t_serial = 0.0
    for j in jobs:
        c = j.config.copy()
        c.precision = sb.FP64
        with sb.Engine(c) as eng:
            if j.green_kubo is not None:
                eng.gk_enable(*j.green_kubo)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            eng.set_state(j.state)
            eng.step(j.nsteps)
            eng.get_state()
            if j.green_kubo is not None:
                eng.gk_read()
            t_serial += time.perf_counter() - t0
    serial = total_steps / t_serial
    return {"value": stats["steps_per_s"], "unit": "steps/s (aggregate over jobs)", "p50_s": stats["p50_s"], "p99_s": stats["p99_s"],
            "makespan_s": stats["makespan_s"], "jobs": stats["jobs"], "buckets": stats["buckets"], "total_steps": total_steps,
            "precision": "f32", "plain_fp64_serial_steps_per_s": serial, "served_over_plain_fp64": stats["steps_per_s"] / serial,
            "saturated": {"steps_per_s": sat["steps_per_s"], "p50_s": sat["p50_s"], "p99_s": sat["p99_s"], "makespan_s": sat["makespan_s"],
                          "over_plain_fp64": sat["steps_per_s"] / serial,
                          "what": "the same jobs all arriving at t = 0: serving capacity (the Poisson run is bounded by its arrivals)"},
            "what": SERVED["what"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--precision", choices=("fp32", "fp64"), default="fp32")
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--family", type=int, choices=(0, 1, 2, 3, 4), default=None,
                    help="kernel family instead of the autotuner's choice (0 single-line, 1 pair-line, 2 register row pass, "
                         "3 split row pass, 4 two-pair row pass)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if launch_plan(args.gpus, os.environ) == "spawn":
        import socket
        with socket.socket() as s:
            s.bind(("127.0.0.1", 0))
            port = s.getsockname()[1]
        raise SystemExit(subprocess.call(spawn_command(sys.argv[1:], args.gpus, port)))
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
