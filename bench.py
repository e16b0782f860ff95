"""Benchmark of the firesim-b200 frame pipeline (one JSON line on rank 0).

Workload: the reference's per-frame pipeline (native-firesim's physics, its
ten transported scalars on a MAC grid) on a 128x128x128 grid in FP32, with the
128^3 configuration's solver and render cadence: 60 red-black SOR iterations
at omega 1.8, and one 512x512 HDR raymarch every 10 steps (128 primary samples
requested; the reference ABI clamps them to 120).  Settings are the
reference's validation-harness frames (scene 0, canonical constants), the
scene is reset on the first warm-up step, and the fire develops during the
timed steps.  A "step" is one call of the reference ABI: fireCudaStepD3D11,
or fireCudaStepAndRenderD3D11 on every 10th step (render into a device HDR
buffer).

value  : voxel-steps/s over all ranks, device-timed with CUDA events on the
         scene's own stream, inputs resident in HBM (the per-step state,
         ~270 MB at 128^3, exceeds the 126 MB L2).
e2e    : the same metric through the host path: fireCudaStepD3D11 and, every
         10th step, fireCudaStepAndRender with a host BGRA8 buffer (the frame
         is copied to the host inside the timed region), wall-clock timed.
N > 1  : replicas only -- every rank steps its own scene on its own GPU; the
         ranks meet only at the barriers and the max-reduction of the timings.

--impl reference times the CPU restatement of the reference's step
(OpenMP, all host threads) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def load_package():
    if "firesim_b200" in sys.modules:
        return sys.modules["firesim_b200"]
    pkg_dir = ROOT / "native-firesim_b200"
    spec = importlib.util.spec_from_file_location("firesim_b200", pkg_dir / "__init__.py",
                                                  submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["firesim_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_peaks() -> tuple[dict, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return PEAKS_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self._thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._thread = threading.Thread(target=self._read, daemon=True)
            self._thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl" if os.environ.get("FIRESIM_BENCH_BACKEND", "nccl") == "nccl" else "gloo",
                                timeout=__import__("datetime").timedelta(seconds=120))
    return world, rank, local


def dist_max(x: float, world: int) -> float:
    """The maximum of x over the ranks (a device tensor under NCCL, a host tensor under gloo)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def workload_settings(abi, frame: int, args) -> object:
    s = abi.validation_settings(frame, scene=0, width=args.frame, height=args.frame)
    s.raymarchSteps = args.samples
    s.reset = 1 if frame == 0 else 0
    return s


# Algorithmic bytes per cell of each timed stage (FP32 layout of this library):
# scalars 40 B/cell packed, three face grids ~12 B/cell, p/div 4 B each.
STAGE_BYTES_PER_CELL = {
    "advect_velocity": 24.0,          # read 3 faces + write 3 faces (velocity gathers hit L1/L2)
    "advect_react": 40.0 * 2 + 12.0,  # read + write the 10 scalars, read the 3 faces
    "force_project": 16.0 + 12.0 * 2 + 16.0 + 8.0,  # read heat/soot/k/progress, read+write faces, force scratch w+r, div+p
    "pressure_sor": 6.0,              # per half sweep: 12 B/cell per iteration (read p, write p, read div)
    "subtract_walls": 4.0 + 24.0,     # read p, read+write faces
    "light": 0.0,                     # quarter-resolution grid, small
}


def stage_timings(pkg, sim, args, settings, iters: int = 3) -> dict:
    """Device time of each stage range (best of `iters`), from CUDA events on the scene stream
    around the queued stages."""
    import torch
    ext = torch.cuda.ExternalStream(sim.stream())
    ranges = {
        "advect_velocity": ("advect_velocity", "advect_velocity"),
        "advect_react": ("advect_react", "advect_react"),
        "force_project": ("force", "divergence"),
        "pressure_sor": ("pressure_sor", "pressure_sor"),
        "subtract_walls": ("subtract", "wall_boundary"),
        "light": ("light_build", "light_propagate"),
        "render": ("render", "render"),
        "embers": ("embers", "embers"),
    }
    t_sim, t_render, _ = sim.times()
    out = {}
    for name, (a, b) in ranges.items():
        ms = []
        for _ in range(iters):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            # A spin kernel holds the stream while the host queues the events and the
            # stage, so the interval holds the stage's kernels and not the host's latency.
            with torch.cuda.stream(ext):
                torch.cuda._sleep(400_000)
            e0.record(ext)
            sim.stages(a, b, settings, t_render if name in ("render", "embers") else t_sim, wait=False)
            e1.record(ext)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        sim.synchronize()
        out[name] = min(ms)
    return out


def cpu_baseline(pkg, args, n_sim_steps: int = 2, warmup: int = 1) -> dict:
    """The CPU restatement (OpenMP, all host threads) on a bounded sample of the workload:
    `warmup` untimed steps (the first resets the scene), then `n_sim_steps` timed steps."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as om  # noqa: PLC0415
    abi = pkg.abi
    o = om.OracleFire(abi, args.frame, args.frame, args.grid, args.grid, args.grid)
    o.set_pressure_solver(args.sor_iters, args.omega)
    threads = os.cpu_count() or 1
    om.OracleFire.set_threads(threads)
    for f in range(warmup):
        o.step(workload_settings(abi, f, args), mode=2)  # frame 0 resets the scene
    t0 = time.perf_counter()
    for f in range(warmup, warmup + n_sim_steps):
        o.step(workload_settings(abi, f, args), mode=2)
    t_sim = (time.perf_counter() - t0) / n_sim_steps
    t1 = time.perf_counter()
    o.step(workload_settings(abi, warmup + n_sim_steps, args), mode=3)
    t_render = time.perf_counter() - t1
    per_step = t_sim + t_render / args.render_every
    cells = args.grid ** 3
    return {"value": cells / per_step, "unit": "voxel-steps/s", "cores": threads, "kind": "port",
            "sample": f"{n_sim_steps} simulation steps of the {args.grid}^3 workload after {warmup} warm-up step(s) "
                      f"(the first resets the scene), plus one {args.frame}^2 render amortised over {args.render_every} steps",
            "seconds_per_step": per_step}


def run_reference(args, world: int, rank: int) -> None:
    if rank != 0:
        return
    pkg = load_package()
    # K timed steps, at most --reference-steps of them, after W warm-up steps (at most 10):
    # a 128^3 step of the CPU restatement takes about 0.4 s on 16 threads.
    steps = max(1, min(args.steps, args.reference_steps))
    warmup = max(1, min(args.warmup, 10))
    cb = cpu_baseline(pkg, args, n_sim_steps=steps, warmup=warmup)
    line = {
        "impl": "reference", "metric": "voxel-steps/s", "value": cb["value"], "unit": "voxel-steps/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": warmup, "ms_per_step": cb["seconds_per_step"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_block(args),
        "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": cb["value"], "unit": "voxel-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_block(args) -> dict:
    return {"workload": f"reference frame pipeline (native-firesim physics, 10 scalars, MAC velocity), FP32, "
                        f"{args.grid}^3 grid, SOR {args.sor_iters} iterations omega {args.omega}, "
                        f"{args.precision.upper() + ' storage, ' if args.precision != 'f32' else ''}"
                        f"{args.frame}x{args.frame} HDR raymarch every {args.render_every} steps "
                        f"({args.samples} samples requested, clamped to 120)",
            "grid": [args.grid] * 3, "frame": [args.frame, args.frame], "sor_iterations": args.sor_iters,
            "omega": args.omega, "sor_path": args.sor_path, "render_every": args.render_every,
            "settings": "validation harness frames, scene 0",
            "l2": "per-step state (~270 MB at 128^3) exceeds the 126 MB L2; no flush", "parallelism": "replicas"}


class SplitMix64:
    """SplitMix64 (Steele, Lea, Flood 2014): the host RNG of the batched and serving draws."""

    def __init__(self, seed: int):
        self.state = seed & 0xFFFFFFFFFFFFFFFF

    def next(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        return z ^ (z >> 31)

    def uniform(self, lo: float = 0.0, hi: float = 1.0) -> float:
        return lo + (hi - lo) * (self.next() >> 11) * (1.0 / (1 << 53))

    def normal(self) -> float:
        u1, u2 = max(self.uniform(), 1e-300), self.uniform()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)


def scene_settings(abi, rng: SplitMix64, dims, frame_w: int, frame_h: int, radius_cells: tuple, wind: float):
    """Per-scene settings of the batched and serving mixes on the reference's physics:
    validation-harness settings with the emitter centre drawn in the middle half of
    the floor, its radius drawn in cells (converted to the 2.1 m wide domain) and
    the wind drawn per scene (the reference's wind acts along x only)."""
    nx = dims[0]
    s = abi.validation_settings(1, scene=0, width=frame_w, height=frame_h)
    s.reset = 0
    s.emitterCenterX = rng.uniform(-0.25, 0.25) * 2.10
    s.emitterCenterZ = rng.uniform(-0.25, 0.25) * 1.64
    s.emitterRadius = rng.uniform(*radius_cells) / nx * 2.10
    s.wind = wind
    return s


def config_scene_physics(abi, rng: SplitMix64, dims, seed: int, lib):
    """A batched or served scene of the config physics: emitter centre uniform in
    the middle half of the floor, radius U[4, 12] cells (at most a quarter of the
    smaller floor edge), wind U[-0.5, 0.5] on x and on z, jitter seed `seed`."""
    nx, ny, nz = dims
    cx = rng.uniform(0.25, 0.75) * nx
    cz = rng.uniform(0.25, 0.75) * nz
    r = min(rng.uniform(4.0, 12.0), 0.25 * min(nx, nz))
    return abi.config_scene(nx, ny, nz, cx, cz, r, rng.uniform(-0.5, 0.5), rng.uniform(-0.5, 0.5), seed, lib)


def run_batched(args, pkg, emit: bool = True) -> dict:
    """48 independent scenes of mixed sizes stepped together: one FireBatch for
    the config physics with the multigrid projection, else fireBatchStep."""
    import torch
    abi = pkg.abi
    config = args.physics == "config"
    precision = args.precision if args.precision_set or not config else "f16"
    lib = pkg.load_library(precision)
    rng = SplitMix64(11)
    sizes = [(48, 48, 48), (64, 64, 64), (96, 96, 96), (128, 64, 64), (160, 96, 96)]
    dims = [sizes[rng.next() % len(sizes)] for _ in range(args.scenes)]
    scenes, settings, hdrs = [], [], []
    for i, d in enumerate(dims):
        sc = pkg.Scene(256, 256, *d, precision=precision)
        sc.set_pressure_solver(40, 1.8)
        hdr = torch.zeros((256, 256, 4), dtype=torch.float32, device="cuda")
        sc.set_hdr_buffer(hdr.data_ptr(), 256 * 16, 0)
        scenes.append(sc)
        hdrs.append(hdr)
        if config:
            phys = config_scene_physics(abi, rng, d, 1000 + i, lib)
            if args.solver == "mg":
                phys.pressureTop = 1
            sc.set_physics(phys)
            if args.solver == "mg":
                sc.set_pressure_multigrid(args.mg_cycles, args.mg_pre, args.mg_post)
                sc.set_pressure_tolerance(0.5 * args.div_target, 1)
            s = abi.FireSettings(width=256, height=256, dt=1.0 / 60.0)
        else:
            s = scene_settings(abi, rng, d, 256, 256, (4.0, 12.0), rng.uniform(-0.5, 0.5))
            s.raymarchSteps = 64
        settings.append(s)
    voxels = sum(int(np.prod(d)) for d in dims)
    # The config physics with the multigrid projection runs as one FireBatch
    # (one launch per stage over every scene); otherwise fireBatchStep queues
    # each scene's own launches on its own stream.
    batch = pkg.Batch(scenes) if config and args.solver == "mg" else None

    def sub_step(i):
        for s in settings:
            s.reset = 1 if i == 0 else 0
        render = [(i % args.render_every) == args.render_every - 1] * len(scenes)
        if batch is not None:
            batch.run(settings, render=render)
        else:
            pkg.batch_step(scenes, settings, render=render)

    def sync_all():
        if batch is not None:
            batch.synchronize()
        for sc in scenes:
            sc.synchronize()

    for i in range(args.warmup):
        sub_step(i)
    sync_all()
    torch.cuda.synchronize()
    launches0 = batch.launch_count() if batch is not None else None
    t0 = time.perf_counter()
    for i in range(args.warmup, args.warmup + args.steps):
        sub_step(i)
    sync_all()
    wall = time.perf_counter() - t0
    stats = [sc.pressure_stats() for sc in scenes] if config and args.solver == "mg" else []
    line = {"metric": "voxel-steps/s", "mode": "batched", "value": voxels * args.steps / wall, "unit": "voxel-steps/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_sub_step": wall * 1e3 / args.steps,
            "higher_is_better": True, "dtype": precision, "data": "synthetic (SplitMix64 seed 11 draws)",
            "config": {"workload": f"{args.scenes} independent scenes, sizes drawn from {sizes}, "
                                   f"{'config physics (one disk emitter each, r U[4,12], wind U[-0.5,0.5]^2, seeds 1000+i)' if config else 'reference physics'}, "
                                   f"{precision} storage, "
                                   + (f"p = 0 on the top face, multigrid until max|r| <= {0.5 * args.div_target:g}, "
                                      if config and args.solver == "mg" else "SOR 40 iterations omega 1.8, ")
                                   + "256x256 render (64 samples) every "
                                   f"{args.render_every} steps, one fireBatchStep per sub-step, each scene on its own stream",
                       "voxels_per_sub_step": voxels, "timing": "host wall clock around the sub-steps, synchronised on all scenes",
                       "launch": "FireBatch: one launch per stage over all scenes" if batch is not None else
                                 "fireBatchStep: each scene's launches on its own stream"}}
    if batch is not None:
        line["gpu_launches"] = batch.launch_count() - launches0
    if stats:
        line["multigrid_last_sub_step"] = {"cycles_max": max(st[0] for st in stats), "cycles_mean": float(np.mean([st[0] for st in stats])),
                                           "max_residual": max(st[1] for st in stats)}
    if emit:
        print(json.dumps(line), flush=True)
    if batch is not None:
        batch.close()
    for sc in scenes:
        sc.close()
    return line


def run_serve(args, pkg, emit: bool = True) -> dict:
    """Poisson arrivals of scene requests into the FireServer loop."""
    abi = pkg.abi
    config = args.physics == "config"
    precision = args.precision if args.precision_set or not config else "bf16"
    lib = pkg.load_library(precision)
    rng = SplitMix64(args.seed)
    server = pkg.Server(budget_bytes=int(args.budget_gb * (1 << 30)), precision=precision)
    server.set_limits(int(args.max_active_mvoxels * 1e6))
    if args.latency_target_ms > 0:
        server.set_latency_target(args.latency_target_ms)
    t, n = 0.0, 0
    keep = []
    while True:
        t += -math.log(max(rng.uniform(), 1e-300)) / args.rate
        if t > args.arrival_seconds:
            break
        edge = int(round(min(192.0, max(32.0, 96.0 * math.exp(0.4 * rng.normal()))) / 16.0)) * 16
        r = abi.FireServeRequest()
        r.id = n
        r.nx = r.ny = r.nz = edge
        r.frameW = r.frameH = 256
        r.steps = 30 + int(rng.uniform() * 271)
        r.renderEvery = 4
        r.sorIterations, r.sorOmega = 40, 1.8
        r.arrivalSeconds = t
        if config:
            r.settings = abi.FireSettings(width=256, height=256, dt=1.0 / 60.0)
            r.physics = config_scene_physics(abi, rng, (edge, edge, edge), 5000 + n, lib)
            if args.solver == "mg":
                r.physics.pressureTop = 1
                r.multigridCycles, r.multigridPre, r.multigridPost = args.mg_cycles, args.mg_pre, args.mg_post
                r.pressureTolerance = 0.5 * args.div_target
        else:
            r.settings = scene_settings(abi, rng, (edge, edge, edge), 256, 256, (4.0, 12.0), rng.uniform(-0.5, 0.5))
            r.settings.raymarchSteps = 64
        server.submit(r)
        keep.append(r)
        n += 1
    rep = server.run(args.serve_seconds)
    server.close()
    line = {"metric": "voxel-steps/s", "mode": "serve", "value": rep["voxelSteps"] / max(rep["seconds"], 1e-9),
            "unit": "voxel-steps/s", "n_gpus": 1, "higher_is_better": True, "dtype": precision, "data": "synthetic (SplitMix64 draws)",
            "latency_ms": {"step_p50": rep["stepMsP50"], "step_p95": rep["stepMsP95"], "step_p99": rep["stepMsP99"],
                           "step_max": rep["stepMsMax"], "frame_p50": rep["frameMsP50"], "frame_p95": rep["frameMsP95"],
                           "frame_p99": rep["frameMsP99"], "queue_p50": rep["queueMsP50"], "queue_p99": rep["queueMsP99"]},
            "requests": {"submitted": rep["submitted"], "completed": rep["completed"], "admitted_peak": rep["admittedPeak"]},
            "device_bytes_peak": rep["deviceBytesPeak"], "seconds": rep["seconds"],
            "config": {"workload": f"Poisson arrivals at {args.rate}/s for {args.arrival_seconds} s; cubic edge log-normal "
                                   "(median 96, sigma 0.4) clamped to [32, 192], multiple of 16; steps U[30, 300]; "
                                   f"{'config physics (per-request emitter, wind and seed)' if config else 'reference physics'}, "
                                   f"{precision} storage, "
                                   + (f"p = 0 on the top face, multigrid until max|r| <= {0.5 * args.div_target:g}; "
                                      if config and args.solver == "mg" else "SOR 40; ")
                                   + "256x256 render (64 samples) every 4 steps; "
                                   f"HBM budget {args.budget_gb} GB; at most {args.max_active_mvoxels} M active cells"
                                   + (f", round time target {args.latency_target_ms} ms (batched loop)" if args.latency_target_ms > 0 else "")
                                   + "; "
                                   f"run bounded at {args.serve_seconds} s",
                       "latency": "device time between a scene's consecutive step completions (events)"}}
    if emit:
        print(json.dumps(line), flush=True)
    return line


# Algorithmic bytes per cell of each config-physics stage (FP32 layout: record a
# = heat, fuel, (unused), soot is 16 B; faces ~12 B; vorticity and force 16 B).
CONFIG_STAGE_BYTES_PER_CELL = {
    "advect_velocity": 24.0,                   # read + write the faces (gathers hit L1/L2)
    "advect_react": 16.0 * 2 + 12.0,           # read + write record a, read the faces
    "force": 12.0 + 16.0 + 16.0 * 3 + 12.0 * 2 + 16.0,  # vorticity w, cell force r/w, faces r/w
    "divergence": 12.0 + 8.0,                  # read faces, write div and p
    "pressure_sor": 6.0,                       # per half sweep
    "subtract_walls": 4.0 + 24.0,
}


def config_stage_timings(sim, settings, steps: int = 3) -> dict:
    """Device time of each stage inside real steps: `steps` whole steps (render
    included), each queued stage by stage with events between consecutive
    stages on the scene stream; the minimum per stage over the steps."""
    import torch
    ext = torch.cuda.ExternalStream(sim.stream())
    ranges = [("advect_velocity", "advect_velocity", "advect_velocity"), ("advect_react", "advect_react", "advect_react"),
              ("force", "force", "velocity_boundary"), ("divergence", "divergence", "divergence"),
              ("pressure_sor", "pressure_sor", "pressure_sor"), ("subtract_walls", "subtract", "wall_boundary"),
              ("light", "light_build", "light_build"), ("render", "render", "render")]
    out = {name: float("inf") for name, _, _ in ranges}
    for _ in range(steps):
        # The spin (about 1 ms) holds the stream until every stage of the step is queued.
        with torch.cuda.stream(ext):
            torch.cuda._sleep(2_000_000)
        marks = [torch.cuda.Event(enable_timing=True) for _ in range(len(ranges) + 1)]
        marks[0].record(ext)
        for k, (name, a, b) in enumerate(ranges):
            sim.stages(a, b, settings, 0.0, wait=False)
            marks[k + 1].record(ext)
        marks[-1].synchronize()
        for k, (name, _, _) in enumerate(ranges):
            out[name] = min(out[name], marks[k].elapsed_time(marks[k + 1]))
    sim.synchronize()
    return out


def config_cpu_baseline(pkg, w, n_steps: int = 2, args=None) -> dict:
    """The config-physics oracle (float, OpenMP, all host threads) on a bounded
    sample, with the same pressure solver as the GPU line."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as om  # noqa: PLC0415
    abi = pkg.abi
    n = w["grid"]
    o = om.ConfigOracle(abi, w["frame"][0], w["frame"][1], *n)
    o.set_physics(w["physics"])
    o.set_pressure_solver(*w["sor"])
    if args is not None and args.solver == "mg":
        o.set_multigrid(args.mg_cycles, args.mg_pre, args.mg_post, 0.5 * args.div_target)
    threads = os.cpu_count() or 1
    om.OracleFire.set_threads(threads)
    o.step()
    t0 = time.perf_counter()
    for _ in range(n_steps):
        o.step()
    t_sim = (time.perf_counter() - t0) / n_steps
    t1 = time.perf_counter()
    o.stages("light_build", "render")
    t_render = time.perf_counter() - t1
    per_step = t_sim + t_render / w["render_every"]
    cells = int(np.prod(n))
    return {"value": cells / per_step, "unit": "voxel-steps/s", "cores": threads, "kind": "port",
            "sample": f"{n_steps} config-physics steps of the {w['name']} workload after one warm-up step, plus one "
                      f"{w['frame'][0]}^2 render amortised over {w['render_every']} steps (oracle/config_oracle.cpp, float"
                      f"{', multigrid' if args is not None and args.solver == 'mg' else ''})",
            "seconds_per_step": per_step}




_PINNED = []  # keeps the page-locked tensors behind pinned_frame's arrays alive


def pinned_frame(fh: int, fw: int):
    """A page-locked host BGRA8 frame (the e2e arm reads each frame into pinned memory)."""
    import torch
    t = torch.zeros((fh, fw), dtype=torch.int32).pin_memory()
    _PINNED.append(t)
    return t.numpy().view(np.uint32)


def divergence_after(pkg, lib, sim, settings, fw: int, fh: int) -> dict:
    """|div u| after the projection of one more measured step (FireCudaFrameMetrics, FP64)."""
    import ctypes
    abi = pkg.abi
    m = abi.FireCudaFrameMetrics()
    host = np.zeros((fh, fw), dtype=np.uint32)
    settings.reset = 0
    if not lib.fireCudaStepAndRenderMeasured(host.ctypes.data, ctypes.byref(settings), ctypes.byref(m)):
        raise RuntimeError(pkg.firesim.last_error(lib))
    return {"max": m.divergenceAfterMax, "l2": m.divergenceAfterL2, "before_max": m.divergenceBeforeMax,
            "note": "one measured step after the timed regions; max over cells, every face included"}


def run_config(args, pkg, world: int, rank: int, local: int, emit: bool = True) -> dict | None:
    """One scene of the config physics (FirePhysicsParams mode 1) on workload c1, c2 or c3."""
    import torch
    abi = pkg.abi
    w = abi.config_workload(args.workload)
    precision = args.precision if args.precision_set else w["precision"]
    n = w["grid"]
    cells = int(np.prod(n))
    fw, fh = w["frame"]
    render_every = w["render_every"]
    lib = pkg.load_library(precision)
    if not lib.fireCudaSelectDevice(local):
        raise RuntimeError(pkg.firesim.last_error(lib))
    sim = pkg.FireSim(fw, fh, *n, precision=precision)
    physics = w["physics"]
    if args.solver == "mg":
        # p = 0 on the top face and multigrid V-cycles until max |r| <= half the
        # divergence target (|div u| after the projection equals |r| up to the
        # rounding of the face update).
        physics.pressureTop = 1
        sim.set_physics(physics)
        sim.set_pressure_multigrid(args.mg_cycles, args.mg_pre, args.mg_post)
        sim.set_pressure_tolerance(0.5 * args.div_target, 1)
    else:
        sim.set_physics(physics)
        sim.set_pressure_solver(*w["sor"])
        if w["tolerance"] > 0:
            sim.set_pressure_tolerance(w["tolerance"], w["check_every"])
    sim.set_pressure_path({"auto": 0, "graph": 1, "resident": 2}[args.sor_path])
    hdr = torch.zeros((fh, fw, 4), dtype=torch.float32, device="cuda")
    sim.register_hdr_slot(0, hdr.data_ptr(), fw * 16, 0)
    sim.set_hdr_slot(0)
    ext = torch.cuda.ExternalStream(sim.stream())
    settings = abi.FireSettings(width=fw, height=fh, dt=w["physics"].dt)
    frame = 0

    def one_step(host_bgra=None):
        nonlocal frame
        settings.reset = 1 if frame == 0 else 0
        render = (frame % render_every) == render_every - 1
        if host_bgra is not None and render:
            if not lib.fireCudaStepAndRender(host_bgra.ctypes.data, settings):
                raise RuntimeError(pkg.firesim.last_error(lib))
        elif render:
            sim.step_and_render_hdr(settings)
        else:
            sim.step(settings)
        frame += 1

    for _ in range(args.warmup):
        one_step()
    sim.synchronize()
    sampler = ClockSampler(local)
    dist_barrier(world)
    torch.cuda.synchronize()
    sampler.start()
    launches0 = sim.launch_count()
    marks = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    marks[0].record(ext)
    for i in range(args.steps):
        one_step()
        marks[i + 1].record(ext)
    marks[-1].synchronize()
    torch.cuda.synchronize()
    dist_barrier(world)
    clocks = sampler.stop()
    launches = sim.launch_count() - launches0
    step_ms = np.array([marks[i].elapsed_time(marks[i + 1]) for i in range(args.steps)])
    device_s = dist_max(marks[0].elapsed_time(marks[-1]) / 1e3, world)
    value = cells * args.steps * world / device_s
    stats = sim.pressure_stats()

    e2e = None
    if not args.no_e2e:
        # The same frames as the device-timed region: reset, the same warm-up, then the timed steps.
        host = pinned_frame(fh, fw)
        frame = 0
        for _ in range(args.warmup):
            one_step()
        dist_barrier(world)
        sim.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            one_step(host_bgra=host)
        sim.synchronize()
        wall = dist_max(time.perf_counter() - t0, world)
        renders = sum(1 for f in range(frame - args.steps, frame) if f % render_every == render_every - 1)
        e2e = {"value": cells * args.steps * world / wall, "unit": "voxel-steps/s",
               "h2d_bytes_per_step": int(ctypes_sizeof_settings(abi)),
               "d2h_bytes_per_step": int(renders * fw * fh * 4 / args.steps), "ms_per_step": wall * 1e3 / args.steps}

    divergence = divergence_after(pkg, lib, sim, settings, fw, fh)
    st = config_stage_timings(sim, settings)
    per_step = {k: (v / render_every if k in ("light", "render") else v) for k, v in st.items()}
    dominant = max((k for k in CONFIG_STAGE_BYTES_PER_CELL), key=per_step.get)
    peaks, peak_src = measured_peaks()
    iters = stats[0] if stats[1] >= 0 else w["sor"][0]
    if dominant == "pressure_sor" and args.solver == "mg":
        # One "launch" here is the whole solve: its level-0 half sweeps at 6 B/cell each.
        # Level-0 half sweeps of one V-cycle: pre- and post-smoothing sweeps of two colours.
        level0_half_sweeps = 2 * (args.mg_pre + args.mg_post)
        bytes_launch = CONFIG_STAGE_BYTES_PER_CELL["pressure_sor"] * cells * level0_half_sweeps * iters
        launch_ms = st["pressure_sor"]
    elif dominant == "pressure_sor":
        launches_per = 2 * iters
        bytes_launch = CONFIG_STAGE_BYTES_PER_CELL["pressure_sor"] * cells
        launch_ms = st["pressure_sor"] / launches_per
    else:
        bytes_launch = CONFIG_STAGE_BYTES_PER_CELL[dominant] * cells
        launch_ms = st[dominant]
    achieved = bytes_launch / (launch_ms * 1e-3) / 1e9
    roofline = {"kernel": dominant, "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": None, "peak_source": peak_src,
                "bytes_per_launch": bytes_launch, "launch_ms": launch_ms}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = config_cpu_baseline(pkg, w, args=args)
        cpu = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    if rank == 0:
        p = w["physics"]
        line = {
            "metric": "voxel-steps/s", "value": value, "unit": "voxel-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": device_s * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if precision == "f32" else f"{precision}-storage/f32-arithmetic",
            "data": "synthetic (seeded disk emitters, SplitMix64 jitter)",
            "config": {"workload": f"config physics {w['name']}: {n[0]}^3, {p.emitterCount} disk emitter(s), "
                                   + (f"p = 0 on the top face, multigrid V-cycles until max|r| <= {0.5 * args.div_target:g} "
                                      f"(|div u| <= {args.div_target:g}), at most {args.mg_cycles}, "
                                      f"V({args.mg_pre},{args.mg_post})"
                                      if args.solver == "mg" else
                                      f"SOR {w['sor'][0]} omega {w['sor'][1]}"
                                      f"{' until max|r| <= %g' % w['tolerance'] if w['tolerance'] else ''}") + ", "
                                   f"{fw}x{fh} render every {render_every} steps ({p.primarySamples} samples, "
                                   f"{p.lightSamples} light samples)",
                       "grid": list(n), "physics": "config (FirePhysicsParams mode 1)", "sor_path": args.sor_path,
                       "l2": "no flush", "parallelism": "replicas"},
            "e2e": e2e, "gpu_launches": launches, "clocks": clocks, "roofline": roofline, "stage_ms": per_step,
            "step_latency": {"unit": "ms", "p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99)),
                             "max": float(step_ms.max())},
            "pressure_stats_last_step": {"iterations": stats[0], "max_residual": stats[1], "l2_residual": stats[2],
                                         "solver": args.solver},
            "divergence_after": divergence,
            "cpu_baseline": cpu,
        }
        if emit:
            print(json.dumps(line), flush=True)
    sim.close()
    return line if rank == 0 else None


def headline_block(args, pkg, world: int, rank: int, local: int) -> dict | None:
    """The comparison at |div u| <= --div-target (p = 0 on the top face,
    multigrid until max |r| <= half of it), measured in the same run: the
    plain 128^3 FP32 single scene (workload c2's physics and render cadence),
    the batched mix (48 scenes of mixed sizes, FP16 storage, one FireBatch),
    and a bounded served run (Poisson arrivals, BF16 storage), with the ratios
    of the batched and served rates to the plain one."""
    import copy
    base = copy.copy(args)
    base.physics, base.solver, base.precision_set = "config", "mg", True
    plain_args = copy.copy(base)
    plain_args.workload, plain_args.precision = "c2", "f32"
    plain_args.steps, plain_args.warmup = args.headline_steps, 10
    plain_args.no_cpu_baseline, plain_args.no_e2e = True, False
    plain = run_config(plain_args, pkg, world, rank, local, emit=False)
    if rank != 0:
        return None
    batched_args = copy.copy(base)
    batched_args.mode, batched_args.precision, batched_args.scenes = "batched", "f16", 48
    batched_args.steps, batched_args.warmup, batched_args.render_every = args.headline_batched_steps, 10, 10
    batched = run_batched(batched_args, pkg, emit=False)
    served_args = copy.copy(base)
    served_args.mode, served_args.precision = "serve", "bf16"
    served_args.arrival_seconds, served_args.serve_seconds = args.headline_arrival_seconds, args.headline_serve_seconds
    served = run_serve(served_args, pkg, emit=False)
    pv = plain["value"]
    return {
        "condition": f"|div u| <= {args.div_target:g}: p = 0 on the top face, multigrid until max|r| <= {0.5 * args.div_target:g}",
        "plain": {"value": pv, "e2e": plain["e2e"]["value"] if plain.get("e2e") else None, "unit": "voxel-steps/s",
                  "workload": plain["config"]["workload"], "dtype": plain["dtype"], "ms_per_step": plain["ms_per_step"],
                  "divergence_after_max": plain["divergence_after"]["max"],
                  "multigrid_cycles_last_step": plain["pressure_stats_last_step"]["iterations"]},
        "batched": {"value": batched["value"], "unit": "voxel-steps/s", "dtype": batched["dtype"],
                    "ms_per_sub_step": batched["ms_per_sub_step"], "voxels_per_sub_step": batched["config"]["voxels_per_sub_step"],
                    "gpu_launches": batched.get("gpu_launches"), "multigrid": batched.get("multigrid_last_sub_step"),
                    "workload": batched["config"]["workload"], "ratio_to_plain": batched["value"] / pv},
        "served": {"value": served["value"], "unit": "voxel-steps/s", "dtype": served["dtype"], "latency_ms": served["latency_ms"],
                   "requests": served["requests"], "seconds": served["seconds"], "workload": served["config"]["workload"],
                   "ratio_to_plain": served["value"] / pv},
    }


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--frame", type=int, default=512)
    ap.add_argument("--sor-iters", type=int, default=60)
    ap.add_argument("--omega", type=float, default=1.8)
    ap.add_argument("--render-every", type=int, default=10)
    ap.add_argument("--samples", type=int, default=128)
    ap.add_argument("--reference-steps", type=int, default=120,
                    help="at most this many timed steps of the CPU reference arm")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--physics", default="reference", choices=["reference", "config"],
                    help="reference: native-firesim's physics (the headline line); config: FirePhysicsParams mode 1")
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3"],
                    help="config physics workload (abi.config_workload)")
    ap.add_argument("--solver", default="sor", choices=["sor", "mg"],
                    help="config physics: the workload's red-black SOR, or p = 0 on the top face with multigrid "
                         "V-cycles until |div u| <= --div-target")
    ap.add_argument("--div-target", type=float, default=1e-4)
    ap.add_argument("--mg-cycles", type=int, default=30)
    ap.add_argument("--mg-pre", type=int, default=2, help="pre-smoothing sweeps per multigrid level")
    ap.add_argument("--mg-post", type=int, default=2, help="post-smoothing sweeps per multigrid level")
    ap.add_argument("--precision", default=None, choices=["f32", "f16", "bf16"],
                    help="storage of the transported fields: f32 (the reference's), f16 or bf16 (FP32 arithmetic)")
    ap.add_argument("--mode", default="single", choices=["single", "batched", "serve"],
                    help="single: the 128^3 scene (the headline line); batched: --scenes scenes per fireBatchStep; "
                         "serve: Poisson requests into the FireServer loop")
    ap.add_argument("--scenes", type=int, default=48)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--arrival-seconds", type=float, default=10.0)
    ap.add_argument("--serve-seconds", type=float, default=60.0)
    ap.add_argument("--budget-gb", type=float, default=120.0)
    ap.add_argument("--max-active-mvoxels", type=float, default=24.0,
                    help="serve: admit while the admitted scenes hold at most this many million cells (0 = no limit)")
    ap.add_argument("--latency-target-ms", type=float, default=4.0,
                    help="serve (batched loop): admit while the predicted round time (cells x the rounds' decaying peak "
                         "time per cell) stays within this (0 = off); chosen to keep p99 step latency under 8 ms on the B200")
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--no-headline", action="store_true",
                    help="single mode: skip the headline block (plain, batched and served at |div u| <= --div-target)")
    ap.add_argument("--headline-steps", type=int, default=100)
    ap.add_argument("--headline-batched-steps", type=int, default=20)
    ap.add_argument("--headline-arrival-seconds", type=float, default=5.0)
    ap.add_argument("--headline-serve-seconds", type=float, default=15.0)
    ap.add_argument("--sor-path", default="auto", choices=["auto", "graph", "resident"],
                    help="pressure SOR: per-launch half sweeps in a CUDA graph, one cooperative resident launch, or auto")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    args.precision_set = args.precision is not None
    if args.precision is None:
        args.precision = "f32"

    world, rank, local = dist_setup()
    if args.impl == "reference":
        if args.physics == "config":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "native-firesim has no config physics (disk "
                                  "emitters, confinement, point light); its CPU restatement is this line's cpu_baseline"}),
                      flush=True)
        else:
            run_reference(args, world, rank)
        dist_barrier(world)
        return 0

    # The GPU arms warm up for at least one whole render interval, so the first
    # timed frame does not pay the first render's one-time costs.
    args.warmup = max(args.warmup, args.render_every)
    import torch
    torch.cuda.set_device(local)
    pkg = load_package()
    if args.physics == "config" and args.mode == "single":
        run_config(args, pkg, world, rank, local)
        dist_barrier(world)
        return 0
    if args.mode != "single":
        if rank == 0:
            if args.mode == "batched":
                run_batched(args, pkg)
            else:
                run_serve(args, pkg)
        dist_barrier(world)
        return 0
    abi = pkg.abi
    lib = pkg.load_library(args.precision)
    if not lib.fireCudaSelectDevice(local):
        raise RuntimeError(pkg.firesim.last_error(lib))
    sim = pkg.FireSim(args.frame, args.frame, args.grid, args.grid, args.grid, precision=args.precision)
    sim.set_pressure_solver(args.sor_iters, args.omega)
    sim.set_pressure_path({"auto": 0, "graph": 1, "resident": 2}[args.sor_path])
    hdr = torch.zeros((args.frame, args.frame, 4), dtype=torch.float32, device="cuda")
    sim.register_hdr_slot(0, hdr.data_ptr(), args.frame * 16, 0)
    sim.set_hdr_slot(0)
    ext = torch.cuda.ExternalStream(sim.stream())
    frame = 0

    def one_step(host_bgra=None):
        nonlocal frame
        s = workload_settings(abi, frame, args)
        render = (frame % args.render_every) == args.render_every - 1
        if host_bgra is not None and render:
            ok = lib.fireCudaStepAndRender(host_bgra.ctypes.data, s)
            if not ok:
                raise RuntimeError(pkg.firesim.last_error(lib))
        elif render:
            sim.step_and_render_hdr(s)
        else:
            sim.step(s)
        frame += 1

    for _ in range(args.warmup):
        one_step()
    sim.synchronize()

    # Device-timed region.
    sampler = ClockSampler(local)
    dist_barrier(world)
    torch.cuda.synchronize()
    sampler.start()
    launches0 = sim.launch_count()
    # One event per step boundary on the scene stream: the whole interval is
    # the timed region, the gaps give the per-step device latency.
    marks = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    marks[0].record(ext)
    for i in range(args.steps):
        one_step()
        marks[i + 1].record(ext)
    e0, e1 = marks[0], marks[-1]
    e1.synchronize()
    torch.cuda.synchronize()
    dist_barrier(world)
    clocks = sampler.stop()
    launches = sim.launch_count() - launches0
    step_ms = np.array([marks[i].elapsed_time(marks[i + 1]) for i in range(args.steps)])
    latency = {"unit": "ms", "p50": float(np.percentile(step_ms, 50)), "p95": float(np.percentile(step_ms, 95)),
               "p99": float(np.percentile(step_ms, 99)), "max": float(step_ms.max()),
               "note": "device time per step from events at step boundaries; steps that render a frame form the tail"}
    device_s = dist_max(e0.elapsed_time(e1) / 1e3, world)
    cells = args.grid ** 3
    value = cells * args.steps * world / device_s

    # End-to-end through the host path.
    e2e = None
    if not args.no_e2e:
        # The same frames as the device-timed region: reset, the same warm-up, then the timed steps.
        host = pinned_frame(args.frame, args.frame)
        frame = 0
        for _ in range(args.warmup):
            one_step()
        dist_barrier(world)
        sim.synchronize()
        t0 = time.perf_counter()
        frame_marks = [t0]
        for _ in range(args.steps):
            one_step(host_bgra=host)
            if (frame - 1) % args.render_every == args.render_every - 1:
                frame_marks.append(time.perf_counter())  # the BGRA call returns with its frame on the host
        sim.synchronize()
        wall = dist_max(time.perf_counter() - t0, world)
        frame_ms = np.diff(np.array(frame_marks)) * 1e3
        renders = sum(1 for f in range(frame - args.steps, frame) if f % args.render_every == args.render_every - 1)
        e2e = {"value": cells * args.steps * world / wall, "unit": "voxel-steps/s",
               "h2d_bytes_per_step": int(ctypes_sizeof_settings(abi)),
               "d2h_bytes_per_step": int(renders * args.frame * args.frame * 4 / args.steps),
               "ms_per_step": wall * 1e3 / args.steps}
        if len(frame_ms):
            e2e["frame_latency_ms"] = {"p50": float(np.percentile(frame_ms, 50)), "p95": float(np.percentile(frame_ms, 95)),
                                       "p99": float(np.percentile(frame_ms, 99)),
                                       "note": f"host wall time per BGRA frame: {args.render_every} steps + render + readback"}

    # Per-stage device times and the roofline of the dominant kernel.
    s = workload_settings(abi, frame, args)
    st = stage_timings(pkg, sim, args, s)
    per_step_ms = {k: (v / args.render_every if k in ("render", "embers") else v) for k, v in st.items()}
    # The stage pass renders the final, most developed fire; the timed region's
    # own frames cost less.  Their mean extra device time over a plain step
    # (from the step latencies) gives the render's share of the timed steps.
    render_steps = [i for i in range(args.steps) if (args.warmup + i) % args.render_every == args.render_every - 1]
    plain_steps = [i for i in range(args.steps) if i not in set(render_steps)]
    if render_steps and plain_steps:
        render_in_region_ms = float(np.mean(step_ms[render_steps]) - np.median(step_ms[plain_steps]))
        per_step_ms["render_end_state"] = per_step_ms["render"]
        per_step_ms["render"] = render_in_region_ms / args.render_every
    dominant = max((k for k in per_step_ms if k != "render_end_state"), key=per_step_ms.get)
    peaks, peak_src = measured_peaks()
    roofline = roofline_block(dominant, st, args, cells, peaks, peak_src, sim.pressure_path_used(),
                              clocks.get("sm_mhz") if isinstance(clocks, dict) else None)

    divergence = divergence_after(pkg, lib, sim, workload_settings(abi, frame, args), args.frame, args.frame)
    sim.close()
    headline = None if args.no_headline else headline_block(args, pkg, world, rank, local)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(pkg, args)
        cpu = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}

    if rank == 0:
        line = {
            "metric": "voxel-steps/s", "value": value, "unit": "voxel-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": device_s * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "f32" else f"{args.precision}-storage/f32-arithmetic",
            "data": "synthetic (seeded procedural fuel bed + validation-harness settings)",
            "config": config_block(args), "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
            "roofline": roofline, "stage_ms": per_step_ms, "step_latency": latency, "divergence_after": divergence,
            "cpu_baseline": cpu, "headline": headline,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def ctypes_sizeof_settings(abi) -> int:
    import ctypes
    return ctypes.sizeof(abi.FireSettings)


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of the
# dominant kernel, from one ncu capture of each workload: the resident solve at
# 128^3 (one launch, SOR 60) and one colour-split half sweep at 256^3
# (profiles/sor_split_256cubed_halfsweep.md: 4.72 TB/s x 23.42 us).
NCU_TRAFFIC_BYTES = {("pressure_sor", "resident", 128, 60): 30157312 + 1525760,
                     ("pressure_sor", "split", 256, 60): 110542400}
# Shared-memory wavefronts of one resident solve (l1tex__data_pipe_lsu_wavefronts_mem_shared.sum
# from one ncu capture of sorResident<32,16,16>, profiles/sor_resident_128cubed_sor60.md): the
# resident solve lives in shared memory, so its roofline is the shared-memory pipe, one
# wavefront per clock per SM.
NCU_SMEM_WAVEFRONTS = {("pressure_sor", "resident", 128, 60): 50293124}


def roofline_block(dominant: str, st: dict, args, cells: int, peaks: dict, peak_src: str, sor_path: int,
                   sm_mhz: float | None = None) -> dict:
    """achieved = algorithmic bytes of one launch / that launch's device time.

    The pressure solve's algorithmic bytes are those of the global-memory
    formulation, 12 B per cell per iteration (read p, write p, read div).  The
    resident path runs the whole solve as one launch, so its launch carries
    all N iterations; the colour-split path has one launch per half sweep."""
    traffic = None
    if dominant == "pressure_sor":
        resident = sor_path == 2
        launches = 1 if resident else 2 * args.sor_iters
        per_launch_ms = st["pressure_sor"] / launches
        bytes_per_launch = 12.0 * args.sor_iters * cells / launches
        traffic = NCU_TRAFFIC_BYTES.get(("pressure_sor", "resident" if resident else "split", args.grid, args.sor_iters))
    elif dominant in STAGE_BYTES_PER_CELL and STAGE_BYTES_PER_CELL[dominant] > 0:
        per_launch_ms = st[dominant]
        bytes_per_launch = STAGE_BYTES_PER_CELL[dominant] * cells
    else:
        # render: compulsory bytes = one read of the fields the rays touch + 16 B/pixel; report against HBM too.
        per_launch_ms = st[dominant]
        bytes_per_launch = 40.0 * cells + 16.0 * args.frame * args.frame
    achieved = bytes_per_launch / (per_launch_ms * 1e-3) / 1e9
    peak = float(peaks.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"]))
    out = {"kernel": dominant, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
           "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
           "bytes_per_launch": bytes_per_launch, "launch_ms": per_launch_ms}
    if dominant == "pressure_sor" and sor_path == 2:
        wavefronts = NCU_SMEM_WAVEFRONTS.get(("pressure_sor", "resident", args.grid, args.sor_iters))
        if wavefronts is not None:
            mhz = sm_mhz if sm_mhz else 1965.0
            per_clock = wavefronts / (per_launch_ms * 1e-3 * mhz * 1e6 * 148)
            out["smem"] = {"achieved": per_clock, "peak": 1.0, "unit": "wavefronts/clock/SM", "frac": per_clock,
                           "wavefronts_per_launch": wavefronts, "sm_mhz": mhz,
                           "note": "the resident solve's data stay in shared memory (DRAM traffic per launch is the "
                                   "'traffic' figure); its bound is the shared-memory pipe; wavefronts from one ncu capture"}
    return out


if __name__ == "__main__":
    sys.exit(main())
