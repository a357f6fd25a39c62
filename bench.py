#!/usr/bin/env python
"""Benchmark of the B200 MLS-MPM substep: MPM particle-steps/s.

Workload (default, one GPU): the single large scene — 256^3 grid, dx = 1/256,
16M particles in 4 seeded random boxes (8 particles per cell, per-box elastic
modulus log-uniform in [1e4, 1e5] or snow with theta_c 2.5e-2, theta_s
7.5e-3), FP32 state with the FP64 SVD/polar decomposition, dt = 2e-5.  A
"step" is one substep of the whole scene; the K timed substeps are centred on
substep 250 of the scene's 500-substep run and open with a regrouping.
Particle state (1.8 GB) and grid (0.8 GB) are far larger than the 126 MB L2,
so no L2 flush is needed between steps.  The line also carries the accuracy
against the FP64 oracle on a sample, the batched (64 scenes, graphs) and
served (continuous batching) forms next to the plain one, the end-to-end rate
through the C ABI with host buffers, and the CPU oracle's rate.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload large|medium|cube|cube128|batched|served|precision]

N > 1 runs under torchrun: every rank steps its own replica of the scene
(independent scenes, no data-path collective; "scaling": "weak"); time is the
max over ranks.  `--impl reference` times the CPU restatement of the
reference step (the oracle, OpenMP on all host cores) on the same workload and
prints the same metric.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "MPM particle-steps/sec on 1 B200 (batched-served vs plain) + p50/p99 step ms"
UNIT = "particle-steps/s"

# Algorithmic bytes per launch of the two particle kernels (FP32 state):
#  gather (G2P + F update + return mapping + stress record): reads pos 12,
#    F 36, jp 4, mass 4, volume 4, material 4 = 64 B and writes pos 12, F 36,
#    jp 4 and the 64-byte scatter record (x, m, m v, B) = 116 B per particle
#    (velocity and C are written only by the last substep of a call); reads
#    the grid velocity once per active node (16 B).
#  scatter (P2G deposit): reads the 64-byte record per particle; adds one
#    float4 accumulator per active node (16 B).
KERNEL_BYTES = {
    "GridToParticle": (180, 16),
    "ParticleToGrid": (64, 16),
}
# DRAM bytes per particle per launch (dram__bytes_read.sum +
# dram__bytes_write.sum) from one ncu capture of each kernel of the separate
# substep on the medium workload (128^3 grid, 2M particles, substep ~250),
# scaled by particle count.
MEASURED_TRAFFIC_PER_PARTICLE = {
    "GridToParticle": 156.4,
    "ParticleToGrid": 70.9,
}
# The fused gather + scatter (k_g2p2g, groups of at most 256k particles)
# keeps the 64-byte record in shared memory: 180 - 64 B per particle, and per
# active node the velocity read plus the float4 deposit.
FUSED_BYTES = (116, 32)
# ncu DRAM bytes per particle of k_g2p2g on the 1M-particle scaled cube
# (state 160 MB, just above L2).
MEASURED_TRAFFIC_FUSED_PER_PARTICLE = 76.5
# Whole-step model of the survey (separate P2G and G2P passes):
# 268 B per particle-step + 56 B per active cell-step.
STEP_BYTES_PER_PARTICLE = 268
STEP_BYTES_PER_ACTIVE_CELL = 56


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples the SM clock and the clock-event (throttle) reasons during the
    timed region: through NVML every ~2 ms when it is available (a timed
    region of a few tens of ms still gets many samples), else through
    nvidia-smi every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                   "hw_thermal_slowdown": 0x40}

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.samples = []  # (sm MHz, reason bits) from NVML
        self.sm_max = None
        self.nvml = None
        self.stop = False
        self.source = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        handle = None
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            handle = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            handle = pynvml.nvmlDeviceGetHandleByIndex(self.index)
        return pynvml, handle

    def _poll(self):
        nv, h = self.nvml
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self.stop:
            try:
                self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), int(get_reasons(h))))
            except Exception:
                break
            time.sleep(0.002)

    def __enter__(self):
        try:
            self.nvml = self._nvml_handle()
            nv, h = self.nvml
            self.sm_max = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            self.source = "nvml"
            time.sleep(0.01)
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            self.source = "nvidia-smi"
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        self.stop = True
        if self.nvml:
            self.thread.join(timeout=2)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], self.sm_max, set()
        for mhz, bits in self.samples:
            sm.append(mhz)
            for name, bit in self.REASON_BITS.items():
                if bits & bit:
                    reasons.add(name)
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": smax, "reasons": ["unsampled"], "source": self.source}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm),
                "source": self.source}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_dist(ws, backend):
    if ws <= 1:
        return None
    import datetime

    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return dist


def max_over_ranks(dist, x: float, device=None) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, device=None):
    if dist is not None:
        if device is not None:
            dist.barrier(device_ids=[device.index])
        else:
            dist.barrier()


def make_workload(name: str, rank: int):
    from molla_b200 import scenes
    if name == "large":
        return scenes.boxes_scene(grid_size=256, n_particles=16_000_000, n_boxes=4, seed=1 + rank), \
            {"workload": "single large scene: 256^3 grid, 16M particles in 4 seeded boxes (elastic E 1e4..1e5 / "
                         "snow), FP32 + FP64 SVD, dt 2e-5", "grid": 256, "particles": 16_000_000,
             "svd": "fp64", "l2": "inputs (2.6 GB state) exceed the 126 MB L2; no flush needed"}
    if name == "medium":
        return scenes.boxes_scene(grid_size=128, n_particles=2_000_000, n_boxes=4, seed=1 + rank, dt=4.0e-5), \
            {"workload": "profiling case: the large scene's generator at 128^3 grid, 2M particles, FP32 + FP64 SVD, "
                         "dt 4e-5 (same CFL number)", "grid": 128, "particles": 2_000_000, "svd": "fp64",
             "l2": "state (330 MB) exceeds the 126 MB L2"}
    if name == "cube128":
        return scenes.cube_scene(grid_size=128, seed=rank), \
            {"workload": "elastic cube scaled: 128^3 grid, 1M particles, E 1e4, FP32 + FP64 SVD, dt 5e-5",
             "grid": 128, "particles": 1_000_000, "svd": "fp64",
             "l2": "state (160 MB) exceeds the 126 MB L2"}
    if name == "cube":
        return scenes.cube_scene(grid_size=64, seed=rank, walls=1), \
            {"workload": "elastic cube: 64^3 grid, 132,651 particles, E 1e4, sticky walls 3 cells, FP32, dt 1e-4",
             "grid": 64, "particles": 132651, "svd": "fp32",
             "l2": "state (15 MB) fits in L2; reported for reference only"}
    raise SystemExit(f"unknown workload {name}")


def cpu_sample_scene(n_sample: int, seed: int = 1):
    from molla_b200 import scenes
    return scenes.boxes_scene(grid_size=256, n_particles=n_sample, n_boxes=4, seed=seed)


def time_cpu_oracle(scene, steps: int, warmup: int, threads: int):
    """Times the oracle (FP32 state, FP64 SVD, OpenMP) on `scene`."""
    import molla_b200 as m
    from oracle import oracle as O
    cfg = m.config_for_scene(scene, svd_precision=1)
    sc = O.make_scene(cfg, scene.rows, scene.dt)
    st = O.init_state(scene.positions, mass=cfg.particle_mass, volume=cfg.particle_volume, ids=scene.ids)
    if warmup:
        O.step(sc, st, warmup, precision="f32_svd64", nthreads=threads)
    t0 = time.perf_counter()
    O.step(sc, st, steps, precision="f32_svd64", nthreads=threads)
    dt = time.perf_counter() - t0
    return scene.n * steps / dt, dt


def run_reference(args):
    ws, rank, _ = dist_env()
    dist = init_dist(ws, "gloo")
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    from oracle import oracle as O
    threads = O.max_threads()
    # Size the sample so the whole run stays within about two minutes.
    probe = cpu_sample_scene(200_000)
    rate, _ = time_cpu_oracle(probe, 1, 0, threads)
    budget_s = float(args.reference_budget_s)
    per_step = budget_s / max(args.steps + args.warmup, 1)
    # The whole 16M-particle scene when the run fits the budget, else the
    # largest sample of the same generator that does.
    n_sample = int(min(16_000_000, max(20_000, rate * per_step * 0.8)))
    if n_sample >= 16_000_000 or args.workload != "large":
        scene, meta = make_workload(args.workload, 0)
        whole = True
    else:
        scene = cpu_sample_scene(n_sample)
        whole = False
        _, meta = None, {"workload": f"sample of the single large scene: {scene.n} particles of its generator "
                                    "(256^3 grid, 4 seeded boxes, elastic E 1e4..1e5 / snow), FP32 + FP64 SVD, "
                                    "dt 2e-5", "grid": 256, "particles": scene.n, "svd": "fp64"}
    value, secs = time_cpu_oracle(scene, args.steps, args.warmup, threads)
    sample = (("the whole scene" if whole else f"{scene.n} particles of the same generator (256^3 grid, 4 boxes, "
               "same materials, dt 2e-5)") + f", {args.steps} substeps after {args.warmup} warm-up")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * secs / max(args.steps, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (fp64 svd)", "data": "synthetic (seeded)",
        "config": meta,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


# The large scene's benchmark run is 500 substeps.  The timed window of K
# substeps is centred on its midpoint (substeps 250 - K/2 .. 250 + K/2, at
# least --warmup untimed substeps first), so that a short window costs what
# the run costs on average: the SVD and the scatter both grow as the scene
# deforms and spreads, and a window right after the start would be cheap.
RUN_SUBSTEPS = 500


def window_plan(steps: int, interval: int):
    """(pad, regroupings) of a timed window of `steps` substeps under a
    regroup cadence of `interval`: the cadence restarts `pad` substeps before
    the window, which puts its regroupings at cadence points around the
    window's middle, and the window then holds `regroupings` of them (a
    regrouping due after its last substep opens the next call instead; with
    pad 0 one opens the window's own call)."""
    pad = (interval - (steps // 2) % interval) % interval
    regroups = (pad + steps - 1) // interval if pad else 1 + (steps - 1) // interval
    return pad, regroups


def measure_accuracy(n_sample: int, substeps: int, threads: int):
    """Errors of the GPU's FP32 + FP64-SVD step against the FP64 oracle (FP64
    state, FP64 Jacobi SVD to 1e-14) on a sample of the large scene's
    generator: positions, grid mass and momentum of the last substep, and the
    GPU's own mass / momentum bookkeeping (grid against particles)."""
    import molla_b200 as m
    from oracle import oracle as O
    scene = cpu_sample_scene(n_sample)
    cfg = m.config_for_scene(scene, svd_precision=1)
    engine = m.Engine(0)
    sim = m.MpmSimulation.new(engine, cfg)
    sim.set_particles(scene.positions)
    sim.set_materials(scene.rows, scene.ids)
    sim.step_n(scene.dt, substeps)
    pos = sim.read_positions().astype(np.float64)
    gmass, gmom = sim.read_grid_mass_momentum()
    tot = sim.conservation_totals()
    sim.close()
    engine.close()
    osc = O.make_scene(cfg, scene.rows, scene.dt, svd_tol=1e-14, svd_sweeps=30)
    st = O.cast_state(O.init_state(scene.positions, mass=cfg.particle_mass, volume=cfg.particle_volume,
                                   ids=scene.ids), np.float64)
    t0 = time.perf_counter()
    om, op = O.step(osc, st, substeps, precision="f64", nthreads=threads, want_grid=True)
    secs = time.perf_counter() - t0
    ref = st["pos"]
    d = pos - ref
    ref_mom = op.reshape(-1, 3).sum(axis=0)
    ref_pmom = (st["vel"] * st["mass"][:, None]).sum(axis=0)
    gpu_mom = gmom.astype(np.float64).reshape(-1, 3).sum(axis=0)
    node_mom_err = np.abs(gmom.astype(np.float64) - op).max() / max(np.abs(op).max(), 1e-30)
    mass0 = float(np.float32(cfg.particle_mass)) * scene.n
    return {
        "reference": "FP64 CPU oracle (FP64 state, FP64 Jacobi SVD tol 1e-14)",
        "sample": f"{scene.n} particles of the large scene's generator, {substeps} substeps from rest",
        "oracle_s": round(secs, 2),
        "pos_rel_max": float((np.abs(d) / np.maximum(np.abs(ref), 1e-30)).max()),
        "pos_rel_l2": float(np.linalg.norm(d) / np.linalg.norm(ref)),
        "grid_mass_rel": float(abs(float(gmass.astype(np.float64).sum()) - float(om.sum())) / float(om.sum())),
        "grid_momentum_rel": float(np.linalg.norm(gpu_mom - ref_mom) / max(np.linalg.norm(ref_mom), 1e-30)),
        "grid_node_momentum_max_rel": float(node_mom_err),
        "mass_drift": float(tot[0] / mass0 - 1.0),
        # particle momentum after the last substep against the oracle's
        "momentum_drift": float(np.linalg.norm(tot[5:8] - ref_pmom) / max(np.linalg.norm(ref_pmom), 1e-30)),
    }


def run_ours(args):
    import torch

    import molla_b200 as m

    ws, rank, local = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA GPU (the MPM path has no CPU fallback)")
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    dist = init_dist(ws, "nccl")

    scene, meta = make_workload(args.workload, rank)
    svd_prec = 1 if meta["svd"] == "fp64" else 0
    engine = m.Engine(local)
    cfg = m.config_for_scene(scene, svd_precision=svd_prec)
    sim = m.MpmSimulation.new(engine, cfg)
    sim.set_particles(scene.positions)
    sim.set_materials(scene.rows, scene.ids)
    n = scene.n

    # Untimed: advance to the fixed trajectory point (the --warmup substeps
    # are part of it), picking the regroup interval on the way: fixed by
    # --sort-interval, or (0) by the autotuner on a snapshot of the state.
    start_at = args.trajectory_start if args.trajectory_start >= 0 else RUN_SUBSTEPS // 2 - args.steps // 2
    start_at = max(args.warmup, start_at)
    first = max(3, min(start_at, start_at - 50))
    sim.step_n(scene.dt, first)
    engine.synchronize()
    tune = None
    shapes = None
    if args.sort_interval > 0:
        interval = args.sort_interval
    else:
        # interval, item size, fused or separate kernels, CTAs per SM
        shapes, tune = sim.autotune_shapes(scene.dt, probe_substeps=32)
        interval = shapes["sort_interval"]
    # The regroup cadence restarts `pad` substeps before the window, so that
    # the window's regroupings fall at cadence points around its middle (one
    # at its middle when K < interval, where it is more than its share): the
    # window holds its share of them rounded, and at least one.  The timed
    # call is a stepping loop's next call: it starts on the records the
    # previous call's last gather left, unless a regrouping opens it (pad 0).
    pad, regroups_in_window = window_plan(args.steps, interval)
    sim.set_sort_interval(interval)
    if start_at - pad > first:
        sim.step_n(scene.dt, start_at - pad - first)
    engine.synchronize()
    gm, _ = sim.read_grid_mass_momentum()
    active = int((gm > 0).sum())
    del gm
    sim.set_sort_interval(interval)  # the cadence starts afresh: the next call opens with a regrouping
    if pad:
        sim.step_n(scene.dt, pad)
    start_at = max(start_at, first + pad)

    # timed region: K substeps in one step_n call, bracketed by a barrier
    # and synchronisation on both sides; device time from CUDA events
    # recorded on the engine's stream (the stream every kernel launches on).
    engine.reset_profile()
    engine.profile(True)
    launches0 = engine.launch_count
    stream = torch.cuda.ExternalStream(engine.stream_handle, device=device)
    barrier(dist, device)
    engine.synchronize()
    torch.cuda.synchronize(device)
    with ClockSampler(local) as clocks:
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        start.record(stream)
        sim.step_n(scene.dt, args.steps)
        stop.record(stream)
        stop.synchronize()
        wall = time.perf_counter() - t0
    engine.synchronize()
    engine.profile(False)
    launches = engine.launch_count - launches0
    prof = engine.read_profile()
    elapsed = start.elapsed_time(stop) / 1000.0
    elapsed_max = max_over_ranks(dist, elapsed, device)
    value = n * args.steps * ws / elapsed_max

    # per-step latency distribution (single-step calls)
    lat = []
    for _ in range(args.latency_samples):
        engine.synchronize()
        t = time.perf_counter()
        sim.step_n(scene.dt, 1)
        engine.synchronize()
        lat.append(1000.0 * (time.perf_counter() - t))

    # End to end through the C ABI with host buffers: each call uploads the
    # scene (positions and material ids from pinned host memory), runs the
    # benchmark's whole trajectory (e2e_substeps, 500 by default) and reads
    # the positions back into a pinned buffer.
    pos_host = torch.from_numpy(scene.positions).pin_memory().numpy()
    ids_host = torch.from_numpy(scene.ids.astype(np.int32)).pin_memory().numpy().view(np.uint32)
    out_host = torch.empty((n, 3), dtype=torch.float32).pin_memory().numpy()
    e2e_times = []
    for it in range(args.e2e_iters + 1):
        engine.synchronize()
        t = time.perf_counter()
        sim.set_particles(pos_host)
        sim.set_materials(scene.rows, ids_host)
        sim.step_n(scene.dt, args.e2e_substeps)
        out = sim.read_positions(out=out_host)
        e2e_times.append(time.perf_counter() - t)
    e2e_s = float(np.median(e2e_times[1:])) if len(e2e_times) > 1 else float(e2e_times[0])
    e2e_s = max_over_ranks(dist, e2e_s, device)
    e2e_value = n * args.e2e_substeps * ws / e2e_s
    sim.close()
    engine.close()

    result = None
    if rank == 0:
        hbm, peak_kind = peaks()
        kernels = {}
        for name, (bp, bc) in KERNEL_BYTES.items():
            cnt, tot = prof.get(name, (0, 0.0))
            avg_ms = tot / max(cnt, 1)
            nbytes = bp * n + bc * active
            ach = nbytes / (avg_ms / 1000.0) / 1e9 if avg_ms > 0 else 0.0
            kernels[name] = {"launches": cnt, "avg_launch_ms": avg_ms, "bytes_per_launch": nbytes,
                             "achieved_gbs": ach, "frac": ach / hbm, "total_ms": tot}
        # The fused substep records its kernel under GridToParticle and runs the
        # separate scatter only once per call.
        fused = kernels["ParticleToGrid"]["launches"] * 2 < kernels["GridToParticle"]["launches"]
        if fused:
            g = kernels["GridToParticle"]
            g["bytes_per_launch"] = FUSED_BYTES[0] * n + FUSED_BYTES[1] * active
            g["achieved_gbs"] = g["bytes_per_launch"] / (g["avg_launch_ms"] / 1000.0) / 1e9 if g["avg_launch_ms"] else 0.0
            g["frac"] = g["achieved_gbs"] / hbm
            g["kernel"] = "k_g2p2g (fused)"
        dom = max(kernels, key=lambda k: kernels[k]["total_ms"])
        fused_bytes = kernels[dom]["bytes_per_launch"]
        fused_ms = kernels[dom]["avg_launch_ms"]
        achieved = kernels[dom]["achieved_gbs"]
        if fused and dom == "GridToParticle":
            kernel_name = "k_g2p2g<gather + return mapping + deposit>"
            per_particle = MEASURED_TRAFFIC_FUSED_PER_PARTICLE
            traffic_source = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of k_g2p2g on the 1M-particle "
                              "scaled cube, scaled by particle count")
        else:
            kernel_name = {"GridToParticle": "k_g2p<G2P + return mapping + record>", "ParticleToGrid": "k_p2g"}[dom]
            per_particle = MEASURED_TRAFFIC_PER_PARTICLE[dom]
            traffic_source = ("ncu dram__bytes_read.sum + dram__bytes_write.sum on the medium workload, scaled by "
                              "particle count")
        step_bytes = STEP_BYTES_PER_PARTICLE * n + STEP_BYTES_PER_ACTIVE_CELL * active
        step_achieved = step_bytes / (elapsed / args.steps) / 1e9
        cpu = None
        accuracy = None
        threads = None
        if ws == 1 and not args.no_cpu_baseline:
            from oracle import oracle as O
            threads = O.max_threads()
            probe = cpu_sample_scene(200_000)
            rate, _ = time_cpu_oracle(probe, 1, 0, threads)
            n_sample = int(min(16_000_000, max(20_000, rate * 15.0 / 3)))
            cs = cpu_sample_scene(n_sample)
            cval, csecs = time_cpu_oracle(cs, 3, 0, threads)
            cpu = {"value": cval, "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"{cs.n} particles of the same generator (256^3 grid, 4 boxes), 3 substeps, "
                             f"{csecs:.1f} s"}
            if args.workload == "large" and not args.no_accuracy:
                accuracy = measure_accuracy(n_sample, 3, threads)
        batched = served = None
        if ws == 1 and args.workload == "large" and not args.no_batched:
            batched = measure_batched(args, quiet=True)
        if ws == 1 and args.workload == "large" and not args.no_served:
            served = measure_served(args, quiet=True)
        e2e_h2d = int(pos_host.nbytes + ids_host.nbytes)
        e2e_d2h = int(out.nbytes)
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": start_at, "ms_per_step": 1000.0 * elapsed_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (fp64 svd)" if svd_prec else "f32",
            "data": "synthetic (seeded boxes; no dataset)",
            "config": dict(meta, active_cells=active, sort_interval=interval, shapes=shapes,
                           autotune_probes=[{"knob": k, "value": v, "ms_per_substep": round(ms, 4)}
                                            for k, v, ms in (tune or [])],
                           timed_substeps=f"{start_at}..{start_at + args.steps} of the scene's trajectory "
                                          f"(untimed advance of {start_at} substeps, --warmup included)",
                           regroups_in_window=regroups_in_window,
                           parallelism=f"replicas x{ws}" if ws > 1 else "single scene"),
            "p50_step_ms": float(np.percentile(lat, 50)) if lat else None,
            "p99_step_ms": float(np.percentile(lat, 99)) if lat else None,
            "stages_ms_per_step": {k: v[1] / max(args.steps, 1) for k, v in prof.items()},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": per_particle * n if per_particle else None,
                         "traffic_source": traffic_source,
                         "peak_kind": peak_kind,
                         "kernel": kernel_name,
                         "bytes_per_launch": fused_bytes, "avg_launch_ms": fused_ms},
            "kernels": kernels,
            "step_roofline": {"achieved": step_achieved, "frac": step_achieved / hbm,
                              "bytes_per_step": step_bytes, "model": "268 B/particle + 56 B/active cell"},
            "cpu_baseline": cpu,
            "accuracy": accuracy,
            "batched": batched,
            "served": served,
            "e2e": {"value": e2e_value, "unit": UNIT, "substeps_per_call": args.e2e_substeps,
                    "h2d_bytes_per_step": e2e_h2d / args.e2e_substeps,
                    "d2h_bytes_per_step": e2e_d2h / args.e2e_substeps,
                    "h2d_bytes_per_call": e2e_h2d, "d2h_bytes_per_call": e2e_d2h,
                    "call": f"set_particles + set_materials (pinned host), step_n({args.e2e_substeps}) from rest, "
                            f"read_positions (pinned host)",
                    "call_s": [round(x, 4) for x in e2e_times]},
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
            "wall_s": wall,
        }
    barrier(dist, device)
    if rank == 0:
        print(json.dumps(result), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def _stage_roofline(prof, n, active, hbm):
    kernels = {}
    for name, (bp, bc) in KERNEL_BYTES.items():
        cnt, tot = prof.get(name, (0, 0.0))
        avg_ms = tot / max(cnt, 1)
        nbytes = bp * n + bc * active
        ach = nbytes / (avg_ms / 1000.0) / 1e9 if avg_ms > 0 else 0.0
        kernels[name] = {"launches": cnt, "avg_launch_ms": avg_ms, "bytes_per_launch": nbytes, "achieved_gbs": ach,
                         "frac": ach / hbm, "total_ms": tot}
    dom = max(kernels, key=lambda k: kernels[k]["total_ms"])
    return dom, kernels


def run_precision(args):
    """Precision study: the cube scene (config 0 geometry, sticky walls) at
    --precision-grid (128: 1M particles, dt 5e-5) run on the GPU as all-FP32,
    FP32 + FP64 SVD and all-FP64, against the FP64 CPU oracle (FP64 Jacobi
    SVD, tol 1e-14); position and grid-momentum errors every 100 substeps."""
    import torch

    import molla_b200 as m
    from molla_b200 import scenes
    from oracle import oracle as O

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA GPU (the MPM path has no CPU fallback)")
    g = args.precision_grid
    scene = scenes.cube_scene(grid_size=g, seed=0, walls=1)
    total = args.precision_steps
    every = 100
    engine = m.Engine(0)
    runs = {}
    for name, prec in (("fp32", 0), ("fp32_svd64", 1)):
        cfg = m.config_for_scene(scene, svd_precision=prec)
        sim = m.MpmSimulation.new(engine, cfg)
        sim.set_particles(scene.positions)
        sim.set_materials(scene.rows, scene.ids)
        runs[name] = (sim, cfg)
    cfg64 = m.config_for_scene(scene, svd_precision=1)
    sim64 = m.MpmSimulation64(engine, cfg64)
    sim64.set_particles(scene.positions.astype(np.float64))
    sim64.set_materials(scene.rows, scene.ids)
    osc = O.make_scene(cfg64, scene.rows, scene.dt, svd_tol=1e-14, svd_sweeps=30)
    st = O.cast_state(O.init_state(scene.positions, mass=cfg64.particle_mass, volume=cfg64.particle_volume,
                                   ids=scene.ids), np.float64)
    threads = O.max_threads()
    mass0 = float(np.float32(cfg64.particle_mass)) * scene.n
    dt = float(np.float32(scene.dt))
    rows = []
    gpu_ms = {k: 0.0 for k in ("fp32", "fp32_svd64", "fp64_gpu")}
    cpu_s = 0.0
    done = 0
    while done < total:
        k = min(every, total - done)
        for name, (sim, _) in runs.items():
            engine.synchronize()
            t = time.perf_counter()
            sim.step_n(scene.dt, k)
            engine.synchronize()
            gpu_ms[name] += 1000.0 * (time.perf_counter() - t)
        engine.synchronize()
        t = time.perf_counter()
        sim64.step_n(dt, k)
        engine.synchronize()
        gpu_ms["fp64_gpu"] += 1000.0 * (time.perf_counter() - t)
        t = time.perf_counter()
        gm, gp = O.step(osc, st, k, precision="f64", nthreads=threads, want_grid=True)
        cpu_s += time.perf_counter() - t
        done += k
        ref = st["pos"]
        ref_mom = gp.reshape(-1, 3).sum(axis=0)
        ref_norm = float(np.linalg.norm(ref_mom)) or 1.0
        row = {"step": done, "oracle_grid_mass_drift": float(gm.sum() / mass0 - 1.0)}
        outs = {name: (sim.read_positions().astype(np.float64), sim.conservation_totals())
                for name, (sim, _) in runs.items()}
        m64 = sim64.grid_totals()
        outs["fp64_gpu"] = (sim64.read_positions(), np.array([m64[0], *m64[1], 0, 0, 0, 0]))
        for name, (pos, tot) in outs.items():
            d = pos - ref
            row[name] = {
                "pos_rel_max": float((np.abs(d) / np.maximum(np.abs(ref), 1e-30)).max()),
                "pos_rel_l2": float(np.linalg.norm(d) / np.linalg.norm(ref)),
                "pos_abs_max": float(np.abs(d).max()),
                "grid_momentum_rel": float(np.linalg.norm(tot[1:4] - ref_mom) / ref_norm),
                "grid_mass_drift": float(tot[0] / mass0 - 1.0),
            }
        rows.append(row)
        print(json.dumps({"progress": row}), file=sys.stderr, flush=True)
    last = rows[-1]
    line = {
        "metric": "position / grid-momentum error vs the FP64 CPU oracle per 100 substeps", "unit": "relative",
        "value": last["fp32_svd64"]["pos_rel_max"], "higher_is_better": False, "n_gpus": 1,
        "steps": total, "warmup": 0, "dtype": "f32 | f32 (fp64 svd) | f64",
        "data": "synthetic (seeded jittered cube; no dataset)",
        "config": {"workload": f"precision study: elastic cube [0.3,0.7]^3, {g}^3 grid, {scene.n} particles, "
                               f"E 1e4, nu 0.2, rho 1, sticky walls 3 cells, dt {scene.dt:g}",
                   "oracle": "FP64 CPU restatement, FP64 Jacobi SVD tol 1e-14 / 30 sweeps",
                   "modes": ["fp32", "fp32_svd64", "fp64_gpu"]},
        "gate_pos_rel_1e-4_at_end": {k: last[k]["pos_rel_max"] < 1e-4 for k in ("fp32", "fp32_svd64", "fp64_gpu")},
        "gpu_ms_per_step": {k: v / total for k, v in gpu_ms.items()},
        "oracle_s_per_step": cpu_s / total, "oracle_threads": threads,
        "errors": rows,
    }
    print(json.dumps(line), flush=True)
    for sim, _ in runs.values():
        sim.close()
    sim64.close()
    engine.close()


def measure_batched(args, quiet=False):
    """64 independent scenes of uneven size (grids log-uniform
    32^3..128^3, 10k..2M particles at 8 per cell, half elastic half snow,
    FP32) stepped in the same launches through captured CUDA graphs, with the
    regroup interval autotuned; compared with the plain form (one simulation
    per scene, stepped one after the other without graphs) at the same point
    of the same scenes' trajectories on the same GPU.  Both forms first
    advance `batched_advance` substeps untimed."""
    import torch

    import molla_b200 as m
    from molla_b200 import scenes

    ss = scenes.batch_scenes(count=args.scenes, seed=3)
    total = sum(s.n for s in ss)
    cells = sum(s.grid_size ** 3 + 256 for s in ss)
    engine = m.Engine(0)
    stream = torch.cuda.ExternalStream(engine.stream_handle, device=torch.device("cuda", 0))
    steps = args.batched_steps
    g = m.MpmGroup(engine, len(ss), total, cells)
    for s in ss:
        g.add_scene(m.config_for_scene(s), s.rows, s.positions, s.ids, s.dt)
    g.step_graph(max(3, args.batched_advance // 2), 1)
    shapes, tune = g.autotune_shapes(probe_substeps=32)
    chosen = shapes["sort_interval"]
    g.step_graph(max(3, args.batched_advance - args.batched_advance // 2), 1)
    g.step_graph(steps, 1)  # captures the timed sequence's graph
    engine.synchronize()
    launches0 = engine.launch_count
    with ClockSampler(0) as clocks:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.step_graph(steps, 1)
        e1.record(stream)
        e1.synchronize()
    launches = engine.launch_count - launches0
    t_batched = e0.elapsed_time(e1) / 1000.0
    value = total * steps / t_batched
    lat = []
    for _ in range(args.latency_samples):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        g.step_graph(1, 1)
        b.record(stream)
        b.synchronize()
        lat.append(a.elapsed_time(b))
    engine.profile(True)
    engine.reset_profile()
    g.step(8)
    engine.synchronize()
    engine.profile(False)
    prof = engine.read_profile()
    g.close()
    # plain form: one simulation per scene, sequential step_n calls
    sims = []
    for s in ss:
        sim = m.MpmSimulation.new(engine, m.config_for_scene(s))
        sim.set_particles(s.positions)
        sim.set_materials(s.rows, s.ids)
        sim.set_sort_interval(chosen)
        sims.append((sim, s))
    for sim, s in sims:
        sim.step_n(s.dt, args.batched_advance + steps)
    engine.synchronize()
    e0.record(stream)
    for sim, s in sims:
        sim.step_n(s.dt, steps)
    e1.record(stream)
    e1.synchronize()
    t_plain = e0.elapsed_time(e1) / 1000.0
    plain = total * steps / t_plain
    for sim, _ in sims:
        sim.close()
    engine.close()
    return {
        "workload": f"batched: {len(ss)} scenes, grids 32^3..128^3, {total} particles, mixed elastic/snow, FP32, "
                    f"CUDA-graph captured, autotuned shapes (regroup interval, item size, fused or separate kernels, CTAs per SM); {steps} substeps timed after "
                    f"{args.batched_advance + steps} untimed",
        "value": value, "unit": UNIT, "ms_per_step": 1000.0 * t_batched / steps,
        "plain": {"value": plain, "ms_per_step": 1000.0 * t_plain / steps,
                  "form": "one MpmSimulation per scene, step_n one after the other, no graphs"},
        "batched_over_plain": value / plain,
        "p50_step_ms": float(np.percentile(lat, 50)) if lat else None,
        "p99_step_ms": float(np.percentile(lat, 99)) if lat else None,
        "scenes": len(ss), "particles": total, "regroup_interval": chosen, "shapes": shapes,
        "autotune_probes": [{"knob": k, "value": v, "ms_per_substep": round(ms, 4)} for k, v, ms in tune],
        "stages_ms_per_step": {k: v[1] / 8 for k, v in prof.items()},
        "gpu_launches": int(launches), "clocks": clocks.summary(),
    }


def run_batched(args):
    d = measure_batched(args)
    line = {"metric": METRIC, "value": d["value"], "unit": UNIT, "n_gpus": 1, "steps": args.batched_steps,
            "warmup": args.batched_advance, "ms_per_step": d["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scenes; no dataset)",
            "config": {"workload": d["workload"]}, **{k: v for k, v in d.items() if k not in ("value", "workload")}}
    print(json.dumps(line), flush=True)


def measure_served(args, quiet=False):
    """configs[4], continuous batching: Poisson arrivals (200 scenes/s) of
    scenes sized as the batched workload, 200..2000 substeps each, admitted by
    an HBM budget as slots and memory free up, stepped together in
    fixed-length ticks (each scene stops on the device after its own step
    count), retired at the next regrouping.  The offered load exceeds the
    GPU's throughput, so the queue grows; arrivals beyond 512 queued requests
    are refused and counted."""
    import time as _t

    import molla_b200 as m
    from molla_b200 import scenes

    pool = scenes.batch_scenes(count=args.scenes, seed=3)
    cfgs = [m.config_for_scene(s) for s in pool]
    engine = m.Engine(0)
    srv = m.MpmServer(engine, hbm_budget_bytes=int(args.budget_gb * (1 << 30)), max_scenes=2048)
    rng = np.random.default_rng(7)
    t0 = _t.perf_counter()
    next_arrival = 0.0
    submitted = refused = 0
    first_ticket = None
    while _t.perf_counter() - t0 < args.serve_seconds:
        now = _t.perf_counter() - t0
        while next_arrival <= now:
            k = submitted % len(pool)
            s = pool[k]
            st = srv.stats()
            if submitted - st["admitted"] >= 512:
                refused += 1
            else:
                steps = int(rng.integers(200, 2001))
                tk = srv.submit(cfgs[k], s.rows, s.positions, s.ids, s.dt, steps)
                first_ticket = tk if first_ticket is None else first_ticket
                submitted += 1
            next_arrival += rng.exponential(1.0 / args.arrival_rate)
        srv.run(1, substeps_per_tick=args.tick_substeps)
    if first_ticket is not None:
        srv.poll(first_ticket)  # completes the tick still running
    elapsed = _t.perf_counter() - t0
    st = srv.stats()
    srv.close()
    engine.close()
    return {
        "workload": f"served: Poisson {args.arrival_rate}/s arrivals, scenes as the batched workload, 200..2000 "
                    f"substeps each, HBM budget {args.budget_gb} GB, {args.tick_substeps}-substep ticks "
                    "(graph-replayed), device-side per-scene budgets",
        "value": st["particle_steps"] / elapsed, "unit": UNIT, "seconds": elapsed,
        "p50_step_ms": st["tick_ms_p50"], "p99_step_ms": st["tick_ms_p99"],
        "queue_ms_p50": st["queue_ms_p50"], "queue_ms_p99": st["queue_ms_p99"],
        "submitted": submitted, "refused": refused, "admitted": st["admitted"], "completed": st["completed"],
        "resident_scenes": st["resident_scenes"], "resident_bytes": st["resident_bytes"],
        "ticks": st["ticks"], "host_ms": {"admit": st["admit_ms"], "step": st["step_ms"], "retire": st["retire_ms"],
                                          "graph_build": st["graph_build_ms"]},
        "graph_builds": st["graph_builds"], "faulted": st["faulted"],
    }


def run_served(args):
    d = measure_served(args)
    line = {"metric": METRIC, "value": d["value"], "unit": UNIT, "n_gpus": 1, "steps": None, "warmup": 0,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scenes; no dataset)", "config": {"workload": d["workload"]},
            **{k: v for k, v in d.items() if k not in ("value", "workload")}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="large", choices=["large", "medium", "cube", "cube128", "batched", "served", "precision"])
    ap.add_argument("--scenes", type=int, default=64)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--arrival-rate", type=float, default=200.0)
    ap.add_argument("--serve-seconds", type=float, default=15.0)
    ap.add_argument("--tick-substeps", type=int, default=20)
    ap.add_argument("--sort-interval", type=int, default=0,
                    help="substeps between regroups; 0 = autotuned on the warmed-up scene")
    ap.add_argument("--latency-samples", type=int, default=20)
    ap.add_argument("--e2e-iters", type=int, default=2)
    ap.add_argument("--e2e-substeps", type=int, default=500,
                    help="substeps per end-to-end call (the large scene's whole 500-substep trajectory)")
    ap.add_argument("--trajectory-start", type=int, default=-1,
                    help="substep of the scene's trajectory where the timed window starts (default: the window "
                         "is centred on substep 250 of the 500-substep run)")
    ap.add_argument("--batched-steps", type=int, default=64)
    ap.add_argument("--batched-advance", type=int, default=64)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--precision-grid", type=int, default=128)
    ap.add_argument("--precision-steps", type=int, default=1000)
    ap.add_argument("--reference-budget-s", type=float, default=120.0,
                    help="CPU seconds the reference arm sizes its sample for")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "served":
        run_served(args)
    elif args.workload == "precision":
        run_precision(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
