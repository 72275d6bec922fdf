#!/usr/bin/env python
"""Benchmark of the world DEM step on B200: grain-steps/s at 2^20 grains, FP32.

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

Workload (default): granular column collapse at 2^20 grains, lognormal diameters
(mean 5 mm, log-sigma 0.15, clipped to [0.7 d, 1.4 d]), mu = 0.5 with tangential
springs and per-pair history, restitution 0.5, k_n = 1e5 N/m, semi-implicit Euler,
dt = 1e-5 s, 453 x 453 x 226 collision grid, 128^3 CIC grid; synthetic seeded input
(world_b200/scenes.py). A step is one take_step() over all grains.

value  -- device time of K steps (CUDA events on the library's stream around each
          step; a 512 MiB write queued on the same stream before every step flushes
          L2 and is not timed), max over ranks; grains x ranks x K / time.
e2e    -- the same metric through the C ABI with host buffers: each step
          wd_set_state_async() from pinned host memory, wd_step(1),
          wd_get_positions_async() to pinned host memory, all inside the timed region
          (copies on two copy streams, overlapped with the neighbouring steps).
neighbor search -- Verlet lists, skin and contact-kernel block size chosen by the
          library's autotuner before the warm-up (--skin S fixes the skin; 0 searches
          the grid every step as the reference does): the grid search and sort run
          only when a grain has moved 0.49 skin since the last build; the results are
          bit-identical either way.
roofline -- the contact kernel (forces + integrator, the dominant kernel): its
          algorithmic bytes per launch over its average event-timed duration,
          against the measured HBM copy bandwidth.
cpu_baseline -- the oracle port (C, OpenMP on all host cores) on a bounded sample
          of the same workload, rank 0 at N = 1 only.
settled / batched / adjoint -- (N = 1, default workload) the same metric in the
          contact-bearing regime (the same column after 30,000 steps, when it has
          collapsed onto the floor), for the two batched ensembles (from rest, and
          after the same 30,000 steps beside the settled column), and the reverse
          pass's cost, each beside the plain step measured above on the same GPU.

--impl reference: the reference's step has no CPU implementation (it is CUDA only),
so the reference arm times the oracle port (oracle/dem_oracle.c, the reference's step
restated in C with OpenMP) on all host cores, on the same workload and config, with
W untimed and K timed steps (K capped so that the run ends within a few minutes; the
line says how many ran). It loads no part of libworld_b200.

Multi-GPU: one process per GPU (torchrun), each rank advancing its own ensemble
member of the same workload (seed 12345 + rank); no collective on the data path,
scaling "weak"; only the timing max-reduction uses NCCL.

--workload adjoint_32k: the reverse pass (world_b200.adjoint) over a 200-step window of
the 32,768-grain column, its throughput and its cost relative to the forward window.

Batched workloads (--workload ensemble_64x32k: 64 perturbed 32,768-grain columns;
design_256: 256 columns with n log-uniform in [4096, 131072], H/R in [1, 6], mu in
[0, 0.8]): all scenes step as one SceneBatch; with N ranks the scenes are shared out
by grain count (world_b200.batch.shard_scenes), total work fixed ("strong").
"""
from __future__ import annotations

import argparse
import datetime
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "grain-steps/s at 2^20 grains FP32"
UNIT = "grain-steps/s"
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="collapse_1m_sie_mu05")
    ap.add_argument("--grains", type=int, default=None, help="override the grain count")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=50)
    ap.add_argument("--phase-steps", type=int, default=50)
    ap.add_argument("--settled-steps", type=int, default=30000,
                    help="steps from rest before the contact-bearing (settled) measurement")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the settled, batched and adjoint sub-measurements")
    ap.add_argument("--build-steps", type=int, default=200,
                    help="settled column: steps timed one at a time to cost a list build")
    ap.add_argument("--settled-only", action="store_true",
                    help="of the sub-measurements, run the settled one only")
    ap.add_argument("--field-reps", type=int, default=5,
                    help="timed CIC deposits and energy reductions of the headline state")
    ap.add_argument("--save-after", type=int, default=0, metavar="K",
                    help="with --checkpoint PATH: advance the workload K steps from rest, write "
                         "the checkpoint (state file + sidecar with springs) and exit")
    ap.add_argument("--checkpoint", default=None, metavar="PATH",
                    help="start the workload from this checkpoint instead of from rest (or, "
                         "with --save-after, write it)")
    ap.add_argument("--skin", type=float, default=-1.0,
                    help="Verlet-list skin in m (simulation.neighbor_skin); negative: chosen by "
                         "the autotuner; 0: grid search every step, as the reference")
    ap.add_argument("--contact-kernel", default=None, metavar="BLOCK,VARIANT",
                    help="with --skin >= 0: the list contact kernel (block size, variant 48/64 "
                         "per-lane, 0 cooperative, 1/2 bulk-staged); default: the library's")
    ap.add_argument("--direct", action="store_true",
                    help="launch each step's kernels directly instead of as one CUDA graph "
                         "(for per-kernel profilers, which cannot see inside graphs with "
                         "conditional nodes or device-launched graphs)")
    return ap.parse_args()


def env_int(name: str, default: int) -> int:
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def workload_config(spec, workload: str, grains: int, scenes=None) -> dict:
    """The workload's description, identical in both arms (`spec` is the scene's
    ConfigSpec: no library needed)."""
    out = {
        "workload": workload,
        "grains": grains,
        "integrator": spec.time_integrator,
        "mu": spec.physics.friction,
        "tangential_history": bool(spec.history),
        "diameters": "lognormal(mean 5 mm, sigma 0.15) clipped [0.7d, 1.4d]"
        if "1m" in workload else "see world_b200/scenes.py",
        "collision_grid": [spec.collision_grid_size_x, spec.collision_grid_size_y,
                           spec.collision_grid_size_z],
        "cic_grid": spec.density_grid_size_x,
        "dt": spec.dt,
        "l2": "flushed (512 MiB write) before every timed step, flush not timed",
    }
    if scenes is not None:
        out["scenes"] = scenes
        out["diameters"] = "uniform [0.9d, 1.1d]"
        out["collision_grid"] = "per scene (world_b200/scenes.py)"
        out["mu"] = "per scene" if workload == "design_256" else spec.physics.friction
    return out


# ------------------------------------------------------------------ clocks -------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, indices):
        self.indices = set(indices)
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        # the timed region starts only once the sampler is producing samples
        t0 = time.time()
        while time.time() - t0 < 10.0 and self.proc.poll() is None:
            self.fh.flush()
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.02)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    idx = int(parts[0])
                except ValueError:
                    continue
                if idx not in self.indices:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for name, val in zip(names, parts[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_hbm_peak() -> tuple[float, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            v = float(json.load(f)["hbm_gbs"])
        return v, "measured"
    except (OSError, KeyError, ValueError, TypeError):
        return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(workload: str, kernel: str):
    """DRAM bytes per contact-kernel launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "contact_kernel_traffic.json")
    try:
        with open(path) as f:
            data = json.load(f)
        entry = data.get(workload)
        return entry.get(kernel) if isinstance(entry, dict) else None
    except (OSError, ValueError):
        return None


# ------------------------------------------------------------------ CPU side -----
def _oracle_sim(scene, threads: int):
    from oracle.oracle import OracleSim, lib as oracle_lib, params_from_config
    from world_b200.scenes import grain_properties
    import numpy as np
    oracle_lib().dem_set_num_threads(threads)
    material = np.full(scene.n, scene.spec.particle_material, np.int32)
    radius, mass = grain_properties(scene.spec, material, scene.radius)
    return OracleSim(params_from_config(scene.spec), scene.state, radius, mass), \
        oracle_lib().dem_num_threads()


def cpu_oracle_rate(scene, seconds: float, max_steps: int, warmup: int = 1,
                    threads: int | None = None):
    """The oracle port on the host cores (all unless `threads`): (grain-steps/s, steps,
    elapsed, threads)."""
    sim, used = _oracle_sim(scene, threads or os.cpu_count() or 1)
    for _ in range(max(0, warmup)):
        sim.step()
    steps = 0
    t0 = time.perf_counter()
    while steps < max_steps and (steps == 0 or time.perf_counter() - t0 < seconds):
        sim.step()
        steps += 1
    elapsed = time.perf_counter() - t0
    return scene.n * steps / elapsed, steps, elapsed, used


def run_reference(args) -> int:
    """The reference arm: the oracle port on all host cores (module docstring)."""
    rank = env_int("RANK", 0)
    if rank != 0:
        return 0
    from world_b200.scenes import BATCHED_WORKLOADS, scene_for
    if args.workload in BATCHED_WORKLOADS or args.workload == "adjoint_32k":
        print(json.dumps({"impl": "reference", "unavailable":
                          f"the reference arm times single-scene workloads only ({args.workload})"}))
        return 0
    scene = scene_for(args.workload, n=args.grains, seed=12345)
    sim, threads = _oracle_sim(scene, os.cpu_count() or 1)
    for _ in range(args.warmup):
        sim.step()
    # one step gives the rate; K is capped so the run ends within about four minutes
    t0 = time.perf_counter()
    sim.step()
    first = time.perf_counter() - t0
    steps = max(1, min(args.steps, int(240.0 / max(first, 1e-6))))
    t0 = time.perf_counter()
    for _ in range(steps):
        sim.step()
    elapsed = time.perf_counter() - t0
    rate = scene.n * steps / elapsed
    sample = (f"{steps} of {args.steps} requested steps of the full {scene.n}-grain workload "
              f"after {args.warmup} untimed warm-up steps ({elapsed:.1f} s on {threads} host "
              "threads); the reference's step is CUDA only, so this is its algorithm "
              "restated in C (oracle/dem_oracle.c)")
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT,
        "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * elapsed / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
        "data": "synthetic (seeded column collapse, world_b200/scenes.py)",
        "config": workload_config(scene.spec, args.workload, scene.n),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU side -----
class L2Flush:
    """Untimed L2 flush queued before a step: a 512 MiB write (larger than L2)."""

    def __init__(self):
        import torch
        self.buf = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def __call__(self, k: int) -> None:
        self.buf.fill_(float(k))


def _timed_steps(sim, stream, flush, steps: int) -> float:
    """Device time (ms) of `steps` steps: each an L2 flush (L2Flush) queued on the
    library's stream, then the step bracketed by events on that stream. Nothing syncs
    the host inside the loop, so launches run ahead of the GPU and the events time only
    the steps."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush(k)
            ev[k][0].record(stream)
            sim.take_step()
            ev[k][1].record(stream)
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in ev)


def _resorts(sim) -> int:
    """Grains whose contacts a cell crossing re-ordered so far (0 where the library
    predates the counter)."""
    try:
        return sim.list_resort_count()
    except AttributeError:
        return 0


def _build_cost(sim, stream, flush, steps: int) -> dict | None:
    """Cost of a list build inside the step graph: `steps` steps one at a time (L2 flushed
    before each, events around each), each classed by whether the build counter moved
    during it; the build's cost is the mean step with a build minus the mean without."""
    import torch
    if sim.tuning()["neighbor_skin_m"] <= 0:
        return None
    with_b, without = [], []
    radix0 = sim.radix_search_count()[0]
    for k in range(steps):
        b0 = sim.list_stats()[0]
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            flush(k)
            a.record(stream)
            sim.take_step()
            b.record(stream)
        b.synchronize()
        (with_b if sim.list_stats()[0] > b0 else without).append(a.elapsed_time(b))
    radix = sim.radix_search_count()[0] - radix0
    if not with_b or not without:
        return {"steps": steps, "builds": len(with_b), "radix_builds": radix, "build_ms": None}
    return {"steps": steps, "builds": len(with_b), "radix_builds": radix,
            "step_ms_without_build": statistics.mean(without),
            "build_ms": statistics.mean(with_b) - statistics.mean(without)}


def _contact_roofline(sim, stream, flush, spec, phase_steps: int, direct: bool) -> dict:
    """The contact kernel's algorithmic bytes per launch over its event-timed duration,
    from a direct-launch pass of `phase_steps` steps of the same workload (L2 flushed
    before each step)."""
    import numpy as np
    import torch
    n = sim.n
    lists = sim.tuning()["neighbor_skin_m"] > 0
    picard = spec.time_integrator != "semi_implicit_euler"
    sim.set_kernel_timing(True)
    iters0 = sim.picard_counts()[0]
    t0 = sim._timings()
    builds0 = sim.list_stats()[0]
    exact0 = sim.list_exact_count()
    resort0 = _resorts(sim)
    with torch.cuda.stream(stream):
        for k in range(phase_steps):
            flush(k)
            sim.take_step()
    sim.synchronize()
    t1 = sim._timings()
    sim.set_kernel_timing(direct)
    build_frac = (sim.list_stats()[0] - builds0) / phase_steps
    resort_frac = (_resorts(sim) - resort0) / (phase_steps * sim.n)
    exact_frac = (sim.list_exact_count() - exact0) / phase_steps
    search_ms = float(t1[0] - t0[0]) / phase_steps
    contact_ms = float(t1[1] - t0[1]) / phase_steps
    # backward Euler / Picard: the timed contact phase is the whole step, one contact
    # launch per executed iteration (plus, without lists, each iteration's search)
    phase_iters = (sim.picard_counts()[0] - iters0) / phase_steps if picard else 1.0
    mean_list = sim.list_stats()[2]
    cnt, _, _ = sim.get_history()
    entries = int(cnt.astype(np.int64).sum())
    # contact kernel, algorithmic bytes per launch. Searched step: read x,r / v,m / id
    # (36 B) and write x,r / v,m / id / a (52 B) per grain. History rows read and
    # written (16 B per entry each way) plus the per-grain counts (4 B each way).
    hist_bytes = (2 * 16 * entries + 8 * n) if spec.history else 0
    if not lists:
        contact_bytes = 88 * n + hist_bytes
    elif not picard:
        # lists, semi-implicit Euler: read x,r / v,m / id and the list count (40 B), the
        # list (4 B per entry), the build position on the steps that measure it; write
        # x,r / v,m / a (48 B) and the id only on the step after a build
        contact_bytes = int(88 * n + hist_bytes + 4 * mean_list * n + 16 * n * exact_frac
                            + 4 * n * build_frac)
    else:
        # lists, one Picard iteration: as the searched step plus the list count, the
        # build position, the step-start state (32 B) and the rhs copy (20 B)
        contact_bytes = int(88 * n + hist_bytes + 4 * mean_list * n + 72 * n)
    kernel_ms = contact_ms / phase_iters
    achieved = contact_bytes / (kernel_ms / 1e3) / 1e9
    peak, peak_kind = measured_hbm_peak()
    variant = sim.tuning()["contact_variant"]
    symbol = ("k_force_list_staged" if variant.startswith("bulk-staged") else
              "k_force_list_coop" if variant.startswith("warp-cooperative") else
              "k_force_list") if lists else "k_force"
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "symbol": symbol,
            "kernel": (f"{symbol} (contacts from Verlet lists + integrator; {variant})" if lists
                       else "k_force (contact forces + integrator)"),
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
            if peak_kind == "measured" else "fallback 6.65 TB/s",
            "algorithmic_bytes_per_launch": contact_bytes,
            "measuring_step_fraction": exact_frac if lists else None,
            "build_step_fraction": build_frac if lists else None,
            "kernel_ms": kernel_ms, "search_ms": search_ms,
            "history_entries_per_grain": entries / n,
            "mean_list_length": mean_list if lists else None,
            "resorted_grain_fraction": resort_frac if lists else None}


def _fields(sim, stream, flush, reps: int) -> dict:
    """The CIC deposit into a device grid (wd_compute_density_grid_device) and the total
    energy (wd_compute_total_energy: a search and gather of the current state, the FP64
    per-grain terms and their sums) of the current state, each bracketed by events on the
    library's stream after an L2 flush; medians over `reps`."""
    import torch
    from world_b200._lib import check, lib, ptr
    nodes = sim.density_grid_nodes()
    grid = torch.empty(4 * nodes, dtype=torch.float32, device="cuda")
    dep, en = [], []
    for k in range(reps):
        for fn, acc in ((lambda: check(lib.wd_compute_density_grid_device(sim.handle, ptr(grid)))
                         , dep), (sim.compute_total_energy, en)):
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                flush(k)
                a.record(stream)
                fn()
                b.record(stream)
            b.synchronize()
            acc.append(a.elapsed_time(b))
    return {"deposit_ms": statistics.median(dep), "energy_ms": statistics.median(en),
            "cic_nodes": nodes, "reps": reps,
            "note": "energy includes the search and gather of the current state and an "
                    "8-byte copy to the host"}


def _settled(sim, scene, stream, flush, args, plain_value: float, done: int,
             total_steps: int) -> dict:
    """The same column once it has collapsed onto the floor: advance the plain run from
    `done` to `total_steps` steps from rest, re-tune, then time K steps and the contact
    kernel's roofline as for the headline."""
    import torch
    t0 = time.perf_counter()
    sim.advance(max(0, total_steps - done))
    sim.synchronize()
    preroll_s = time.perf_counter() - t0
    tuned = None
    if args.skin < 0:
        sim.autotune(steps=40)
        tuned = sim.tuning()
    sim.advance(args.warmup)
    builds0 = sim.list_stats()[0]
    ms = _timed_steps(sim, stream, flush, args.steps)
    builds = sim.list_stats()[0] - builds0
    value = sim.n * args.steps / (ms / 1e3)
    roof = _contact_roofline(sim, stream, flush, scene.spec, args.phase_steps, args.direct)
    build = _build_cost(sim, stream, flush, args.build_steps) if args.build_steps > 0 else None
    torch.cuda.synchronize()
    return {"value": value, "unit": UNIT, "ms_per_step": ms / args.steps, "build": build,
            "steps": args.steps, "after_steps": total_steps,
            "pre_roll_seconds": preroll_s, "over_plain": value / plain_value,
            "builds_timed": builds, "mean_list_length": roof["mean_list_length"],
            "history_entries_per_grain": roof["history_entries_per_grain"],
            "roofline": {k: roof[k] for k in ("achieved", "peak", "frac", "kernel",
                                               "algorithmic_bytes_per_launch", "kernel_ms",
                                               "measuring_step_fraction",
                                               "build_step_fraction",
                                               "resorted_grain_fraction")},
            "autotuned": tuned}


def _batched(workload: str, args, flush, plain_value: float,
             settled_plain: float | None = None) -> dict:
    """One batched ensemble on this GPU: every scene in one SceneBatch, the autotuner's
    schedule, K timed steps with the L2 flushed before each; then the same batch once
    its columns have collapsed (`settled_steps` steps from rest, re-tuned), K timed steps
    against the plain column's settled value."""
    import torch
    from world_b200 import SceneBatch
    from world_b200.scenes import ensemble_for
    t0 = time.perf_counter()
    members = ensemble_for(workload)
    batch = SceneBatch.from_scenes(members)
    setup_s = time.perf_counter() - t0
    batch.autotune(steps=20) if args.skin < 0 else batch.set_neighbor_skin(max(args.skin, 0.0))
    stream = torch.cuda.ExternalStream(batch.stream_ptr())
    batch.advance(args.warmup)
    batch.synchronize()
    ms = _timed_steps(batch, stream, flush, args.steps)
    value = batch.n * args.steps / (ms / 1e3)
    out = {"value": value, "unit": UNIT, "scenes": len(members), "grains": batch.n,
           "ms_per_step": ms / args.steps, "steps": args.steps, "over_plain": value / plain_value,
           "setup_seconds": setup_s, "schedule": batch.tuning(),
           "mean_list_length": batch.list_stats()[2]}
    if settled_plain:
        t0 = time.perf_counter()
        batch.advance(max(0, args.settled_steps - args.warmup - args.steps))
        batch.synchronize()
        preroll_s = time.perf_counter() - t0
        if args.skin < 0:
            batch.autotune(steps=20)
        batch.advance(args.warmup)
        ms = _timed_steps(batch, stream, flush, args.steps)
        v = batch.n * args.steps / (ms / 1e3)
        out["settled"] = {"value": v, "ms_per_step": ms / args.steps,
                          "after_steps": args.settled_steps, "pre_roll_seconds": preroll_s,
                          "over_plain_settled": v / settled_plain, "schedule": batch.tuning(),
                          "mean_list_length": batch.list_stats()[2]}
    batch.close()
    return out


def run_ours(args) -> int:
    import numpy as np
    import torch
    import torch.distributed as dist

    from world_b200 import ParticleDynamics, SceneBatch
    from world_b200._lib import check, lib, ptr
    from world_b200.batch import shard_scenes
    from world_b200.scenes import BATCHED_WORKLOADS, ensemble_for, scene_for

    rank, world, local = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180),
                                device_id=torch.device("cuda", local))

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def barrier():
        if world > 1:
            dist.barrier()

    scenes_total = None
    if args.workload in BATCHED_WORKLOADS:
        # scenes shared out over the ranks, balanced by grain count; each rank steps
        # its share as one batch
        members = ensemble_for(args.workload)
        mine = shard_scenes([m.n for m in members], world)[rank]
        for i in mine:
            members[i].cfg.neighbor_skin = max(args.skin, 0.0)
        sim = SceneBatch.from_scenes([members[i] for i in mine])
        scene = members[mine[0]]
        scenes_total = len(members)
    else:
        scene = scene_for(args.workload, n=args.grains, seed=12345 + rank)
        scene.cfg.neighbor_skin = max(args.skin, 0.0)
        if args.checkpoint and not args.save_after:
            sim = ParticleDynamics.from_checkpoint(scene.cfg, args.checkpoint)
        else:
            sim = ParticleDynamics(scene.cfg, state=scene.state, radius=scene.radius)
        if args.save_after:
            # a contact-bearing starting point for profilers: K steps from rest, saved
            if not args.checkpoint:
                raise SystemExit("--save-after needs --checkpoint PATH")
            sim.advance(args.save_after)
            sim.write_checkpoint(args.checkpoint)
            cnt = sim.get_history()[0]
            print(json.dumps({"checkpoint": args.checkpoint, "steps": args.save_after,
                              "grains": sim.n, "springs_per_grain": float(cnt.sum()) / sim.n}))
            sim.close()
            return 0
    sim.set_kernel_timing(args.direct)
    tuned = None
    if args.skin < 0:
        # the autotuner picks the skin and the contact kernel's block size (untimed;
        # the state is restored and the results do not depend on the choice)
        sim.autotune(steps=40)
        tuned = sim.tuning()
    elif args.contact_kernel:
        block, variant = (int(v) for v in args.contact_kernel.split(","))
        sim.set_contact_kernel(block, variant)
    skin = sim.tuning()["neighbor_skin_m"]
    lists = skin > 0
    n = sim.n
    stream = torch.cuda.ExternalStream(sim.stream_ptr())
    flush = L2Flush()

    sim.advance(args.warmup)
    sim.synchronize()
    barrier()

    sampler = ClockSampler(range(world) if world > 1 else [local]) if rank == 0 else None
    if sampler:
        sampler.start()
    torch.cuda.synchronize()
    radix0, radix_each = sim.radix_search_count()
    builds0, build_kernels, _ = sim.list_stats()
    picard = scene.spec.time_integrator != "semi_implicit_euler"
    iters0, redos0 = sim.picard_counts()
    barrier()
    local_ms = _timed_steps(sim, stream, flush, args.steps)
    barrier()
    clocks = sampler.stop() if sampler else None
    radix_searches = sim.radix_search_count()[0] - radix0
    builds, _, mean_list = sim.list_stats()
    builds -= builds0
    iters1, redos1 = sim.picard_counts()
    # list mode: a build launches the whole search (its radix kernels gated) and the
    # list kernels; otherwise a search adds the radix kernels only when it takes them
    launches = sim.kernels_per_step() * args.steps + (
        builds * build_kernels if lists else radix_searches * radix_each)
    total_ms = max_over_ranks(local_ms)
    all_grains = n
    if world > 1:
        t = torch.tensor([float(n)], dtype=torch.float64, device="cuda")
        dist.all_reduce(t)
        all_grains = int(t.item())
    value = all_grains * args.steps / (total_ms / 1e3)

    roof = _contact_roofline(sim, stream, flush, scene.spec, args.phase_steps, args.direct)
    roof["traffic"] = profiled_traffic(args.workload, roof["symbol"])
    fields = _fields(sim, stream, flush, args.field_reps) if args.field_reps > 0 else None

    # e2e through the C ABI with pinned host buffers: every step uploads its state and
    # downloads its positions; the asynchronous calls overlap the upload of one step
    # with the step before and the download of the one before that
    h_state = torch.from_numpy(sim.get_state()).pin_memory()
    h_pos = [torch.empty(3 * n, dtype=torch.float32).pin_memory() for _ in range(2)]
    sim.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    check(lib.wd_get_state(sim.handle, ptr(h_state)))
    for k in range(2):   # untimed: copy streams, staging buffers, first touch of the pages
        check(lib.wd_set_state_async(sim.handle, ptr(h_state)))
        check(lib.wd_step(sim.handle, 1))
        check(lib.wd_get_positions_async(sim.handle, ptr(h_pos[k % 2])))
    check(lib.wd_synchronize(sim.handle))
    e0.record(stream)
    check(lib.wd_io_join(sim.handle))
    for k in range(args.e2e_steps):
        check(lib.wd_set_state_async(sim.handle, ptr(h_state)))
        check(lib.wd_step(sim.handle, 1))
        check(lib.wd_get_positions_async(sim.handle, ptr(h_pos[k % 2])))
    check(lib.wd_io_join(sim.handle))
    e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e_value = all_grains * args.e2e_steps / (e2e_ms / 1e3)

    scene_results = None
    if scenes_total:
        # per-scene energies of every rank's shard, gathered (the batched workloads'
        # only exchange: a final gather of per-scene results)
        from world_b200.batch import gather_scene_values
        energies = sim.scene_energies()
        if world > 1:
            energies = gather_scene_values(energies, mine, scenes_total)[:, 0]
        scene_results = {"scenes": int(len(energies)), "energy_sum_J": float(np.sum(energies)),
                         "energy_min_J": float(np.min(energies))}

    # contact-bearing regime, batched ensembles and the reverse pass beside the plain
    # step (one GPU, default workload only)
    extras = world == 1 and not args.no_extras and args.workload == "collapse_1m_sie_mu05" \
        and args.grains is None
    settled = batched = adjoint = None
    if extras:
        # steps from rest so far: warm-up, timed, roofline pass, and the last e2e step
        # (each e2e step restarts from the same uploaded state)
        done = args.warmup + args.steps + args.phase_steps + 1
        settled = _settled(sim, scene, stream, flush, args, value, done, args.settled_steps)
    sim.close()
    if extras and not args.settled_only:
        batched = {w: _batched(w, args, flush, value, settled["value"] if settled else None)
                   for w in BATCHED_WORKLOADS}
        adjoint = adjoint_measure(args, plain_value=value)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, steps, elapsed, threads = cpu_oracle_rate(scene, args.cpu_seconds, 10_000)
        rate1, steps1, elapsed1, _ = cpu_oracle_rate(scene, max(2.0, args.cpu_seconds / 3), 10_000,
                                                     warmup=0, threads=1)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{steps} steps of the same {n}-grain workload on {threads} host "
                         f"threads ({elapsed:.1f} s), oracle/dem_oracle.c with OpenMP",
               "one_core": {"value": rate1, "steps": steps1, "seconds": elapsed1}}

    if rank == 0:
        roofline = {k: roof[k] for k in ("bound", "achieved", "peak", "unit", "frac", "traffic",
                                         "kernel", "peak_source", "algorithmic_bytes_per_launch",
                                         "measuring_step_fraction", "build_step_fraction",
                                         "kernel_ms", "search_ms",
                                         "resorted_grain_fraction")}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "strong" if scenes_total else "weak", "vs_baseline": None,
            "dtype": "fp32",
            "data": "synthetic (seeded column collapse, world_b200/scenes.py)",
            "config": workload_config(scene.spec, args.workload, all_grains, scenes=scenes_total),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 24 * n,
                    "d2h_bytes_per_step": 12 * n, "steps": args.e2e_steps},
            "clocks": clocks,
            "fields": fields,
            "gpu_launches": launches,
            "radix_searches_timed": radix_searches,
            "neighbor_lists": {"skin_m": skin, "builds_timed": builds,
                               "mean_list_length": mean_list} if lists else None,
            "picard": {"iterations_per_step": (iters1 - iters0) / args.steps,
                       "redone_steps_timed": redos1 - redos0} if picard else None,
            "history_entries_per_grain": roof["history_entries_per_grain"],
            "scene_results": scene_results,
            "autotuned": tuned,
            "settled": settled,
            "batched": batched,
            "adjoint": adjoint,
        }
        print(json.dumps(line), flush=True)
    del flush
    if world > 1:
        dist.destroy_process_group()
    return 0


def adjoint_measure(args, plain_value: float | None = None) -> dict:
    """Gradient of a density loss over a 200-step window of the 32,768-grain column
    after 12,000 steps (0.12 s: the lower layers have reached the floor and the column
    is collapsing; before about 2,700 steps the lattice falls without a contact): loss =
    mean((rho_64^3(T) - rho_target)^2), target from the same window with mu = 0.4,
    e = 0.6; gradients in v0 and (mu, e, k_n). The window's reverse pass in grain-steps/s
    and its cost relative to the plain forward window on the same GPU."""
    import torch

    from world_b200 import ParticleDynamics
    from world_b200.adjoint import deposit, window
    from world_b200.scenes import column_collapse

    scene = column_collapse(32768, diameters="uniform", cic=64)
    cfg = scene.cfg
    cfg.kernel_timing = False
    ph = cfg.physics
    mu, e, k = float(ph.friction), float(ph.restitution), float(ph.normal_stiffness)
    sim = ParticleDynamics(cfg, state=scene.state, radius=scene.radius)
    pre_roll = 12000
    sim.advance(pre_roll)
    start = torch.from_numpy(sim.get_state()).cuda().reshape(-1, 6)
    springs = sim.get_history()   # every window starts from the pre-rolled springs
    x0, v0 = start[:, :3].contiguous(), start[:, 3:].contiguous()
    steps, every = 200, 20
    stream = torch.cuda.ExternalStream(sim.stream_ptr())

    def timed(fn):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        out = fn()
        b.record(stream)
        torch.cuda.synchronize()
        return out, a.elapsed_time(b)

    # target field: the same window with mu = 0.4, e = 0.6
    sim.set_contact_params(0.4, 0.6, k)
    sim.set_state_tensor(start.reshape(-1))
    sim.set_history(*springs)
    sim.advance(steps)
    sim.compute_density_grid()
    target = torch.from_numpy(sim.host_density_grid[:sim.density_grid_nodes()].copy()).cuda()
    target = target.reshape(cfg.density_grid_size_x, cfg.density_grid_size_y, cfg.density_grid_size_z)
    sim.set_contact_params(mu, e, k)
    for _ in range(max(1, args.warmup // 3)):
        sim.set_state_tensor(start.reshape(-1))
        sim.set_history(*springs)
        sim.advance(steps)
    sim.set_state_tensor(start.reshape(-1))
    sim.set_history(*springs)
    _, fwd_ms = timed(lambda: sim.advance(steps))

    def gradient():
        sim.set_history(*springs)
        tv0 = v0.clone().requires_grad_(True)
        theta = torch.tensor([mu, e, k], dtype=torch.float64, requires_grad=True)
        (x, v), rec_ms = timed(lambda: window(sim, x0, tv0, theta, steps, every))
        grid = deposit(sim, x, v)
        loss = ((grid[0].double() - target.double()) ** 2).mean()
        _, bwd_ms = timed(lambda: loss.backward())
        return tv0, theta, loss, rec_ms, bwd_ms

    gradient()   # untimed: allocates the checkpoints and the tape, captures the graphs
    tv0, theta, loss, rec_ms, bwd_ms = gradient()
    n = sim.n
    sim.close()
    out = {
        "value": n * steps / (bwd_ms / 1e3), "unit": "grain-steps/s (reverse pass)",
        "grains": n, "pre_roll_steps": pre_roll, "window_steps": steps,
        "checkpoint_every": every, "cic_grid": 64,
        "loss_definition": "mean((rho_T - rho_target)^2), target mu=0.4 e=0.6",
        "forward_window_ms": fwd_ms, "record_ms": rec_ms, "backward_ms": bwd_ms,
        "record_over_forward": rec_ms / fwd_ms, "backward_over_forward": bwd_ms / fwd_ms,
        "gradient_over_forward": (rec_ms + bwd_ms) / fwd_ms,
        "loss": float(loss.detach()),
        "grad_theta": theta.grad.tolist(),
        "grad_v0_norm": float(tv0.grad.norm()),
    }
    if plain_value is not None:
        out["forward_window_grain_steps_per_s"] = n * steps / (fwd_ms / 1e3)
    return out


def run_adjoint(args) -> int:
    """--workload adjoint_32k: adjoint_measure() as its own line. One GPU."""
    import torch
    if env_int("RANK", 0) != 0:
        return 0
    torch.cuda.set_device(env_int("LOCAL_RANK", 0))
    out = adjoint_measure(args)
    line = {"metric": "adjoint grain-steps/s, 200-step window at 32,768 grains FP32",
            "value": out["value"], "unit": "grain-steps/s", "n_gpus": 1,
            "steps": out["window_steps"], "warmup": args.warmup, "higher_is_better": True,
            "dtype": "fp32", "data": "synthetic (seeded column collapse, world_b200/scenes.py)",
            "config": {"workload": "adjoint_32k", "grains": out["grains"],
                       "pre_roll_steps": out["pre_roll_steps"],
                       "window_steps": out["window_steps"],
                       "checkpoint_every": out["checkpoint_every"], "cic_grid": 64,
                       "loss": out["loss_definition"]}}
    line.update({k: v for k, v in out.items() if k not in ("value", "unit")})
    print(json.dumps(line), flush=True)
    return 0


def main() -> int:
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "adjoint_32k":
        return run_adjoint(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
