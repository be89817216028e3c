#!/usr/bin/env python
"""Benchmark of the MLS-MPM step on B200: particle-steps/s.

One unit of the metric is one particle advanced through one substep (P2G, grid update,
G2P + constitutive update); a benchmark "step" is one `Simulation::step()` call (one frame
of config.dt = 0.05, with as many CFL-limited substeps as the reference loop takes).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

Default workload: the mixed granular scene the metric is quoted on (~4M particles in seeded
blocks of DruckerPrager sand, Stomakhin snow and NACC soil at 4 particles per cell on a 1024^2
grid), with the learned return-mapping closure timed on the same scene in the same line
(`learned_closure`: its rate, its ratio to the plain step and its judged stress error).  Inputs are resident in HBM when the timed region starts; L2 is
flushed (512 MiB device write) before every timed step.  `e2e` repeats the measurement
through the C ABI with the particle state uploaded from pinned host memory before and read
back (asynchronously, overlapping the next upload) after every step.  `--impl reference` times the CPU oracle (the reference step restated
in C++) on the host cores instead.  Under torchrun each rank runs an independent replica
(replicas only: the single-scene step does not shard), timed on the device, max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "particle-steps/s on 1 B200 (plain CUDA vs learned closure at stated error) vs CPU"
UNIT = "particle-steps/s"

WORKLOADS = {
    "dam_break_1m": dict(builder="dam_break", kwargs=dict(grid_res=1024, column=512),
                         desc="dam break: 512x512-cell water column, 4 ppc, 1024^2 grid, "
                              "NewtonianFluid Tait rho0=1000 k=1e4 gamma=7, SlipBoundary(2), "
                              "dt=0.05, adaptive CFL substeps",
                         material="NewtonianFluid", grid_res=1024),
    "dam_break_262k": dict(builder="dam_break", kwargs=dict(grid_res=512, column=256),
                           desc="dam break: 256x256-cell water column, 4 ppc, 512^2 grid",
                           material="NewtonianFluid", grid_res=512),
    "mixed_granular_4m": dict(builder="mixed_granular",
                              kwargs=dict(grid_res=1024, target_particles=4_000_000),
                              desc="mixed granular: seeded blocks 16-128 cells, DruckerPrager / "
                                   "Stomakhin snow / NACC, 4 ppc, 1024^2 grid",
                              material="DP+Snow+NACC", grid_res=1024),
    "material_zoo_4m": dict(builder="model_blocks",
                            kwargs=dict(grid_res=1024, target_particles=4_000_000),
                            desc="the seven further constitutive models at scale: seeded blocks "
                                 "16-128 cells, each Corotated / VonMises / Rankine / mu(I) / "
                                 "Viscoelastic / GranularFluid / Bingham, 4 ppc, 1024^2 grid",
                            material="ZOO7", grid_res=1024),
    "material_zoo_1m": dict(builder="model_blocks",
                            kwargs=dict(grid_res=512, target_particles=1_000_000),
                            desc="material_zoo_4m's generator on a 512^2 grid with 1M particles "
                                 "(profiling case)",
                            material="ZOO7", grid_res=512),
    "fields_asflip_1m": dict(builder="field_dam_break", kwargs=dict(grid_res=1024, column=512),
                             desc="dam break 1M with ASFLIP (blend 0.5) and three force fields "
                                  "(gravity well with cutoff, linear drag, radial confinement)",
                             material="NewtonianFluid+fields", grid_res=1024),
    "nbody_160k": dict(builder="nbody_scene", kwargs=dict(grid_res=512, scale=8, G=1.0),
                       desc="self-gravitating NeoHookean clumps (blocks of 144, 112 and 80 cells at "
                            "4 ppc, 158,720 particles) under NBodyGravityField(G 1, softening 1, "
                            "theta 0.5, depth 8, 4 bodies per leaf), no gravity, 512^2 grid",
                       material="NeoHookean-nbody", grid_res=512),
    "sleep_slab_1m": dict(builder="sleep_slab", kwargs=dict(grid_res=1024, slab=768),
                          desc="sleep partition: NeoHookean 768 x 384-cell slab at 4 ppc "
                               "(1.18M particles, asleep after its first substep) and a disk of "
                               "radius 40 launched into it; units count awake particles only",
                          material="NeoHookean-sleep", grid_res=1024, active_units=True),
    "contact_1m": dict(builder="contact_slab", kwargs=dict(grid_res=1024),
                       desc="multi-field contact: NeoHookean 896 x 192-cell slab on the floor and a "
                            "320 x 256-cell grip block (contact_group 1) on it thrown at (1.5, -3), "
                            "4 ppc, DirectionalContactGrip(0.1, 0.9, (1, 0)); fused pipeline (field "
                            "sums with the total, per-base-cell point lists, LR contact normals)",
                       material="NeoHookean-contact", grid_res=1024),
    "mixture_1m": dict(builder="mixture_overlap", kwargs=dict(grid_res=1024, side=362, iterations=0),
                       desc="two-phase mixture without gravity: DruckerPrager sand (solid phase) and "
                            "water (fluid phase) squares of 362 x 362 cells at 4 ppc each, "
                            "overlapping, water at (0, -3), drag 5, no pressure projection; "
                            "fused pipeline (phase sums with the total)",
                       material="DP+NewtonianFluid-mixture", grid_res=1024),
    "batched_256": dict(builder="batched_scenes", kwargs=dict(n_scenes=256, pair_sizes=True),
                        desc="256 independent scenes in one batch: grid G ~ U{64..256}, "
                             "N ~ logU[4k, 200k] particles, the two draws paired by rank so every "
                             "block fits at 4 ppc (~12.8M particles), material uniform over "
                             "{NewtonianFluid, DruckerPrager, Stomakhin snow, NeoHookean}, block on "
                             "the floor, SlipBoundary(2), dt=0.05; autotuned tile shape, particles "
                             "per CTA, sort interval and P2G aggregation (on-disk cache)",
                        material="batched", grid_res=0),
}
DEFAULT_WORKLOAD = "mixed_granular_4m"

# Algorithmic bytes per particle of one launch of the fused particle pass (k_particle):
# the hot state it must read and write once per substep, plus its share of grid traffic
# (grid velocity gather 8 B/cell, mass+momentum+stress reductions 24 B/cell, 4 ppc).
#   fluid:    read x8 v8 C16 F16 m4 V0 4 V4 rho4 mat4 plastic16 rho_dp4 = 88,
#             write x8 v8 C16 V4 rho4 = 40, grid 32/4 = 8              -> 136 B
#   granular: read 84, write x8 v8 C16 F16 V4 rho4 plastic16 = 72, grid 8 -> 164 B
#   NeoHookean: read x8 v8 C16 F16 m4 V0 4 V4 rho4 mat4 = 68, write x8 v8 C16 F16 V4 rho4 = 56,
#             contact group 4, grid 8                                  -> 136 + 20 (sleep flag,
#             field velocities) = 156 B
#   mixture:  the mean of the granular (164) and fluid (136) particles    -> 150 B
# k_density per particle (fluid scenes): read x8 mat4 C16 mass4, write rho_dp 4, grid
# (mass gather 4 B + stress reduction 8 B per cell) / 4 ppc = 3                   -> 39 B
K_DENSITY_BYTES = 39
K_PARTICLE_BYTES = {"NewtonianFluid": 136, "DP+Snow+NACC": 164, "ZOO7": 164, "NeoHookean-nbody": 156,
                    "NewtonianFluid+fields": 136, "NeoHookean-sleep": 156,
                    "NeoHookean-contact": 156, "DP+NewtonianFluid-mixture": 150}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(workload: str):
    """DRAM bytes per k_particle launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", f"k_particle_{workload}.md")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", f.read())
    return float(m.group(1)) if m else None


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons, read through NVML (the library behind
    nvidia-smi) every 5 ms on a background thread while the benchmark runs.  Reading only;
    nothing is set.  Falls back to `nvidia-smi -lms 200` where NVML is unavailable."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local_rank: int):
        self.local_rank = local_rank
        self.samples = []  # (time, sm MHz, set of reason names)
        self.max_mhz = None
        self.source = None
        self._stop = threading.Event()
        self.thread = None
        self.proc = None

    def _nvml_handle(self, nv):
        ident = str(self.local_rank)
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        if vis:
            items = [v.strip() for v in vis.split(",") if v.strip()]
            if self.local_rank < len(items):
                ident = items[self.local_rank]
        if ident.startswith("GPU-") or ident.startswith("MIG-"):
            return nv.nvmlDeviceGetHandleByUUID(ident)
        return nv.nvmlDeviceGetHandleByIndex(int(ident))

    def start(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._nvml_handle(nv)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
        except Exception:
            self._start_smi()
            return
        self.source = "nvml (5 ms)"

        def run():
            while not self._stop.is_set():
                try:
                    mhz = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                    bits = int(get_reasons(h))
                except Exception:
                    break
                names = {k for k, b in self.REASONS.items() if bits & b}
                self.samples.append((time.perf_counter(), mhz, names))
                self._stop.wait(0.005)

        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()

    def _start_smi(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-i", str(self.local_rank), "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self.source = "nvidia-smi (200 ms)"
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

        def run():
            for line in self.proc.stdout:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    mhz, self.max_mhz = float(parts[1]), float(parts[2])
                except ValueError:
                    continue
                self.samples.append((time.perf_counter(), mhz,
                                     {n for n, v in zip(names, parts[5:9]) if v.lower() == "active"}))

        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()

    def stop(self, t_begin: float, t_end: float, t_load: float) -> dict | None:
        """Summary of the samples taken in [t_begin, t_end] (the timed region); when that
        window holds fewer than 3 samples, of [t_load, t_end] (warm-up included)."""
        self._stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        window = "timed region"
        sel = [s for s in self.samples if t_begin <= s[0] <= t_end]
        if len(sel) < 3:
            sel = [s for s in self.samples if t_load <= s[0] <= t_end]
            window = "warm-up + timed region"
        if not sel:
            return None
        reasons = sorted(set().union(*(s[2] for s in sel)))
        return {"sm_mhz": statistics.median(s[1] for s in sel), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(sel), "window": window,
                "source": self.source}


def _timed_frames(sim, steps: int) -> tuple:
    """(device ms, substeps) of `steps` frames, L2 flushed before each (the main loop's
    timing)."""
    sub0 = sim.stats()["substeps"]
    total_ms = 0.0
    for _ in range(steps):
        sim.flush_l2()
        sim.event_record(0)
        sim.step()
        sim.event_record(1)
        total_ms += sim.event_elapsed_ms(0, 1)
    return total_ms, sim.stats()["substeps"] - sub0


def closure_ab(sim, n: int, steps: int, plain_value: float) -> dict:
    """Learned return-mapping closure on the same scene: log the plain mapping for one step,
    train the networks with the library's kernels, then time `steps` frames of the plain step
    and `steps` frames with the closure on, both from the same particle state (each after an
    untimed frame from that state), and report the closure's live judged error."""
    sim.closure_log(2_000_000, 8)
    sim.step()
    sim.closure_log(0, 1)
    logged = sim.closure_stats()["logged"]
    train = {}
    for model, name in ((0, "drucker_prager"), (1, "nacc")):
        if logged[model] < 1024:
            train[name] = {"samples": int(logged[model]), "trained": False,
                           "note": "too few samples on the smooth plastic branch"}
            continue
        rep = sim.closure_train(model, epochs=20, batch=8192, lr=3e-3, lr_decay=0.9, seed=1)
        train[name] = {"trained": True, "samples": int(rep["n_train"] + rep["n_val"]),
                       "epochs": 20, "seconds": rep["seconds"], "val_err_mean": rep["val_err_mean"],
                       "val_err_p99": rep["val_err_p99"], "val_err_max": rep["val_err_max"],
                       "val_err_trial_mean": rep["val_err_trial_mean"]}
    start = sim.particles()
    runs = {}
    for mode in ("plain", "closure"):
        sim.closure_enable(mode == "closure", judge_stride=64)
        sim.set_particles(start)
        sim.step()  # untimed: builds this mode's step graph
        sim.set_particles(start)
        sim.synchronize()
        sim.closure_stats(reset=True)
        runs[mode] = _timed_frames(sim, steps)
    st = sim.closure_stats()
    sim.closure_enable(False)
    total_ms, subs = runs["closure"]
    value = n * subs / (total_ms / 1000.0)
    plain_ms, plain_subs = runs["plain"]
    plain_same = n * plain_subs / (plain_ms / 1000.0)
    smooth = max(st["smooth"], 1)
    return {"value": value, "unit": UNIT, "ms_per_step": total_ms / steps,
            "vs_plain": value / plain_same, "plain_same_state": plain_same,
            "vs_plain_note": "closure and plain step timed over the same frames from the same "
                             "particle state (the main value is an earlier frame range)",
            "judge_stride": 64,
            "err_mean": st["err_mean"], "err_p50": st["err_p50"], "err_p99": st["err_p99"],
            "err_max": st["err_max"], "judged": st["judged"],
            "judge_replaced": st["judge_replaced"], "judge_bar": 1e-3,
            "net_frac": st["net"] / smooth, "hull_fallback_frac": st["hull_fallback"] / smooth,
            "error_metric": "relative error of the principal Kirchhoff stress vs the plain mapping "
                            "(judged sample, before the judge's replacement; percentiles are upper "
                            "edges of quarter-decade bins)",
            "evaluation": "deferred: the particle pass queues the network's particles, a tcgen05 "
                          "tile kernel evaluates them 128 at a time and finishes their update",
            "train": train, "nacc": nacc_closure()}


def nacc_closure() -> dict:
    """The NACC network: the benchmark scene's NACC soil never reaches the ellipse branch
    (the reference does not advance a NACC particle's F), so it is logged and trained on
    a scene of pre-deformed soil blocks (tests/scenes.py nacc_ellipse) and judged live on
    another seeded scene of the same kind."""
    from emerge_engine_b200 import Simulation
    from tests import scenes
    sim = scenes.nacc_ellipse(Simulation)
    sim.closure_log(2_000_000, 1)
    sim.step()
    sim.closure_log(0, 1)
    logged = int(sim.closure_stats()["logged"][1])
    rep = sim.closure_train(1, epochs=40, batch=4096, lr=2e-3, lr_decay=0.93, seed=3)
    params, norm = sim.closure_params(1)
    x, _ = sim.closure_log_samples(1, 2_000_000)
    xn = (x - norm[:6]) * norm[6:12]
    hull = np.concatenate([xn.min(0), xn.max(0)]).astype(np.float32)
    live = scenes.nacc_ellipse(Simulation, seed=12)
    live.set_closure_params(1, params, norm, hull)
    live.closure_enable(True, judge_stride=4)
    live.step()
    ls = live.closure_stats()
    sim.close()
    live.close()
    return {"scene": "nacc_ellipse (seed 11 logged and trained, seed 12 live)", "samples": logged,
            "seconds": rep["seconds"], "val_err_mean": rep["val_err_mean"],
            "val_err_p99": rep["val_err_p99"], "val_err_max": rep["val_err_max"],
            "val_err_trial_mean": rep["val_err_trial_mean"],
            "live": {k: ls[k] for k in ("net", "judged", "err_mean", "err_p50", "err_p99", "err_max",
                                         "judge_replaced", "hull_fallback")}}


def reduce_over_ranks(dist, device, total_ms: float, units: float, launches: int):
    """Replica aggregation: device time is the max over ranks (the job ends with the slowest
    replica); particle-substeps and kernel launches add up."""
    import torch
    t = torch.tensor([total_ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    u = torch.tensor([units, float(launches)], dtype=torch.float64, device=device)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u[0].item()), int(u[1].item())


def build_scene(sim_cls, workload: str, **kw):
    from tests import scenes
    spec = WORKLOADS[workload]
    return getattr(scenes, spec["builder"])(sim_cls, **spec["kwargs"], **kw)


def _oracle_scenes(workload: str):
    from oracle.oracle import OracleSimulation
    sims = build_scene(OracleSimulation, workload)
    return sims if isinstance(sims, list) else [sims]


def _oracle_run(sims, max_steps: int, budget_s: float):
    """Steps every scene once per round until max_steps rounds or the time budget;
    returns (rounds, particle-substeps, substeps, seconds)."""
    units = subs = rounds = 0
    t0 = time.perf_counter()
    while rounds < max_steps:
        for sim in sims:
            sim.step()
            k = sim.last_substeps()
            subs += k
            units += sim.particle_count() * k
        rounds += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    return rounds, units, subs, time.perf_counter() - t0


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def time_oracle(workload: str, warmup_steps: int, warmup_budget_s: float, runs: int,
                run_budget_s: float, max_steps_per_run: int = 1 << 30) -> dict:
    """The CPU oracle (the reference step restated in C++) on this host's cores: up to
    `warmup_steps` warm-up frames (stopping early once `warmup_budget_s` is spent), then
    `runs` timed runs of whole frames, each run ending after `max_steps_per_run` frames or
    `run_budget_s` seconds; the value is the median run's particle-substeps per second."""
    from oracle.oracle import set_threads
    threads = set_threads(0)
    sims = _oracle_scenes(workload)
    n = sum(s.particle_count() for s in sims)
    w_rounds, _, _, w_dt = _oracle_run(sims, warmup_steps, warmup_budget_s)
    rates, frames, subs_total, secs = [], 0, 0, 0.0
    for _ in range(runs):
        rounds, units, subs, dt = _oracle_run(sims, max_steps_per_run, run_budget_s)
        rates.append(units / dt)
        frames += rounds
        subs_total += subs
        secs += dt
    med = statistics.median(rates)
    return {"value": med, "unit": UNIT, "cores": threads, "cpu_model": cpu_model(),
            "kind": "port", "runs": runs, "run_values": rates,
            "spread": (max(rates) - min(rates)) / med if med > 0 else None,
            "warmup_steps": w_rounds, "frames": frames, "substeps": subs_total,
            "particles": n, "scenes": len(sims), "seconds": secs,
            "sample": f"{workload}: median of {runs} timed runs ({frames} full steps, {subs_total} "
                      f"substeps of {n} particles in {len(sims)} scene(s), {secs:.1f} s) after "
                      f"{w_rounds} warm-up step(s) ({w_dt:.1f} s); P2G, density and constitutive "
                      "update sequential as in the reference, G2P gather on all threads"}


def cpu_baseline(workload: str, budget_s: float = 15.0) -> dict:
    """Bounded sample of the CPU oracle for the cpu_baseline key: warm-up frames (at most 10,
    within a third of the budget), then the median of 3 timed runs."""
    return time_oracle(workload, 10, budget_s / 3.0, 3, budget_s / 3.0)


def run_reference(args):
    """--impl reference: the oracle on the host cores, same workload and metric."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # Bounded sample: the warm-up and each timed run stop early once their time budget is
    # spent, so the run ends within a few minutes whatever the workload.
    runs = 3
    cb = time_oracle(args.workload, max(args.warmup, 1), args.ref_warmup_budget, runs,
                     args.ref_budget / runs, max(1, -(-args.steps // runs)))
    value = cb["value"]
    ms_per_step = cb["seconds"] * 1000.0 / max(cb["frames"], 1)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded scene generator, tests/scenes.py)",
        "config": workload_config(args.workload, cb["particles"], args.gpus),
        "substeps_per_step": cb["substeps"] / max(cb["frames"], 1),
        "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "cpu_model", "kind", "runs",
                                             "run_values", "spread", "warmup_steps", "sample")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# The parity bar the measured path meets (the fast path; tests/test_gpu_parity_scale.py holds
# it against the oracle).  The reference-order mode (DeterministicSimulation) is bit identical
# to the oracle on the same scenes.
PARITY = {
    "path": "fast (P2G summed by L2 reductions in a run-to-run order)",
    "bars": {"dam_break_1m, one frame": "x <= 1e-5, v p50 <= 1e-5, p99 <= 3e-5, max <= 2e-3",
             "mixed_granular_4m, one substep": "v <= 1e-5 per particle",
             "100 frames (dam break 262k, granular 160k)": "region statistics within max(1e-3, 2x the "
                                                            "reference's own reordering distance)",
             "always": "mass exact, momentum within 1e-6 of the total |momentum|"},
    "reference_order_mode": "bit identical to the oracle (1M dam break frame, 4M granular substep)",
    "tests": "tests/test_gpu_parity_scale.py, tests/test_gpu_parity.py",
}


def workload_config(workload: str, particles: int, world: int) -> dict:
    """The `config` object of both arms' lines (identical keys and values for one workload)."""
    spec = WORKLOADS[workload]
    return {"workload": workload, "description": spec["desc"], "particles_per_gpu": particles,
            "grid": spec["grid_res"],
            "l2": "GPU arm: flushed (512 MiB device write) before every timed step",
            "parallelism": f"replicas x{world}"}


def run_batched(args, spec, rank: int, world: int, dist, local_rank: int) -> dict:
    """Batched scenes: all scenes of the workload advanced together (one launch per kernel
    per substep); value = sum over scenes of particles x substeps per second.  Weak scaling:
    one fixed list of 256 x N seeded scenes is placed on the N ranks by
    sharding.shard_scenes (longest-processing-time first on particle counts), and each rank
    advances its share as one batch, with no collective on the data path."""
    from emerge_engine_b200 import Batch, Simulation
    from emerge_engine_b200.build import build
    from emerge_engine_b200.sharding import shard_loads, shard_scenes
    from tests import scenes as scene_lib
    build()
    kw = dict(WORKLOADS[args.workload]["kwargs"])
    kw["n_scenes"] = kw.get("n_scenes", 256) * world
    draws = scene_lib.batched_scene_draws(
        **{k: v for k, v in kw.items() if k in ("n_scenes", "seed", "pair_sizes")})
    costs = scene_lib.batched_scene_particles(draws)
    shards = shard_scenes(costs, world)
    placement = {"scenes_total": len(draws), "particles_total": int(sum(costs)),
                 "rank_particles": [int(x) for x in shard_loads(costs, shards)],
                 "method": "LPT on particle counts (emerge_engine_b200.sharding)"}
    sims = scene_lib.batched_scenes(Simulation, only=shards[rank], device=local_rank, **kw)
    counts = np.array([s.particle_count() for s in sims], dtype=np.int64)
    batch = Batch(sims)
    for s in sims:
        s.close()
    del sims
    cache = os.environ.get("EMERGE_CUDA_TUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "emerge_engine_b200", "batch_tune.txt")
    os.makedirs(os.path.dirname(cache), exist_ok=True)
    tune = batch.autotune(steps_per_trial=1, cache_path=cache) if not args.no_extras else None
    batch.step(args.warmup)
    clocks = ClockSampler(local_rank)
    clocks.start()
    t_load = time.perf_counter()
    _, tot0 = batch.substeps()
    t_begin = time.perf_counter()
    total_ms = batch.time_steps(args.steps, flush_l2=True)
    clock_info = clocks.stop(t_begin, time.perf_counter(), t_load)
    _, tot1 = batch.substeps()
    units = float(np.sum(counts * (tot1 - tot0).astype(np.int64)))
    if dist is not None:
        total_ms, units, _ = reduce_over_ranks(dist, f"cuda:{local_rank}", total_ms, units, 0)
    value = units / (total_ms / 1000.0)
    peak, peak_kind = load_peaks()
    ppc = 4.0
    b_alg = 156.0 + 24.0 / ppc + 8.0 / ppc  # per particle-substep (fluid scenes add the mass field)
    achieved = b_alg * value / 1e9
    out = {"value": value, "ms_per_step": total_ms / args.steps, "clocks": clock_info,
           "scenes": int(len(counts)), "particles": int(counts.sum()),
           "substeps_per_step_mean": float(np.mean(tot1 - tot0)) / args.steps,
           "substeps_per_step_max": float(np.max(tot1 - tot0)) / args.steps,
           "roofline": {"kernel": "whole substep, all scenes (B_alg = 156 + 32/ppc B per "
                                  "particle-substep)", "bound": "hbm", "achieved": achieved,
                        "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                        "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)"},
           "autotune": tune, "placement": placement}
    batch.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-extras", action="store_true",
                    help="skip e2e, roofline instrumentation and CPU baseline (profiling runs)")
    ap.add_argument("--cpu-budget", type=float, default=30.0,
                    help="cpu_baseline: seconds for the warm-up and for each of the 3 timed runs x 3")
    ap.add_argument("--no-closure", action="store_true",
                    help="skip the learned-closure A/B on scenes with plastic materials")
    ap.add_argument("--ref-budget", type=float, default=60.0,
                    help="--impl reference: seconds of timed CPU steps at most")
    ap.add_argument("--ref-warmup-budget", type=float, default=20.0)
    ap.add_argument("--p2g-aggregate", type=int, default=None, choices=[0, 1, 2],
                    help="EMERGE_OPT_P2G_AGGREGATE for the run (default: the library's)")
    ap.add_argument("--skip", default="",
                    help="comma list of parts to leave out: e2e, closure, cpu (roofline and phases stay)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    if args.impl == "reference":
        run_reference(args)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist_mod
        torch.cuda.set_device(local_rank)
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = dist_mod

    spec = WORKLOADS[args.workload]
    if spec["material"] == "batched":
        r = run_batched(args, spec, rank, world, dist, local_rank)
        if rank == 0:
            line = {
                "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded scene generator, tests/scenes.py)",
                "config": workload_config(args.workload, r["particles"], world),
                "scenes": r["scenes"], "substeps_per_step_mean": r["substeps_per_step_mean"],
                "substeps_per_step_max": r["substeps_per_step_max"],
                "clocks": r["clocks"], "roofline": r["roofline"], "autotune": r["autotune"],
                "placement": r["placement"],
            }
            if world == 1 and not args.no_extras:
                line["cpu_baseline"] = cpu_baseline(args.workload, args.cpu_budget)
            print(json.dumps(line), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return

    from emerge_engine_b200 import Simulation
    from emerge_engine_b200.abi import OPT_USE_GRAPH
    from emerge_engine_b200.build import build
    build()

    sim = build_scene(Simulation, args.workload, device=local_rank)
    if args.p2g_aggregate is not None:
        from emerge_engine_b200.abi import OPT_P2G_AGGREGATE
        sim.set_option(OPT_P2G_AGGREGATE, args.p2g_aggregate)
    skip = set(filter(None, args.skip.split(",")))
    n = sim.particle_count()
    clocks = ClockSampler(local_rank)
    clocks.start()
    t_load = time.perf_counter()
    for _ in range(args.warmup):
        sim.step()
    sim.synchronize()

    def barrier():
        if dist is not None:
            import torch
            dist.barrier(device_ids=[local_rank])
            torch.cuda.synchronize()
        sim.synchronize()

    st0 = sim.stats()
    barrier()
    t_begin = time.perf_counter()
    total_ms = 0.0
    active_units = 0.0  # sleep partition: awake particles x substeps
    for _ in range(args.steps):
        sim.flush_l2()
        a0 = sim.active_count() if spec.get("active_units") else 0
        sim.event_record(0)
        sim.step()
        sim.event_record(1)
        total_ms += sim.event_elapsed_ms(0, 1)
        if spec.get("active_units"):
            active_units += 0.5 * (a0 + sim.active_count()) * sim.last_substeps()
    sim.synchronize()
    clock_info = clocks.stop(t_begin, time.perf_counter(), t_load)
    st1 = sim.stats()
    barrier()
    substeps = st1["substeps"] - st0["substeps"]
    launches = st1["kernel_launches"] - st0["kernel_launches"]
    units = active_units if spec.get("active_units") else float(n * substeps)
    n_eff = units / max(substeps, 1)  # particles a pass works on (awake ones with a partition)
    if dist is not None:
        total_ms, units, launches = reduce_over_ranks(dist, f"cuda:{local_rank}", total_ms, units,
                                                      launches)
    value = units / (total_ms / 1000.0)
    ms_per_step = total_ms / args.steps

    extras = {}
    if not args.no_extras:
        # Roofline of the dominant kernel: the fused particle pass, timed per launch with
        # CUDA events on the simulation's stream (host-driven substep loop, same kernels).
        sim.set_option(OPT_USE_GRAPH, 0)
        part_us, subs_i = 0.0, 0
        phase_keys = ("cfl_us", "project_us", "density_us", "p2g_us", "grid_update_us", "g2p_us")
        phases = dict.fromkeys(phase_keys, 0.0)
        for _ in range(3):
            sim.flush_l2()
            sim.step_n(1, timing=True)
            part_us += sim.last_timing["g2p_us"]
            subs_i += sim.last_substeps()
            for k in phase_keys:
                phases[k] += sim.last_timing[k]
        if os.environ.get("EMERGE_CUDA_USE_GRAPH", "1") != "0":  # else keep the host loop
            sim.set_option(OPT_USE_GRAPH, 1)
        peak, peak_kind = load_peaks()
        per_launch_s = part_us * 1e-6 / max(subs_i, 1)
        alg_bytes = K_PARTICLE_BYTES[spec["material"]] * n_eff
        achieved = alg_bytes / per_launch_s / 1e9
        traffic = profile_traffic(args.workload)
        extras["roofline"] = {
            "kernel": "k_particle (fused G2P + update + CFL + projection + P2G)",
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic,
            "algorithmic_bytes_per_launch": alg_bytes, "launch_us": per_launch_s * 1e6,
            "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured"
            else "fallback 6.65 TB/s"}
        if "nbody" in spec["material"]:
            extras["roofline"]["note"] = (
                "with NBodyGravityField the pass runs as two halves around the Barnes-Hut tree "
                "build and walk (k_nb_walk), and the timed g2p phase holds all of them; the walk "
                "(three quarters of a substep) is bound by instruction issue on an L1/L2-resident "
                "tree, not by HBM: the fraction is of k_particle's streaming bytes only")
        # where a substep's time goes (host-driven loop, CUDA events between the phases)
        extras["phases_us_per_substep"] = {k[:-3]: v / max(subs_i, 1) for k, v in phases.items()}
        extras["phases_note"] = ("p2g and project read 0: the fused particle pass (k_particle) does "
                                 "the projection and the P2G scatter of substep k+1 together with "
                                 "the G2P and update of substep k, and is timed as g2p; density is "
                                 "k_density (fluid scenes only); cfl is the controller")
        if "Fluid" in spec["material"]:
            # (the phase reads a few microseconds of event overhead in scenes without the pass)
            # the density pass: reads x, material, C, mass (88 B of the fluid state are not
            # needed), writes rho_dp, gathers 9 masses and scatters 9 stress pairs per particle
            # (12 B per cell at 4 ppc -> 3 B)
            d_us = phases["density_us"] / max(subs_i, 1)
            d_bytes = K_DENSITY_BYTES * n_eff
            d_ach = d_bytes / (d_us * 1e-6) / 1e9
            extras["roofline_density"] = {
                "kernel": "k_density (density gather + fluid stress scatter)", "bound": "hbm",
                "achieved": d_ach, "peak": peak, "unit": "GB/s", "frac": d_ach / peak,
                "traffic": None, "algorithmic_bytes_per_launch": d_bytes, "launch_us": d_us}

    if not args.no_extras and "e2e" not in skip:
        # End to end through the C ABI with host buffers: upload the particle state from
        # pinned memory, step, read it back into a second pinned buffer, every step.  The
        # readback is asynchronous (its own stream), so step k's device-to-host copy overlaps
        # step k+1's upload; the timed region ends after the last readback has landed.
        from emerge_engine_b200.simulation import PinnedBuffer
        host = PinnedBuffer(n * 128)
        host_out = PinnedBuffer(n * 128)
        sim.read_particles_raw(host.ptr, n)
        # one untimed round first: the upload and readback paths set up their staging buffers
        # and streams on first use
        sim.write_particles_raw(host.ptr, n)
        sim.step()
        sim.read_particles_raw_async(host_out.ptr, n)
        sim.synchronize()
        e2e_steps = max(3, min(args.steps, 10))
        sub0 = sim.stats()["substeps"]
        sim.synchronize()
        t0 = time.perf_counter()
        e2e_active = 0.0
        for _ in range(e2e_steps):
            sim.write_particles_raw(host.ptr, n)
            a0 = sim.active_count() if spec.get("active_units") else 0
            sim.step()
            if spec.get("active_units"):
                e2e_active += 0.5 * (a0 + sim.active_count()) * sim.last_substeps()
            sim.read_particles_raw_async(host_out.ptr, n)
        sim.synchronize()
        e2e_s = time.perf_counter() - t0
        e2e_subs = sim.stats()["substeps"] - sub0
        e2e_units = e2e_active if spec.get("active_units") else float(n * e2e_subs)
        if dist is not None:
            e2e_ms, e2e_units, _ = reduce_over_ranks(dist, f"cuda:{local_rank}", e2e_s * 1e3,
                                                     e2e_units, 0)
            e2e_s = e2e_ms / 1e3
        host.free()
        host_out.free()
        extras["e2e"] = {"value": e2e_units / e2e_s, "unit": UNIT,
                         "h2d_bytes_per_step": n * 128, "d2h_bytes_per_step": n * 128,
                         "steps": e2e_steps, "timing": "host wall clock around the C-ABI calls",
                         "readback": "emerge_cuda_read_particles_async (copy stream; overlaps "
                                     "the next step's upload)"}
    if not args.no_extras:
        # the closure's A/B (training included) on one GPU only: a scaling run's ranks would each
        # repeat it, holding every GPU for minutes outside the timed region
        if spec["material"] == "DP+Snow+NACC" and not args.no_closure and "closure" not in skip and world == 1:
            extras["learned_closure"] = closure_ab(sim, n, args.steps, value)
        if world == 1 and rank == 0 and "cpu" not in skip:
            extras["cpu_baseline"] = cpu_baseline(args.workload, args.cpu_budget)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene generator, tests/scenes.py)",
            "config": workload_config(args.workload, n, world),
            "substeps_per_step": substeps / args.steps,
            "gpu_launches": launches,
            "clocks": clock_info,
            "parity": PARITY,
        }
        line.update(extras)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
