"""Benchmark of the PM gravity step: particle-steps/s on one B200 (or N replicas).

Default workload: the cosmic-web field, 16,777,216 particles (256^3 lattice,
Zel'dovich displacements, seed 2) on a 512^3 periodic grid, dt = 1e-3, Newton
units (G = 1, total mass 1), softening 1 cell, sort every step. Synthetic,
seeded; inputs (268 MB of particles, 512^3 grids) exceed L2, so no L2 flush.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs one independent replica per rank (the single-scene step does not
shard); torch.distributed is used only for the barrier and the max-over-ranks
time. `--impl reference` times the CPU restatement of the reference's step
(oracle/, FP32, all host threads) on rank 0 -- the reference itself has no CPU
implementation of this path.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0

WORKLOADS = {
    # name: (particles description, grid, dt)
    "cosmic_web_512": {"grid": 512, "dt": 1e-3, "lattice": 256},
    "two_galaxy_256": {"grid": 256, "dt": 5e-4},
    "disk_64": {"grid": 64, "dt": 1e-3},
}


def model_bytes(n: int, G: int) -> float:
    """Algorithmic bytes of one step: 184 B per particle + 40 B per cell."""
    return 184.0 * n + 40.0 * G ** 3


# kernels of one timed step, in the order of sd_timings.kernel_ms
KERNELS = ["sort", "row_table", "pass_a_deposit", "pass_b", "pass_c", "pass_d", "pass_e", "gather"]


def kernel_bytes(n: int, G: int) -> dict:
    """Algorithmic bytes per launch of each kernel of the tiled-order step."""
    spec = 8.0 * G * G * (G // 2 + 4)  # bricked half spectrum, complex64
    cells = float(G) ** 3
    return {
        # steady state merges: read the new keys, write the permutation, plus the change
        # bits (read twice) and their per-word prefixes (written once, read once)
        "sort": 8 * n + 4 * (n / 32) * 4,
        "row_table": 3 * 4 * (G * G + 1),         # old table and the changed set's in, new table out
        "pass_a_deposit": 20 * n + spec,          # perm + pos once; spectrum written
        "pass_b": 2 * spec,
        "pass_c": 2 * spec,
        "pass_d": 2 * spec,
        "pass_e": spec + 4 * cells,
        "gather": 72 * n + 4 * cells,             # perm, pos+vel in/out, keys, potential
    }


def measured_traffic(kernel: str, workload: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 3 and parts[0] == workload and parts[1] == kernel:
                    return float(parts[2])
    except OSError:
        pass
    return None


def hbm_peak():
    try:
        with open(MEASURED_PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def make_workload(name: str):
    from stardust_b200 import scenes

    w = WORKLOADS[name]
    if name == "cosmic_web_512":
        pos, vel = scenes.zeldovich(w["lattice"], 2)
    elif name == "two_galaxy_256":
        pos, vel = scenes.two_galaxies(4_194_304, 1)
    else:
        pos, vel = scenes.disk_galaxy(262_144, 0)
    return pos, vel, w["grid"], w["dt"]


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def run_ours(args, rank, world):
    import torch

    from stardust_b200 import _lib as L
    from stardust_b200.sim import Sim, SimConfig

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    pos, vel, G, dt = make_workload(args.workload)
    n = len(pos)
    cfg = SimConfig(particle_count=n, grid_size=G, gravity=1.0, units=L.SD_UNITS_NEWTON, softening_cells=1.0,
                    sort_interval=1, order=args.order, keep_density=0,
                    diagnostics=0 if args.no_diagnostics else 1)
    stream = torch.cuda.Stream(device=dev)
    sim = Sim(dev)
    sim.init(cfg)
    L.check(L.lib().sd_set_stream(sim.handle, stream.cuda_stream), "sd_set_stream")
    sim.set_particles(pos, vel)
    dist = world > 1

    def barrier():
        torch.cuda.synchronize()
        if dist:
            torch.distributed.barrier()

    # --- device-resident timed region: K steps through the captured-graph path ---
    sim.steps(dt, args.warmup)
    torch.cuda.synchronize()
    sim.steps(dt, 2)  # settles the merge-or-full-sort choice (and its graph) before timing
    barrier()
    clocks = ClockSampler(dev)
    clocks.start()
    launches0 = Sim.kernel_launches()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        sim.steps(dt, args.steps)
        e1.record(stream)
    barrier()
    clock_info = clocks.stop()
    launches = Sim.kernel_launches() - launches0
    ms = e0.elapsed_time(e1) / args.steps
    diag = None
    if not args.no_diagnostics:  # the FP64 records of the timed steps
        h = sim.diagnostics_history(args.steps)
        e = h[:, 1] + h[:, 2]
        diag = {"records": int(len(h)), "kinetic_first": float(h[0, 1]), "potential_first": float(h[0, 2]),
                "energy_drift_rel_to_potential": float((e[-1] - e[0]) / abs(h[0, 2])),
                "max_abs_momentum": float(np.abs(h[:, 3:6]).max()),
                "note": "FP64 energy and momentum every step, accumulated inside the gather"}
    t = torch.tensor([ms], device="cuda")
    if dist:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms = float(t.item())

    # --- per-kernel times (eager steps with events between kernels) for the roofline ---
    kms = []
    phases = {"sort_ms": [], "deposit_ms": [], "poisson_ms": [], "gather_ms": [], "total_ms": []}
    for _ in range(3):
        sim.step(dt)
        tm = sim.timings()
        kms.append(tm["kernel_ms"])
        for k in phases:
            phases[k].append(tm[k])
    phase_ms = {k: float(np.median(v)) for k, v in phases.items()}
    kernel_ms = dict(zip(KERNELS, np.median(np.array(kms), axis=0).tolist()))

    # --- end to end through the C ABI with pinned host buffers, every step ---
    hp = torch.from_numpy(pos).pin_memory()
    hv = torch.from_numpy(vel).pin_memory()
    op = torch.empty_like(hp).pin_memory()
    ov = torch.empty_like(hv).pin_memory()
    lib = L.lib()
    e2e_steps = max(2, min(args.steps, 10))

    def e2e_step():
        # the pipelined offload call: host pos/vel in, one step, host pos/vel out
        # (pinned buffers); consecutive calls overlap one step's download, the next
        # step and the upload after it
        L.check(lib.sd_step_host_async(sim.handle, hp.data_ptr(), hv.data_ptr(), n, float(dt), op.data_ptr(),
                                       ov.data_ptr()), "step_host_async")

    e2e_step()
    L.check(lib.sd_step_host_wait(sim.handle), "step_host_wait")
    barrier()
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(e2e_steps):
            e2e_step()
        L.check(lib.sd_step_host_wait(sim.handle), "step_host_wait")  # every step's outputs are on the host
        e1.record(stream)
    barrier()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    e2e_wall_ms = (time.perf_counter() - t0) * 1e3 / e2e_steps
    t = torch.tensor([e2e_ms], device="cuda")
    if dist:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    e2e_ms = float(t.item())
    # the force error of the step's field: the accelerations of the current
    # positions against FP64 particle-mesh on the same grid, at 65,536 sampled
    # particles (the error against FP64 Ewald forces is reported by the learned comparison)
    from stardust_b200.ewald import force_error, pm_accel_f64

    p_now, _ = sim.get_particles()
    a_now = sim.accel()
    live = np.nonzero(p_now[:, 0] >= 0.0)[0]
    sample = np.random.default_rng(0).choice(live, min(65536, len(live)), replace=False)
    pot_scale = 4.0 * np.pi * float(G) ** 3 / n  # Newton units, G = 1, each particle 1/N
    ferr = force_error(a_now[sample, :3], pm_accel_f64(p_now, sample, G, pot_scale, 1.0))
    del p_now, a_now
    sim.close()

    peak, peak_kind = hbm_peak()
    B = model_bytes(n, G)
    achieved_step = B / (ms * 1e-3) / 1e9
    kbytes = kernel_bytes(n, G)
    dom = max(KERNELS, key=lambda k: kernel_ms[k])
    dom_achieved = kbytes[dom] / (kernel_ms[dom] * 1e-3) / 1e9
    traffic = measured_traffic(dom, args.workload)
    value = world * n / (ms * 1e-3)
    out = {
        "metric": "particle-steps/s at 16M/512^3; learned vs plain PM at equal force error vs FP64",
        "value": value,
        "unit": "particle-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded Zel'dovich field, no dataset)",
        "config": {"workload": args.workload, "particles_per_gpu": n, "grid": G, "dt": dt,
                   "order": ["rowmajor", "morton", "tiled"][args.order], "sort_every_step": True,
                   "units": "newton G=1 M=1", "softening_cells": 1.0, "parallelism": f"replicas x{world}",
                   "fp64_diagnostics_every_step": not args.no_diagnostics,
                   "l2": "inputs exceed L2 (no flush)", "timed_path": "sd_steps (CUDA graph, 2 steps/replay)"},
        "roofline": {"bound": "hbm", "achieved": dom_achieved, "peak": peak, "unit": "GB/s",
                     "frac": dom_achieved / peak, "traffic": traffic, "kernel": dom,
                     "algorithmic_bytes": kbytes[dom], "kernel_ms": kernel_ms[dom],
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                     else "fallback 6650 GB/s"},
        "step_roofline": {"model_bytes": B, "model": "184 N + 40 G^3", "achieved_gbs": achieved_step,
                          "frac": achieved_step / peak},
        "kernel_ms": kernel_ms,
        "phase_ms": phase_ms,
        "e2e": {"value": world * n / (e2e_ms * 1e-3), "unit": "particle-steps/s",
                "h2d_bytes_per_step": 2 * 16 * n, "d2h_bytes_per_step": 2 * 16 * n,
                "path": "sd_step_host_async x steps + sd_step_host_wait: pinned host pos/vel in, one step, "
                        "host pos/vel out, each step",
                "wall_ms_per_step": e2e_wall_ms},
        "gpu_launches": int(launches),
        "force_error": {"vs": "FP64 particle-mesh on the same grid", "particles": int(len(sample)),
                        "rms_rel": ferr["rms_rel"], "max_rel": ferr["max_rel"],
                        "metric": "RMS|a - a_ref| / RMS|a_ref|"},
        "clocks": clock_info,
        "diagnostics": diag,
    }
    return out


def time_workload(name: str, order: int = 2, steps: int = 20, warmup: int = 4, full_sort: int = 0) -> dict:
    """One workload on this rank's GPU: graph-replayed ms/step (CUDA events on the
    handle's stream), per-kernel ms of eager steps, and the step's byte model
    (184 N + 40 G^3) as a fraction of the HBM peak."""
    import torch

    from stardust_b200 import _lib as L
    from stardust_b200.sim import Sim, SimConfig

    pos, vel, G, dt = make_workload(name)
    n = len(pos)
    cfg = SimConfig(particle_count=n, grid_size=G, gravity=1.0, units=L.SD_UNITS_NEWTON, softening_cells=1.0,
                    sort_interval=1, order=order, keep_density=0, full_sort=full_sort)
    stream = torch.cuda.Stream()
    with Sim(torch.cuda.current_device()) as sim:
        sim.init(cfg)
        sim.set_stream(stream)
        sim.set_particles(pos, vel)
        sim.steps(dt, warmup)
        torch.cuda.synchronize()
        # a second call settles the merge-or-full-sort choice the warm-up measured
        # (and captures its graph) before the timed region
        sim.steps(dt, 2)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.steps(dt, steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        kms = []
        for _ in range(3):
            sim.step(dt)
            kms.append(sim.timings()["kernel_ms"])
        frac, merging = sim.changed_fraction(), sim.merge_sorting()
    peak, _ = hbm_peak()
    B = model_bytes(n, G)
    return {"particles": n, "grid": G, "dt": dt, "order": ["rowmajor", "morton", "tiled"][order],
            "changed_fraction": frac, "sort": "merge" if merging else "full radix",
            "ms_per_step": ms, "value": n / (ms * 1e-3), "unit": "particle-steps/s",
            "kernel_ms": dict(zip(KERNELS, np.median(np.array(kms), axis=0).tolist())),
            "step_roofline": {"model_bytes": B, "achieved_gbs": B / (ms * 1e-3) / 1e9,
                              "frac": B / (ms * 1e-3) / 1e9 / peak}}


def run_ensemble(rank, world, steps: int = 100, warmup: int = 3, dt: float = 1e-3) -> dict:
    """The batched ensemble: 64 seeded scenes (disk or Zel'dovich recipe, N
    log-uniform in [16K, 1M], grids 32/64/128 matched to N), split across ranks
    by LPT on step bytes; each rank advances its scenes with one graph launch per
    step after autotuning. Value = all scenes' particle-steps / max-over-ranks time."""
    import torch

    from stardust_b200.ensemble import Ensemble, member_config, partition
    from stardust_b200.scenes import ensemble_members, make_member

    members = ensemble_members(64, 4)
    mine = partition(members, world)[rank]
    ens = Ensemble(torch.cuda.current_device())
    n_local = 0
    for i in mine:
        p, v = make_member(members[i])
        ens.add(member_config(members[i]), p, v)
        n_local += len(p)
    t0 = time.perf_counter()
    tuning = ens.autotune(dt)
    tune_s = time.perf_counter() - t0
    ens.steps(dt, warmup)
    ens.synchronize()
    if world > 1:
        torch.distributed.barrier()
    stream = torch.cuda.ExternalStream(ens.stream_handle)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ens.steps(dt, steps)
    e1.record(stream)
    ens.synchronize()
    ms = e0.elapsed_time(e1) / steps
    t = torch.tensor([ms, float(n_local)], device="cuda", dtype=torch.float64)
    if world > 1:
        tm = t[:1].clone()
        torch.distributed.all_reduce(tm, op=torch.distributed.ReduceOp.MAX)
        nt = t[1:].clone()
        torch.distributed.all_reduce(nt, op=torch.distributed.ReduceOp.SUM)
        ms, n_total = float(tm.item()), float(nt.item())
    else:
        n_total = float(n_local)
    kernels = ens.graph_kernels()
    ens.close()
    tiled = sum(1 for tt in tuning if tt["order"] == "tiled")
    # the byte model summed over this rank's scenes, against the HBM peak; and the
    # spread of the scenes' solo step times (the autotuner's measurements), whose sum
    # over the ensemble's step time is how much the branches overlap
    B = float(sum(model_bytes(members[i]["n"], members[i]["grid"]) for i in mine))
    peak, peak_kind = hbm_peak()
    solo = np.array([tt["step_ms"] for tt in tuning], np.float64)
    roof = {"model_bytes": B, "model": "sum of 184 N + 40 G^3", "achieved_gbs": B / (ms * 1e-3) / 1e9,
            "frac": B / (ms * 1e-3) / 1e9 / peak, "peak": peak, "peak_source": peak_kind}
    branches = {"solo_ms_quantiles": {q: float(np.quantile(solo, float(q))) for q in ("0", "0.5", "0.9", "1")},
                "solo_ms_sum": float(solo.sum()), "overlap": float(solo.sum() / ms),
                "largest_scene_share": float(solo.max() / ms)}
    return {"value": n_total / (ms * 1e-3), "unit": "particle-steps/s", "ms_per_step": ms, "steps": steps,
            "step_roofline": roof, "branches": branches,
            "scenes": len(members), "particles": int(n_total),
            "grids": {str(g): sum(1 for m in members if m["grid"] == g) for g in (32, 64, 128)},
            "graph_launches_per_step": 1, "kernels_per_graph_rank0": kernels,
            "autotune": {"seconds": tune_s, "tiled_deposit_scenes": tiled, "atomic_deposit_scenes": len(tuning) - tiled,
                         "deposit_share_particles": sorted({tt["deposit_split"] for tt in tuning if tt["order"] == "tiled"}),
                         "gather_caps": sorted({tt["gather_blocks"] for tt in tuning})},
            "partition": f"LPT over {world} rank(s)"}


def run_reference(args, rank, world):
    from oracle import oracle as O

    pos, vel, G, dt = make_workload(args.workload)
    n = len(pos)
    threads = O.num_threads()
    grav = float(4 * np.pi * G ** 3)
    # warm-up on a small sample, then time whole steps at the full size
    O.step(pos[:4096], vel[:4096], 16, grav, 1.0, dt, dt)
    # each timed step is one full step of the workload (about 1 s on 16 cores);
    # at most 20 of them keep the arm within a few minutes
    steps = max(1, min(args.steps, 20))
    t0 = time.perf_counter()
    p, v = pos, vel
    for _ in range(steps):
        p, v, _, _ = O.step(p, v, G, grav, 1.0, dt, dt)
    sec = (time.perf_counter() - t0) / steps
    value = n / sec
    return {
        "metric": "particle-steps/s at 16M/512^3; learned vs plain PM at equal force error vs FP64",
        "value": value,
        "unit": "particle-steps/s",
        "n_gpus": world,
        "steps": steps,
        "warmup": args.warmup,
        "ms_per_step": sec * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded Zel'dovich field, no dataset)",
        "config": {"workload": args.workload, "particles_per_gpu": n, "grid": G, "dt": dt,
                   "parallelism": "host cores"},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": threads, "kind": "port",
                         "sample": f"{steps} full step(s) of {n} particles on a {G}^3 grid"},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_gpu": reference_gpu_sample(pos, vel, G, dt),
    }


def reference_gpu_sample(pos, vel, G: int, dt: float, steps: int = 10, warmup: int = 3) -> dict:
    """The reference's own GPU step (its Sim class, cuFFT + CUB, built from its
    sources for sm_100a into oracle/_ref by oracle/ref/Makefile) on the same
    workload: a second baseline beside the CPU one. Its stock step() sizes dt by
    the CFL rule (timeScale = dt / 0.0016) and reads vmax back every step."""
    import ctypes
    import tempfile

    so = os.path.join(ROOT, "oracle", "_ref", "libsimref.so")
    if not os.path.exists(so):
        return {"unavailable": "oracle/_ref/libsimref.so was not built (the reference sources were absent)"}
    import torch

    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}
    lib = ctypes.CDLL(so)
    lib.ref_create.restype = ctypes.c_void_p
    lib.ref_destroy.argtypes = [ctypes.c_void_p]
    lib.ref_load.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                             ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_char_p]
    lib.ref_steps.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.ref_timings.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    n = len(pos)
    h = lib.ref_create()
    try:
        with tempfile.TemporaryDirectory() as d:
            rc = lib.ref_load(h, pos.ctypes.data, vel.ctypes.data, n, G, float(4 * np.pi * G ** 3), 1.0,
                              float(dt / 0.0016), 1, os.path.join(d, "state.bin").encode())
        if rc != 0:
            return {"unavailable": f"reference load failed ({rc})"}
        if lib.ref_steps(h, warmup) != 0:
            return {"unavailable": "reference step failed"}
        t0 = time.perf_counter()
        if lib.ref_steps(h, steps) != 0:
            return {"unavailable": "reference step failed"}
        sec = (time.perf_counter() - t0) / steps
        tm = np.zeros(6, np.float32)
        lib.ref_timings(h, tm.ctypes.data)
    finally:
        lib.ref_destroy(h)
    return {"value": n / sec, "unit": "particle-steps/s", "ms_per_step": sec * 1e3, "steps": steps,
            "dt_used": float(tm[4]), "kind": "reference Sim (cuFFT + CUB) built for sm_100a, wall clock per step",
            "phase_ms": {"scatter": float(tm[0]), "poisson": float(tm[1]), "gather": float(tm[2]),
                         "total": float(tm[3])}}


def cpu_baseline_sample(workload: str, steps: int = 8):
    """Full steps of the CPU restatement (oracle/), all host threads: a bounded
    sample of about 10 s on a 16-core host."""
    from oracle import oracle as O

    pos, vel, G, dt = make_workload(workload)
    grav = float(4 * np.pi * G ** 3)
    O.step(pos[:4096], vel[:4096], 16, grav, 1.0, dt, dt)
    t0 = time.perf_counter()
    p, v = pos, vel
    for _ in range(steps):
        p, v, _, _ = O.step(p, v, G, grav, 1.0, dt, dt)
    sec = (time.perf_counter() - t0) / steps
    return {"value": len(pos) / sec, "unit": "particle-steps/s", "cores": O.num_threads(), "kind": "port",
            "sample": f"{steps} full steps of {len(pos)} particles on a {G}^3 grid ({sec:.2f} s each)"}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="cosmic_web_512")
    ap.add_argument("--order", type=int, default=2, help="0 row-major (reference), 1 Morton, 2 tiled (fused deposit)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 64-scene batched ensemble")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other workloads (disk_64, two_galaxy_256) and the row-major / Morton orders")
    ap.add_argument("--no-diagnostics", action="store_true", help="time the step without the per-step FP64 records")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the learned-correction comparison (2M particles, 128^3 + MLP vs 128..512^3)")
    args = ap.parse_args(argv)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(run_reference(args, rank, world)))
        return 0
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    out = run_ours(args, rank, world)
    if world == 1 and not args.no_configs:
        # the other single-scene configurations (the headline's workload is cosmic_web_512)
        out["configs"] = {w: time_workload(w) for w in ("disk_64", "two_galaxy_256") if w != args.workload}
        # the reference's own particle order (row-major cell keys, the atomic deposit) and
        # the 30-bit Morton order on the headline workload
        out["orders"] = {o: time_workload(args.workload, order=k, steps=10) for k, o in ((0, "rowmajor"), (1, "morton"))}
    if not args.no_ensemble:
        out["ensemble"] = run_ensemble(rank, world)
    if world == 1 and not args.no_learned:
        from stardust_b200.learned import compare

        out["learned"] = compare()
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_sample(args.workload)
    if world > 1:
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
