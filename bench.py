#!/usr/bin/env python
"""Throughput of the hoomd-mc hard-sphere sweep on B200: trial moves per second.

Workload (one step = one ParallelSweep::apply, i.e. at least N trial moves):
3-D hard spheres (sigma = 1), N = 2^20, periodic cubic box at packing fraction 0.50,
FCC start with seeded jitter 0.01 sigma, translation moves with the maximum distance
tuned by Tune::tune_with_options (target acceptance 0.30, 8000 samples x 32 rounds, run on
the device by hmc_tune). The headline runs the FP32 pair test with FP64 recheck; the
plain FP64 sweep runs on an identical copy of the state and must end bit-identical
(mismatches = 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun), every rank runs an independent replica (different seed) on its
own GPU; there is no data-path collective. Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "trial moves/s, 1 B200: FP32+FP64-recheck vs plain FP64, 0 mismatches; CPU ref"
UNIT = "trial moves/s"
N_BODIES = 1 << 20
PHI = 0.50
SEED = 0x5EED0002
TARGET_ACCEPTANCE = 0.30


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of the FP32 colour passes of this
# workload from ncu. As the passes run, caches kept (--cache-control none): 88-97 MB over the 16
# passes of a sweep, a mean of 5.7 MB per pass (the first pass after the rebuild about 27 MB, the
# others 4.1-4.7 MB from L2 misses). One pass with the caches flushed first (ncu's default):
# 30.72 MB read + 0.04 MB written.
SPHERE_PASS_DRAM_BYTES = 5.7e6
SPHERE_PASS_DRAM_BYTES_COLD = 30.76e6


def aggregate_over_ranks(elapsed, units, world, device):
    """(max of `elapsed` over ranks, sum of `units` over ranks). The whole-job rate is the sum
    of the units all ranks processed over the slowest rank's time. Every rank calls it at the
    same point (two collectives in the same order); world == 1 needs no process group."""
    if world <= 1:
        return float(elapsed), int(units)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(elapsed)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    n = torch.tensor([float(units)], dtype=torch.float64, device=device)
    dist.all_reduce(n, op=dist.ReduceOp.SUM)
    return float(t.item()), int(n.item())


def workload_config(d, extra=None):
    cfg = {"workload": "3-D hard spheres, N=2^20, packing fraction 0.50, periodic cube, FCC start + 0.01 jitter, "
                       "translation moves tuned by Tune (target 0.30, hmc_tune), one ParallelSweep per step",
           "n_bodies": N_BODIES, "packing_fraction": PHI, "box_length": None, "move_size": d,
           "seed": SEED, "l2": "flushed before every timed step (256 MiB device write)"}
    if extra:
        cfg.update(extra)
    return cfg


TUNE_SAMPLES, TUNE_STEPS, D0 = 8000, 32, 0.13


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class ClockSampler:
    """SM clock and clock-event reasons sampled every 5 ms (NVML) while the timed region runs."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown", 0x4: "sw_power_cap",
               0x80: "hw_power_brake_slowdown"}

    def __init__(self, local_rank):
        self.local_rank = local_rank
        self.samples = []
        self.smax = None
        self.stop_flag = threading.Event()
        self.thread = None
        self.error = None

    def _index(self):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [x.strip() for x in vis.split(",") if x.strip()]
        if ids and all(x.isdigit() for x in ids) and self.local_rank < len(ids):
            return int(ids[self.local_rank])
        return self.local_rank

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self._index())
            self.smax = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # no NVML: report it instead of clocks
            self.error = f"nvml unavailable: {e}"
            return

        def run():
            while not self.stop_flag.is_set():
                try:
                    sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                    reasons = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((sm, reasons))
                except Exception as e:
                    self.error = str(e)
                    return
                self.stop_flag.wait(0.005)

        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()

    def stop(self):
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.smax, "reasons": [self.error or "no samples"], "samples": 0}
        reasons = set()
        for _, bits in self.samples:
            for bit, name in self.REASONS.items():
                if bits & bit:
                    reasons.add(name)
        return {"sm_mhz": statistics.median(x for x, _ in self.samples), "sm_max_mhz": self.smax,
                "reasons": sorted(reasons), "samples": len(self.samples), "source": "nvml, 5 ms"}


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def cpu_baseline(pos, L, d, step, seconds=12.0):
    """The oracle's ParallelSweep (a C++ port of the reference) on all host cores."""
    import oracle
    threads = host_threads()
    o = oracle.System(3, [L] * 3, pos, diameter=1.0, seed=SEED, step=step)
    trials, t0, sweeps = 0, time.perf_counter(), 0
    while True:
        a, r = o.parallel_sweep(oracle.TRANSLATE, d, 1.0, 1.0, threads=threads)
        o.increment_step()
        trials += a + r
        sweeps += 1
        el = time.perf_counter() - t0
        if el >= seconds or sweeps >= 16:
            break
    return {"value": trials / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{sweeps} ParallelSweep sweeps of the same 2^20-sphere state ({trials} trial moves, "
                      f"{el:.1f} s, {threads} threads)"}


def oracle_check(ctx, h, pos, L, d, step):
    """One sampled sweep of the timed state checked against the oracle's ParallelSweep: the GPU's
    FP32+recheck sweep and the oracle's FP64 sweep from the same state and counter must give the
    same Count and the same positions (mismatches = bodies whose position differs)."""
    import oracle
    from hoomd_rs_b200 import FP32_RECHECK, TRANSLATE, Microstate, Periodic
    g = Microstate(ctx, Periodic(1.0, [L] * 3), pos, h, seed=SEED)
    g.set_state(pos, step, 0)
    o = oracle.System(3, [L] * 3, pos, diameter=1.0, seed=SEED, step=step)
    c = g.sweep(TRANSLATE, d, 1.0, FP32_RECHECK, n_sweeps=1, increment_step=True)
    t0 = time.perf_counter()
    a, r = o.parallel_sweep(oracle.TRANSLATE, d, 1.0, 1.0, threads=host_threads())
    t_oracle = time.perf_counter() - t0
    mism = int(np.count_nonzero(np.any(g.positions() != o.state()[0], axis=1)))
    g.close()
    return {"sweeps": 1, "count_equal": (c.accepted, c.rejected) == (a, r), "mismatches": mism,
            "trials": a + r, "oracle_s": t_oracle,
            "what": "one FP32+recheck sweep of the timed state against the oracle's ParallelSweep"}


def run_reference(args, rank):
    """--impl reference: the CPU restatement of ParallelSweep (oracle/), timed on host cores."""
    if rank != 0:
        return
    import oracle
    from hoomd_rs_b200 import lattice
    threads = host_threads()
    pos, L = lattice.hard_sphere_box(N_BODIES, PHI, 3, SEED)
    o = oracle.System(3, [L] * 3, pos, diameter=1.0, seed=SEED)
    # the same tuner as the GPU arm (the reference's single stream gives the identical size)
    d = o.tune_stream(oracle.TRANSLATE, D0, 1.0, TARGET_ACCEPTANCE, TUNE_SAMPLES, TUNE_STEPS)
    for _ in range(args.warmup):
        o.parallel_sweep(oracle.TRANSLATE, d, 1.0, 1.0, threads=threads)
        o.increment_step()
    times, trials = [], 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        a, r = o.parallel_sweep(oracle.TRANSLATE, d, 1.0, 1.0, threads=threads)
        times.append(time.perf_counter() - t0)
        o.increment_step()
        trials += a + r
    total = sum(times)
    v = trials / total
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(d, {"box_length": L, "precision": "fp64 (CPU)"}),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{args.steps} full ParallelSweep sweeps of 2^20 spheres, {threads} host "
                                       f"threads"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


REPLICAS, REPLICA_SEED = 256, 0x5EED0004


def replica_specs(seed=REPLICA_SEED, count=REPLICAS):
    """N log-uniform in [1024, 65536], packing fraction uniform in [0.40, 0.54], FCC start; a
    draw is redrawn when the FCC nearest-neighbour distance L / (m sqrt 2) is below
    1 + 2 sqrt(3) 0.01 (the jitter could make two spheres overlap)."""
    from hoomd_rs_b200 import lattice
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < count:
        n = int(round(math.exp(rng.uniform(math.log(1024), math.log(65536)))))
        phi = float(rng.uniform(0.40, 0.54))
        L = lattice.box_length(n, lattice.sphere_number_density(phi, 3), 3)
        m = int(math.ceil((n / 4.0) ** (1.0 / 3.0) - 1e-9))
        if L / (m * math.sqrt(2.0)) < 1.0 + 2.0 * math.sqrt(3.0) * 0.01:
            continue
        out.append((n, phi, seed + 1 + len(out)))
    return out


def partition_replicas(count, rank, world):
    """The replicas rank `rank` of `world` runs: every world-th one from rank (round robin, so
    the large and small boxes of the log-uniform draw spread evenly). No replica is exchanged;
    the ranks only reduce timings and counts."""
    return list(range(rank, count, world))


def run_replicas(args, local_rank):
    """256 independent hard-sphere boxes (one hmc_batch per GPU: the replicas are split over
    the ranks), each with its move size tuned by Tune (target 0.30) on its own; one step = one
    ParallelSweep of every replica."""
    import torch
    import torch.distributed as dist
    from hoomd_rs_b200 import FP32_RECHECK, Batch, Context, Periodic, lattice
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    ctx = Context(local_rank)
    specs_all = replica_specs()
    mine = partition_replicas(len(specs_all), rank, world)
    specs = [specs_all[i] for i in mine]
    reps = []
    for n, phi, seed in specs:
        pos, L = lattice.hard_sphere_box(n, phi, 3, seed)
        reps.append({"boundary": Periodic(1.0, [L] * 3), "positions": pos, "seed": seed})
    b = Batch(ctx, reps)
    # each replica's move size tuned on its own state (hmc_batch_tune = hmc_tune per replica)
    maxima = b.tune(D0, FP32_RECHECK, TARGET_ACCEPTANCE, 2000, 16)
    # the launch-shape autotuner for the replica pass (restores the state afterwards)
    chosen, ms = b.autotune(maxima, FP32_RECHECK, sweeps=2)

    def timed(captured):
        # captured: every sweep one CUDA-graph launch, all steps in one call with one wait at the
        # end; else one call per step, each launching its kernels and waiting for its counts
        b.set_captured_sweeps(captured)
        for _ in range(args.warmup):
            b.sweep(maxima, FP32_RECHECK, increment_step=True)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        launches0 = b.kernel_launches()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        trials = 0
        if captured:
            _, tot = b.sweep(maxima, FP32_RECHECK, n_sweeps=args.steps, increment_step=True)
            trials = tot.total()
        else:
            for _ in range(args.steps):
                _, tot = b.sweep(maxima, FP32_RECHECK, increment_step=True)
                trials += tot.total()
        e1.record()
        torch.cuda.synchronize()
        t, tr = aggregate_over_ranks(e0.elapsed_time(e1) / 1e3, trials, world, "cuda")
        return t, tr, b.kernel_launches() - launches0

    # captured first (the same sweeps after the start as the single-box headline times), then
    # launched, then captured again: the state moves on from the lattice start, so the two
    # captured runs bracket the launched one
    sampler = ClockSampler(local_rank)
    sampler.start()
    t_max, trials_all, launches = timed(True)
    t_launched, trials_launched, _ = timed(False)
    t_again, trials_again, _ = timed(True)
    clocks = sampler.stop()
    over = b.overlap_counts()
    _, over_sum = aggregate_over_ranks(0.0, int(over.sum()), world, "cuda")
    n_total = sum(n for n, _, _ in specs_all)
    torch.cuda.synchronize()
    t_sdf = time.perf_counter()
    pressures = b.pressures(0.02, 40)
    t_sdf = time.perf_counter() - t_sdf
    line = {"metric": "trial moves/s, 256-replica hard-sphere batch", "value": trials_all / t_max, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "fp32 pair test + fp64 recheck", "data": "synthetic",
            "config": {"workload": "256 hard-sphere boxes, N log-uniform [1024, 65536], packing fraction U[0.40, 0.54], "
                                   "FCC starts, per-replica move sizes tuned to 0.30, one batched ParallelSweep of "
                                   "every replica per step", "n_bodies_total": n_total, "replicas": len(specs_all),
                       "partition": f"round robin over {world} rank(s), {len(specs)} replicas on rank {rank}",
                       "timing": "CUDA events around the batched sweep calls, max over ranks",
                       "sweeps": "captured: each sweep one CUDA-graph launch (rounds loop, origins, counts and "
                                 "Counters on the device), the timed steps in one call",
                       "l2": "not flushed: the batch's body arrays (about 4e6 bodies) exceed L2"},
            "launched": {"value": trials_launched / t_launched, "ms_per_step": 1e3 * t_launched / args.steps,
                         "what": "one hmc_batch_sweep call per step, kernels launched one by one; timed after "
                                 "the captured steps"},
            "captured_after": {"value": trials_again / t_again, "ms_per_step": 1e3 * t_again / args.steps,
                               "what": "captured again, after the launched steps"},
            "launch_variant": {"chosen": chosen, "ms_per_sweep": [round(float(x), 4) for x in ms]},
            "overlaps_after": over_sum, "gpu_launches": launches, "clocks": clocks,
            "sdf_pressure": {"estimator": "beta P per replica from its scale distribution (x_max 0.02, 40 bins), "
                                          "after the timed sweeps (rank 0's replicas)", "min": float(pressures.min()),
                             "median": float(np.median(pressures)), "max": float(pressures.max()),
                             "ms_all_replicas": 1e3 * t_sdf}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    b.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_lj_replicas(args, local_rank):
    """64 independent Lennard-Jones boxes of 8192 bodies (rho 0.8, r_cut = r_shift = 2.5), each
    at its own kT drawn from U[0.8, 2.0], in one hmc_batch; one step = one ParallelSweep of
    every replica. Also timed: FP64, and the same 64 boxes swept one Microstate after another
    (what a caller without batches would do)."""
    import torch
    import torch.distributed as dist
    import oracle
    from hoomd_rs_b200 import (FP32_RECHECK, FP64, TRANSLATE, Batch, Context, Isotropic, LennardJones, Microstate,
                               PairwiseCutoff, Periodic, Shifted, lattice)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    ctx = Context(local_rank)
    n, n_rep, rho, r_cut, d = 8192, 64, 0.8, 2.5, 0.1
    kts_all = np.random.default_rng(0x5EED0050).uniform(0.8, 2.0, n_rep)
    mine = partition_replicas(n_rep, rank, world)  # the replicas of this rank
    kts = kts_all[mine]
    h = PairwiseCutoff(Isotropic(Shifted(LennardJones(1.0, 1.0), r_cut), r_cut))
    reps = []
    for k in mine:
        pos, L = lattice.lennard_jones_box(n, rho, 3, 0x5EED0050 + k)
        reps.append({"boundary": Periodic(r_cut, [L] * 3), "positions": pos, "seed": 0x5EED0050 + k, "hamiltonian": h})

    tuned = {}

    def timed_batch(precision, steps, warmup):
        b = Batch(ctx, reps)
        for _ in range(warmup):
            b.sweep(d, precision, increment_step=True, temperatures=kts)
        # the launch-shape autotuner for the replica pass (restores the state afterwards)
        tuned[precision] = b.autotune(d, precision, sweeps=2, temperatures=kts)
        # every sweep one CUDA-graph launch, the timed steps in one call with one wait at the end
        b.set_captured_sweeps(True)
        b.sweep(d, precision, increment_step=True, temperatures=kts)  # builds the graph
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        launches0 = b.kernel_launches()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        _, tot = b.sweep(d, precision, n_sweeps=steps, increment_step=True, temperatures=kts)
        trials = tot.total()
        e1.record()
        torch.cuda.synchronize()
        el, trials_all = aggregate_over_ranks(e0.elapsed_time(e1) / 1e3, trials, world, "cuda")
        out = (trials_all / el, 1e3 * el / steps, b.kernel_launches() - launches0,
               [b.positions(k) for k in (0, len(reps) // 2)])
        b.close()
        return out

    sampler = ClockSampler(local_rank)
    sampler.start()
    v32, ms32, launches, p32 = timed_batch(FP32_RECHECK, args.steps, args.warmup)
    clocks = sampler.stop()
    v64, ms64, _, p64 = timed_batch(FP64, args.steps, args.warmup)
    if world > 1:  # the rest (one system after another, the CPU baseline) is a one-GPU comparison
        if rank == 0:
            print(json.dumps({"metric": "trial moves/s, 64-replica Lennard-Jones batch", "value": v32, "unit": UNIT,
                              "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms32,
                              "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                              "dtype": "fp32 sums + fp64 recheck (fp64 state)", "data": "synthetic",
                              "config": {"workload": "64 Lennard-Jones boxes of 8192 bodies split round robin over "
                                                     f"{world} ranks", "replicas": n_rep,
                                         "timing": "CUDA events around the batched sweeps, max over ranks"},
                              "fp64": {"value": v64, "ms_per_step": ms64}, "gpu_launches": launches,
                              "clocks": clocks}), flush=True)
        dist.barrier()
        dist.destroy_process_group()
        return
    # the same replicas as separate systems, swept one after another
    singles = [Microstate(ctx, r["boundary"], r["positions"], h, seed=r["seed"]) for r in reps]
    for k, m in enumerate(singles):
        m.sweep(TRANSLATE, d, float(kts[k]), FP32_RECHECK, n_sweeps=args.warmup, increment_step=True)
    s_steps = max(1, min(args.steps, 5))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s_trials = 0
    for _ in range(s_steps):
        for k, m in enumerate(singles):
            s_trials += m.sweep(TRANSLATE, d, float(kts[k]), FP32_RECHECK, n_sweeps=1, increment_step=True).total()
    torch.cuda.synchronize()
    v_single = s_trials / (time.perf_counter() - t0)
    for m in singles:
        m.close()
    line = {"metric": "trial moves/s, 64-replica Lennard-Jones batch", "value": v32, "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms32, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32 sums + fp64 recheck (fp64 state)", "data": "synthetic",
            "config": {"workload": "64 Lennard-Jones boxes of 8192 bodies, rho 0.8, eps = sigma = 1, "
                                   "r_cut = r_shift = 2.5, kT_k ~ U[0.8, 2.0], FCC + 0.01 jitter, translation 0.1, "
                                   "one batched ParallelSweep of every replica per step", "n_bodies_total": n * n_rep,
                       "replicas": n_rep, "timing": "CUDA events around the batched sweep calls",
                       "sweeps": "captured: each sweep one CUDA-graph launch, the timed steps in one call",
                       "l2": "not flushed between sweeps (the timed steps run in one call); the batch's arrays "
                             "(524288 bodies, about 70 MB) fit in L2"},
            "fp64": {"value": v64, "ms_per_step": ms64},
            "mismatches": int(sum(np.count_nonzero(np.any(a != b, axis=1)) for a, b in zip(p32, p64))),
            "one_system_after_another": {"value": v_single, "precision": "fp32_recheck"},
            "launch_variants": {("fp32_recheck" if p == FP32_RECHECK else "fp64"):
                                {"chosen": c, "ms_per_sweep": [round(float(x), 4) for x in m]}
                                for p, (c, m) in tuned.items()},
            "gpu_launches": launches, "clocks": clocks}
    if not args.no_cpu_baseline:
        threads = host_threads()
        r0 = reps[0]
        o = oracle.System(3, r0["boundary"].edge_lengths, r0["positions"], seed=r0["seed"],
                          interaction=oracle.LENNARD_JONES, lj_epsilon=1.0, lj_sigma=1.0, lj_r_cut=r_cut,
                          lj_r_shift=r_cut)
        trials, t0, sweeps = 0, time.perf_counter(), 0
        while True:
            a_, r_ = o.parallel_sweep(oracle.TRANSLATE, d, float(kts[0]), r_cut, threads=threads)
            o.increment_step()
            trials += a_ + r_
            sweeps += 1
            el = time.perf_counter() - t0
            if el >= 10.0 or sweeps >= 200:
                break
        line["cpu_baseline"] = {"value": trials / el, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{sweeps} ParallelSweep sweeps of replica 0 ({el:.1f} s, {threads} threads)"}
    print(json.dumps(line), flush=True)


def run_config(args, local_rank):
    """The other single-box configurations, FP32+recheck and FP64 from the same state,
    device-timed per step like the headline, with the oracle's ParallelSweep on the host cores
    as the CPU baseline (a bounded sample of whole sweeps). A step: one sweep (disks, LJ) or one
    translation plus one rotation sweep (cubes)."""
    import torch
    import oracle
    from hoomd_rs_b200 import (FP32_RECHECK, FP64, ROTATE, TRANSLATE, Anisotropic, ApproximateShapeOverlap, Context,
                               ConvexPolygon, ConvexPolyhedron, ConvexSurfaceMesh2d, HardShape, HardSphere, Isotropic,
                               LennardJones, Microstate, OverlapPenalty, PairwiseCutoff, Periodic, Shifted, lattice,
                               place_single_site_orientable_bodies)
    torch.cuda.set_device(local_rank)
    ctx = Context(local_rank)
    kind = args.workload
    ori, extra = None, {}
    if kind == "disks":
        n, seed = 4096, 0x5EED0001
        pos, L = lattice.hard_sphere_box(n, 0.70, 2, seed)
        h, bound, dim = PairwiseCutoff(HardSphere(1.0)), Periodic(1.0, [L, L]), 2
        moves = [(TRANSLATE, 0.1)]
        okw = dict(diameter=1.0)
        desc = "2-D hard disks, N=4096, area fraction 0.70, square lattice + 0.01 jitter, translation 0.1"
        orng = 1.0
    elif kind == "cubes":
        n, seed = 1 << 18, 0x5EED0003
        cube = np.array([[x, y, z] for x in (-0.5, 0.5) for y in (-0.5, 0.5) for z in (-0.5, 0.5)])
        L = (n / 0.55) ** (1.0 / 3.0)
        pos = lattice.cubic_lattice(n, L, 3, seed, jitter=0.0)
        h, bound, dim = PairwiseCutoff(HardShape(ConvexPolyhedron.with_vertices(cube))), Periodic(math.sqrt(3), [L] * 3), 3
        moves = [(TRANSLATE, 0.08), (ROTATE, 0.1)]
        okw = dict(interaction=oracle.HARD_CONVEX_POLYHEDRON, vertices=cube)
        desc = "hard cubes (vertices +-0.5), N=2^18, packing fraction 0.55, simple-cubic start, identity versors, " \
               "translation 0.08 then rotation 0.1 per step"
        orng = math.sqrt(3)
    elif kind == "hexagons":
        # benchmarks/src/mc/regular_polygon.rs:187-244: ConvexSurfaceMesh2d hexagons (circumradius 0.5) at
        # packing fraction 0.68, placed by place_single_site_orientable_bodies on the device, then one
        # translation (0.2) and one rotation (2 pi / 6) ParallelSweep per step
        n, seed = 1 << 16, 0x5EED0008
        mesh = ConvexSurfaceMesh2d.from_point_set(ConvexPolygon.regular(6).vertices)
        h = PairwiseCutoff(HardShape(mesh))
        r = h.maximum_interaction_range
        insert = PairwiseCutoff(Anisotropic(ApproximateShapeOverlap.new(mesh, OverlapPenalty(), 0.01), r))
        rho = 0.68 / (1.5 * math.sqrt(3.0) * 0.25)
        t0 = time.perf_counter()
        g = place_single_site_orientable_bodies(ctx, n, rho, r, insert, h, 2, seed=seed)
        g.sweep(TRANSLATE, 0.2, 1.0, FP64, n_sweeps=20, increment_step=True)  # a short relaxation
        placed_s = time.perf_counter() - t0
        pos, ori, L = g.positions(), g.orientations(), float(g.box()[0])
        assert g.overlap_count() == 0
        g.close()
        bound, dim = Periodic(r, [L, L]), 2
        moves = [(TRANSLATE, 0.2), (ROTATE, 2.0 * math.pi / 6.0)]
        okw = dict(interaction=oracle.HARD_CONVEX_SURFACE_MESH_2D, vertices=mesh.vertices)
        desc = "2-D hexagons (ConvexSurfaceMesh2d, circumradius 0.5, separating axes), N=2^16, packing fraction " \
               "0.68, placed on the device by QuickInsert/QuickCompress under the approximate shape overlap, " \
               "then 20 translation sweeps; translation 0.2 then rotation 2 pi/6 per step"
        orng = r
        extra = {"placement_s": placed_s}
    elif kind == "squares":
        n, seed = 1 << 18, 0x5EED0007
        square = np.array([[-0.5, -0.5], [0.5, -0.5], [0.5, 0.5], [-0.5, 0.5]])
        L = math.sqrt(n / 0.6)
        pos = lattice.cubic_lattice(n, L, 2, seed, jitter=0.0)
        h = PairwiseCutoff(HardShape(ConvexPolygon.with_vertices(square)))
        bound, dim = Periodic(math.sqrt(2), [L, L]), 2
        moves = [(TRANSLATE, 0.1), (ROTATE, 0.1)]
        okw = dict(interaction=oracle.HARD_CONVEX_POLYGON, vertices=square)
        desc = "2-D hard squares (vertices +-0.5, XenoCollide), N=2^18, area fraction 0.60, square-lattice start, " \
               "angles 0, translation 0.1 then rotation 0.1 per step"
        orng = math.sqrt(2)
    else:
        n, seed = 1 << 19, 0x5EED0005
        pos, L = lattice.lennard_jones_box(n, 0.8, 3, seed)
        h = PairwiseCutoff(Isotropic(Shifted(LennardJones(1.0, 1.0), 2.5), 2.5))
        bound, dim = Periodic(2.5, [L] * 3), 3
        moves = [(TRANSLATE, 0.1)]
        okw = dict(interaction=oracle.LENNARD_JONES, lj_epsilon=1.0, lj_sigma=1.0, lj_r_cut=2.5, lj_r_shift=2.5)
        desc = "Lennard-Jones eps = sigma = 1, r_cut = r_shift = 2.5, N=2^19, rho 0.8, kT 1.0, FCC + 0.01 jitter, " \
               "translation 0.1"
        orng = 2.5
    stream = torch.cuda.Stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def timed(precision):
        m = Microstate(ctx, bound, pos, h, seed=seed, orientations=ori)
        m.set_stream(stream.cuda_stream)
        for _ in range(args.warmup):
            for mv, mx in moves:
                m.sweep(mv, mx, 1.0, precision, n_sweeps=1, increment_step=True)
        # the launch-shape autotuner on the first move (restores the state afterwards)
        chosen, ms_var = m.autotune(moves[0][0], moves[0][1], 1.0, precision, sweeps=2)
        ms, trials, acc, rech, checks, amb = 0.0, 0, 0, 0, 0, 0
        launches0 = m.profile()["kernel_launches"]
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            for mv, mx in moves:
                c = m.sweep(mv, mx, 1.0, precision, n_sweeps=1, increment_step=True)
                trials += c.total()
                acc += c.accepted
                rech += c.rechecks
                amb += c.order_ambiguous
                checks += c.pair_checks
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
        out = {"value": trials / (ms / 1e3), "ms_per_step": ms / args.steps, "acceptance": acc / max(trials, 1),
               "recheck_fraction": rech / max(checks, 1), "launches": m.profile()["kernel_launches"] - launches0,
               "order_ambiguous": amb,
               "launch_variant": {"chosen": chosen, "ms_per_sweep": [round(float(x), 4) for x in ms_var]}}
        pos_end = m.positions()
        m.close()
        return out, pos_end

    sampler = ClockSampler(local_rank)
    sampler.start()
    r32, p32 = timed(FP32_RECHECK)
    clocks = sampler.stop()
    r64, p64 = timed(FP64)
    side = {}
    if kind == "disks":
        # the configuration's 1000 sweeps as one call: the sweeps are enqueued back to back (the
        # host waits once per 64) instead of one call and one wait per sweep
        runs = {}
        for name, prec in (("fp32_recheck", FP32_RECHECK), ("fp64", FP64)):
            m = Microstate(ctx, bound, pos, h, seed=seed, orientations=ori)
            m.set_stream(stream.cuda_stream)
            m.sweep(TRANSLATE, moves[0][1], 1.0, prec, n_sweeps=args.warmup, increment_step=True)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            c = m.sweep(TRANSLATE, moves[0][1], 1.0, prec, n_sweeps=1000, increment_step=True)
            el = time.perf_counter() - t0
            runs[name] = {"value": c.total() / el, "ms_per_sweep": 1e3 * el / 1000, "positions": m.positions()}
            m.close()
        side["sweeps_1000_one_call"] = {
            **{k: {"value": v["value"], "ms_per_sweep": v["ms_per_sweep"]} for k, v in runs.items()},
            "mismatches": int(np.count_nonzero(np.any(runs["fp32_recheck"]["positions"] != runs["fp64"]["positions"],
                                                      axis=1))),
            "what": "1000 sweeps in one Microstate.sweep call, wall clock around the call (L2 not flushed: the "
                    "4096-disk state stays in L2)"}
    line = {"metric": f"trial moves/s, {kind}", "value": r32["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r32["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32 pair test + fp64 recheck (fp64 state)", "data": "synthetic",
            "config": {"workload": desc, "n_bodies": n, "box_length": L,
                       "l2": "flushed before every timed step (256 MiB device write)", **extra},
            "fp64": {"value": r64["value"], "ms_per_step": r64["ms_per_step"]},
            "mismatches": int(np.count_nonzero(np.any(p32 != p64, axis=1))), "acceptance": r32["acceptance"],
            "recheck_fraction": r32["recheck_fraction"], "gpu_launches": r32["launches"], "clocks": clocks,
            "order_ambiguous": {"fp32_recheck": r32["order_ambiguous"], "fp64": r64["order_ambiguous"],
                                "what": "decisions another summation order of the FP64 pair energies could change"},
            "launch_variants": {"fp32_recheck": r32["launch_variant"], "fp64": r64["launch_variant"]}, **side}
    if not args.no_cpu_baseline:
        threads = host_threads()
        o = oracle.System(dim, [L] * dim, pos, ori, seed=seed, **okw)
        trials, t0, sweeps = 0, time.perf_counter(), 0
        while True:
            for mv, mx in moves:
                a, r = o.parallel_sweep(oracle.TRANSLATE if mv == TRANSLATE else oracle.ROTATE, mx, 1.0, orng,
                                        threads=threads)
                o.increment_step()
                trials += a + r
                sweeps += 1
            el = time.perf_counter() - t0
            if el >= 10.0 or sweeps >= 64:
                break
        line["cpu_baseline"] = {"value": trials / el, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{sweeps} ParallelSweep sweeps from the start state ({el:.1f} s, "
                                          f"{threads} threads)"}
    print(json.dumps(line), flush=True)


def run_gsd(args, local_rank):
    """GSD snapshot output of the headline state (2^20 spheres): one step appends one HOOMD
    frame (configuration/step, particles/N, FP32 site positions, dimensions, box) from device
    state and ends it, through HoomdGsdFile.append_microstate (hmc_gsd_append_system). The file
    lives in a temporary directory (page cache); the sync at close is outside the timed steps.
    The CPU baseline is the oracle's restatement of the same frame (site transform and FP32
    conversion in C++, file layer in Python) writing the same bytes."""
    import tempfile

    import torch
    import oracle
    from oracle import gsd_oracle
    from hoomd_rs_b200 import FP32_RECHECK, TRANSLATE, Context, HardSphere, Microstate, PairwiseCutoff, Periodic
    from hoomd_rs_b200 import lattice
    from hoomd_rs_b200.gsd import HoomdGsdFile

    torch.cuda.set_device(local_rank)
    ctx = Context(local_rank)
    pos, L = lattice.hard_sphere_box(N_BODIES, PHI, 3, SEED)
    m = Microstate(ctx, Periodic(1.0, [L] * 3), pos, PairwiseCutoff(HardSphere(1.0)), seed=SEED)
    m.sweep(TRANSLATE, D0, 1.0, FP32_RECHECK, n_sweeps=2, increment_step=True)
    frame_bytes = N_BODIES * 12 + 8 + 4 + 1 + 24
    with tempfile.TemporaryDirectory() as tmp:
        f = HoomdGsdFile.create(os.path.join(tmp, "frames.gsd"))
        for _ in range(args.warmup):
            f.append_microstate(m).end()
        launches0 = m.profile()["kernel_launches"]
        sampler = ClockSampler(local_rank)
        sampler.start()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            f.append_microstate(m).end()
        el = time.perf_counter() - t0
        clocks = sampler.stop()
        launches = m.profile()["kernel_launches"] - launches0
        f.close()
    value = args.steps / el
    line = {"metric": "GSD frames/s, 2^20 hard spheres (FP32 positions from device state)", "value": value,
            "unit": "frames/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 state -> f32 frame", "data": "synthetic",
            "config": {"workload": "append_microstate + end per step, 2^20 hard spheres at packing fraction 0.50 "
                                   "(headline state after 2 sweeps), file in a temporary directory",
                       "n_bodies": N_BODIES, "frame_bytes": frame_bytes,
                       "l2": "state (33.5 MB) smaller than L2; the frame's cost is the host write"},
            "file_write_gbs": frame_bytes * args.steps / el / 1e9,
            "roofline": None, "roofline_note": "host-bound: one encoding kernel and one 12.6 MB device-to-host "
                                               "copy per frame; the page-cache write dominates",
            "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": N_BODIES * 12},
            "gpu_launches": launches, "clocks": clocks}
    if not args.no_cpu_baseline:
        o = oracle.System(3, [L] * 3, m.positions(), seed=SEED)
        w = gsd_oracle.Writer("hoomd-rs-b200", "hoomd", (1, 4))
        frames, t0 = 0, time.perf_counter()
        with tempfile.TemporaryDirectory() as tmp:
            while True:
                p32, _ = o.gsd_frame()
                w.append_microstate(frames, 3, [L] * 3, p32)
                w.end_frame()
                w.sync_all()
                frames += 1
                if time.perf_counter() - t0 >= 5.0 or frames >= 50:
                    break
            with open(os.path.join(tmp, "frames.gsd"), "wb") as fh:
                fh.write(w.image)
        el = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": frames / el, "unit": "frames/s", "cores": 1, "kind": "port",
                                "sample": f"{frames} frames of the same state through the oracle's frame "
                                          f"restatement and file layer ({el:.1f} s, 1 thread)"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="hard_spheres",
                    choices=["hard_spheres", "replicas", "lj_replicas", "disks", "cubes", "squares", "hexagons", "lj",
                             "gsd"],
                    help="hard_spheres: the headline (2^20 spheres); replicas: 256 independent boxes in one batch; "
                         "disks: 4096 hard disks; cubes: 2^18 hard cubes; hexagons: 2^16 hexagons placed on the "
                         "device; lj: 2^19 Lennard-Jones sites; "
                         "gsd: GSD frames of the 2^20-sphere state")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload == "replicas":
        run_replicas(args, local_rank)
        return
    if args.workload == "lj_replicas":
        run_lj_replicas(args, local_rank)
        return
    if args.workload in ("disks", "cubes", "squares", "hexagons", "lj"):
        run_config(args, local_rank)
        return
    if args.workload == "gsd":
        run_gsd(args, local_rank)
        return

    import torch
    import torch.distributed as dist
    from hoomd_rs_b200 import FP32_RECHECK, FP64, TRANSLATE, Context, HardSphere, Microstate, PairwiseCutoff, Periodic
    from hoomd_rs_b200 import lattice

    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    ctx = Context(local_rank)
    seed = SEED + rank
    pos, L = lattice.hard_sphere_box(N_BODIES, PHI, 3, seed)
    h = PairwiseCutoff(HardSphere(1.0))
    tuner = Microstate(ctx, Periodic(1.0, [L] * 3), pos, h, seed=seed)
    d = tuner.tune(TRANSLATE, D0, 1.0, FP32_RECHECK, TARGET_ACCEPTANCE, TUNE_SAMPLES, TUNE_STEPS)
    # a few sweeps away from the lattice before the copies start
    tuner.sweep(TRANSLATE, d, 1.0, FP32_RECHECK, n_sweeps=4, increment_step=True)
    start_pos, step0, _ = tuner.state()
    # the launch-shape autotuner, per precision: it records its choice for this workload's density
    # band, which the timed systems below pick up (it restores the tuner's state afterwards)
    variants = {}
    for name, prec in (("fp32_recheck", FP32_RECHECK), ("fp64", FP64)):
        # both passes (a lane or a warp per trial) and their variants; the fastest is recorded
        chosen, ms = tuner.autotune(TRANSLATE, d, 1.0, prec, sweeps=4)
        variants[name] = {"chosen": chosen, "cooperative_pass": tuner.cooperative_pass(prec),
                          "ms_per_sweep": [round(float(x), 4) for x in ms]}
    tuner.close()

    stream = torch.cuda.Stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def make_system():
        m = Microstate(ctx, Periodic(1.0, [L] * 3), pos, h, seed=seed)
        m.set_state(start_pos, step0, 0)
        m.set_stream(stream.cuda_stream)
        return m

    def timed(m, precision, steps, warmup, profile=False):
        for _ in range(warmup):
            m.sweep(TRANSLATE, d, 1.0, precision, n_sweeps=1, increment_step=True)
        if profile:
            m.profile(enable=True, reset=True)
        launches0 = m.profile()["kernel_launches"]
        ms, acc, trials, rech, checks, maxerr = 0.0, 0, 0, 0, 0, 0.0
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            c = m.sweep(TRANSLATE, d, 1.0, precision, n_sweeps=1, increment_step=True)
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
            acc += c.accepted
            trials += c.total()
            rech += c.rechecks
            checks += c.pair_checks
            maxerr = max(maxerr, c.max_fp32_error)
        prof = m.profile(enable=False)
        return {"ms": ms, "trials": trials, "accepted": acc, "rechecks": rech, "pair_checks": checks,
                "max_err": maxerr, "launches": prof["kernel_launches"] - launches0, "profile": prof}

    a = make_system()
    b = make_system()
    sampler = ClockSampler(local_rank)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    ra = timed(a, FP32_RECHECK, args.steps, args.warmup, profile=True)
    clocks = sampler.stop()
    rb = timed(b, FP64, args.steps, args.warmup)
    # like for like: FP64 in the one-lane-per-trial pass that the FP32 mode runs (the FP64 mode
    # runs the warp-cooperative pass, the faster one in FP64)
    c1 = make_system()
    c1.set_cooperative_pass(FP64, False)
    rc1 = timed(c1, FP64, args.steps, args.warmup)
    torch.cuda.synchronize()
    pa, pb, pc = a.positions(), b.positions(), c1.positions()
    c1.close()
    mismatches = int(np.count_nonzero(np.any(pa != pb, axis=1)) + np.count_nonzero(np.any(pa != pc, axis=1)))
    overlaps = a.overlap_count()

    # whole-job aggregate: units of all ranks over the slowest rank's device time
    t_max, trials_all = aggregate_over_ranks(ra["ms"], ra["trials"], world, "cuda")
    value = trials_all / (t_max / 1e3)
    fp64_value = rb["trials"] / (rb["ms"] / 1e3)
    fp64_lane_value = rc1["trials"] / (rc1["ms"] / 1e3)

    # roofline of the dominant kernel (the colour-pass sweep), algorithmic bytes per launch
    prof = ra["profile"]
    launches = max(prof["sweep_launches"], 1)
    t_launch = prof["sweep_ms"] / 1e3 / launches
    shape = math.floor(L / 1.0)
    shape -= shape % 2  # compute_dimensions (hoomd-mc/src/hypercuboid.rs:188-228)
    cells = shape ** 3
    trials_per_launch = ra["trials"] / launches
    acc_per_launch = ra["accepted"] / launches
    bytes_per_launch = N_BODIES * 12 + (cells + 1) * 4 + trials_per_launch * 24 + acc_per_launch * 84
    peak, peak_kind = measured_peak_hbm()
    achieved = bytes_per_launch / t_launch / 1e9

    # end to end through the C ABI with pinned host buffers: every step uploads the state
    # (hmc_set_state), sweeps, and downloads the new state (hmc_get_state)
    e2e_steps = max(3, min(args.steps, 10))
    host_in = torch.empty((N_BODIES, 3), dtype=torch.float64, pin_memory=True).numpy()
    host_out = torch.empty((N_BODIES, 3), dtype=torch.float64, pin_memory=True).numpy()
    host_in[:] = pa
    e2e_trials, t_e2e = 0, 0.0
    for _ in range(e2e_steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        a.set_state(host_in, a.step(), 0)
        c = a.sweep(TRANSLATE, d, 1.0, FP32_RECHECK, n_sweeps=1, increment_step=True)
        a.state(out=host_out)
        t_e2e += time.perf_counter() - t0
        e2e_trials += c.total()
        host_in, host_out = host_out, host_in
    t_e2e_max, e2e_trials_all = aggregate_over_ranks(t_e2e, e2e_trials, world, "cuda")
    e2e_value = e2e_trials_all / t_e2e_max

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32 pair test + fp64 recheck (fp64 state)", "data": "synthetic",
        "config": workload_config(d, {"box_length": L, "precision": "fp32_recheck", "replicas": world}),
        "fp64": {"value": fp64_value, "ms_per_step": rb["ms"] / args.steps,
                 "speedup_fp32_recheck_over_fp64": value / world / fp64_value if world == 1 else None,
                 "one_lane_per_trial": {"value": fp64_lane_value, "ms_per_step": rc1["ms"] / args.steps,
                                        "speedup_fp32_recheck_over_it":
                                            value / world / fp64_lane_value if world == 1 else None,
                                        "what": "FP64 in the FP32 mode's pass structure, one lane per trial"}},
        "mismatches": mismatches, "overlaps_after": overlaps,
        "acceptance": ra["accepted"] / max(ra["trials"], 1),
        "recheck_fraction": ra["rechecks"] / max(ra["pair_checks"], 1), "max_fp32_error": ra["max_err"],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": SPHERE_PASS_DRAM_BYTES, "kernel": "k_sweep_sphere<3,fp32>",
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per FP32 colour pass, "
                                       "mean over the 16 passes of a sweep as they run (--cache-control none)",
                     "traffic_cold": SPHERE_PASS_DRAM_BYTES_COLD,
                     "bytes_per_launch": bytes_per_launch, "launch_ms": t_launch * 1e3,
                     "peak_source": f"{peak_kind} hbm_gbs"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": N_BODIES * 3 * 8,
                "d2h_bytes_per_step": N_BODIES * 3 * 8},
        "gpu_launches": ra["launches"],
        "clocks": clocks,
        "launch_variants": variants,
        "time_split": {"unit": "ms per sweep (CUDA events inside the timed FP32 sweeps)",
                       "cell_list_rebuild": prof["rebuild_ms"] / max(prof["sweeps"], 1),
                       "colour_passes": prof["sweep_ms"] / max(prof["sweeps"], 1),
                       "whole_step": t_max / args.steps},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(start_pos, L, d, step0)
        line["oracle_check"] = oracle_check(ctx, h, pa, L, d, a.step())
    if rank == 0:
        print(json.dumps(line), flush=True)
    a.close()
    b.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
