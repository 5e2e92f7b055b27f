#!/usr/bin/env python
"""Timestep throughput of the B200 pipe-flow hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload batched|cfg2|cfg1]

Default workload ("batched"): 64 independent pipes with sizes drawn by
numpy default_rng(3) uniformly from N in {32,48,64}, K in {16,32,64},
M in {12,24,32}, Re uniform in [1800,3000], alpha uniform in [0.8,1.6],
Mp=1, dt=0.01, each seeded (seeds 1000+) with a solenoidal perturbation at
1e-3 of the laminar energy, run in mixed precision (FP32 transforms and
u x curl(u), FP64 elsewhere) as one CUDA graph per batch timestep.  A "step"
is one pass of the main.f90 loop body for every pipe (nonlinear terms,
predictor, corrector iterated to convergence per pipe); `value` counts
pipe-timesteps per second.  The line also reports the plain FP64 drop-in
(the same pipes stepped one at a time) and the single large pipe N=64,
K=128, M=48, Mp=2, Re=5300, alpha=0.5, dt=0.005 in FP64.

Multi-GPU runs are independent replicas (one batch per rank, seeds offset
by rank, no collective on the data path); the only collectives are the
barrier and the max over ranks of the timed duration.

--impl reference times the CPU restatement of the reference's step (the FP64
oracle; the Fortran reference has no compiler on this image) on a bounded
sample of the same workload, on rank 0 only.
"""
from __future__ import annotations

import argparse
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
sys.path.insert(0, str(ROOT / "softx-d-17-00015_b200"))

METRIC = "batched timesteps/s vs plain at ≤1e-6 rel-L2 vs FP64; serve p50/p99 latency"
PHYS = ("N", "K", "M", "Mp", "Re", "alpha", "dt")
SINGLE = {
    "cfg2": dict(N=64, K=128, M=48, Mp=2, Re=5300.0, alpha=0.5, dt=0.005, energy=0.1, seed=2, spinup=500),
    "cfg1": dict(N=40, K=24, M=16, Mp=1, Re=2000.0, alpha=1.25, dt=0.01, energy=1e-3, seed=1, spinup=0),
}


def batched_configs(npipes: int = 64, seed: int = 3):
    """The uneven pipe mix of the batched workload (sizes, Re, alpha)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(npipes):
        out.append(dict(N=int(rng.choice([32, 48, 64])), K=int(rng.choice([16, 32, 64])),
                        M=int(rng.choice([12, 24, 32])), Mp=1, Re=float(rng.uniform(1800, 3000)),
                        alpha=float(rng.uniform(0.8, 1.6)), dt=0.01))
    return out


def transform_flops(d):
    """FFT flops of one nonlinear evaluation of a pipe (5 L log2 L per complex
    FFT of length L): six inverse and three forward z transforms of length 3K
    over M columns, and per z-row pair six inverse and three forward packed
    theta transforms of length 3M, at each radial point."""
    Z, Th = 3 * d["K"], 3 * d["M"]
    fz, ft = 5 * Z * math.log2(Z), 5 * Th * math.log2(Th)
    return d["N"] * (9 * d["M"] * fz + 9 * (Z / 2) * ft)


def harmonics_count(d):
    return (2 * d["K"] - 1) * d["M"] - (d["K"] - 1)


def coll_bytes(d):
    return d["N"] * harmonics_count(d) * 16  # one FP64 complex coll field, S


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.rows = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                      f"--id={self.idx}"], capture_output=True, text=True, timeout=5).stdout
                for line in out.strip().splitlines():
                    self.rows.append([x.strip() for x in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def cpu_baseline(workload: str, nsample: int):
    """Time the CPU restatement of the reference step (oracle/pipeflow_cpu.cpp:
    C++, OpenMP over modes and radial points, every host thread) on a bounded
    sample of the workload: one step of each of the first `nsample` pipes of
    the mix after one warm-up step (batched), or `nsample` steps of the single
    pipe.  The set-up (mesh, factors, influence matrices) comes from the numpy
    oracle and is not timed."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pipeflow_oracle as O
    import pipeflow_cpu as PC
    threads = PC.threads()
    if workload == "batched":
        cfgs = batched_configs()[:nsample]
        pipes = []
        for i, d in enumerate(cfgs):
            o = O.Pipe(O.PipeConfig(**d))
            o.vel_matrices()
            o.set_state(*O.seeded_state(o, 1000 + i, 1e-3))
            c = PC.CpuPipe(o)
            c.timestep()
            pipes.append(c)
        t0 = time.perf_counter()
        for c in pipes:
            c.timestep()
        dt = time.perf_counter() - t0
        return {"value": len(pipes) / dt, "unit": "timesteps/s", "cores": threads, "kind": "port",
                "sample": f"one main-loop step of each of {'all' if len(pipes) == 64 else 'the first'} {len(pipes)} pipes of the 64-pipe mix in FP64, "
                          f"C++/OpenMP restatement of the reference step on {threads} host threads, after one "
                          f"warm-up step (set-up not timed)"}
    w = SINGLE[workload]
    o = O.Pipe(O.PipeConfig(**{k: w[k] for k in PHYS}))
    o.vel_matrices()
    o.set_state(*O.seeded_state(o, w["seed"], w["energy"]))
    c = PC.CpuPipe(o)
    c.timestep()
    t0 = time.perf_counter()
    for _ in range(nsample):
        c.timestep()
    dt = time.perf_counter() - t0
    return {"value": nsample / dt, "unit": "timesteps/s", "cores": threads, "kind": "port",
            "sample": f"{nsample} steps of the C++/OpenMP restatement of the reference step on {threads} host "
                      f"threads (after matrices, seed and 1 warm-up step; no spin-up)"}


def read_traffic(kernel: str, workload: str):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    p = ROOT / "profiles" / "traffic.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 3 and parts[0] == workload and parts[1] == kernel:
            try:
                return float(parts[2])
            except ValueError:
                return None
    return None


# algorithmic bytes of one launch of each kernel category, in units of the
# coll field size S: the coll fields it must read and write once (factors,
# twiddles and transform scratch are not algorithmic).  In the fused step the
# pressure solve ("ppe") reads its right-hand side and writes the pressure
# (2S); the three Helmholtz solves ("lusolve") read three right-hand sides and
# write three solutions (6S).
PER_LAUNCH_S = {"lusolve": 6, "ppe": 2, "stencil": 2, "ew": 2, "infl": 4, "zinv": 3, "thinv": 3, "thfwd": 3,
                "zfwd": 3, "step": 10, "factor": 0}


def config_of(args, w=None):
    if args.workload == "batched":
        cfgs = batched_configs(args.pipes)
        return {"workload": f"batched: {args.pipes} uneven pipes (N in 32/48/64, K in 16/32/64, M in 12/24/32, "
                            f"Re 1800-3000, alpha 0.8-1.6, dt=0.01) in mixed precision, one CUDA graph per "
                            f"batch step, corrector to convergence per pipe",
                "pipes_per_gpu": args.pipes, "precision": "mixed (FP32 transforms, FP64 solves)",
                "sum_H": sum(harmonics_count(d) for d in cfgs), "parallelism": f"replicas x{args.gpus}",
                "l2": "working set of 64 pipes (~1-2 GB) larger than the 126 MB L2; no flush"}
    return {"workload": f"{args.workload}: plain FP64 drop-in, N={w['N']} K={w['K']} M={w['M']} Mp={w['Mp']} "
                        f"Re={w['Re']} alpha={w['alpha']} dt={w['dt']}, seeded perturbation E={w['energy']} E_lam, "
                        f"spin-up {w['spinup']} steps",
            "N": w["N"], "K": w["K"], "M": w["M"], "Mp": w["Mp"], "H": harmonics_count(w), "Re": w["Re"],
            "alpha": w["alpha"], "dt": w["dt"], "pipes_per_gpu": 1, "parallelism": f"replicas x{args.gpus}",
            "l2": "working set (~0.7 GB) larger than the 126 MB L2; no flush"}


def run_reference(args, rank):
    if rank != 0:
        return
    # batched: one step of every pipe of the mix (--ref-steps pipes, all 64 by
    # default); single pipe: that many steps, at most --steps
    nsample = max(1, args.ref_steps if args.workload == "batched" else min(args.steps, args.ref_steps))
    base = cpu_baseline(args.workload, nsample)
    w = SINGLE.get(args.workload)
    line = {
        "impl": "reference", "metric": METRIC, "value": base["value"], "unit": "timesteps/s",
        "n_gpus": args.gpus, "steps": nsample, "warmup": 1, "ms_per_step": 1e3 / base["value"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config_of(args, w), "cpu_baseline": base,
        "e2e": {"value": base["value"], "unit": "timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def rank_seeds(rank: int, pipes: int):
    """Seeds of one rank's pipes: every replica integrates different states."""
    return [1000 + rank * pipes + i for i in range(pipes)]


def max_over_ranks(dist, torch, values, device):
    """Element-wise max of per-rank timings (the slowest rank sets the time)."""
    if dist is None:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def dev_timer(torch, stream):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    return e0, e1


def plain_sequential(P, torch, cfgs, seeds, steps=3):
    """The plain FP64 drop-in on the same pipes, one pipe at a time."""
    total_ms, total_steps = 0.0, 0
    stream = torch.cuda.Stream()
    for d, sd in zip(cfgs, seeds):
        p = P.Pipe(P.PipeConfig(**d))
        p.lib.pf_ctx_set_stream(p.ctx, stream.cuda_stream)
        p.vel_matrices()
        P.seeded_state(p, sd, 1e-3)
        for _ in range(3):  # eager step + both graph parities captured
            p.timestep()
        e0, e1 = dev_timer(torch, stream)
        e0.record(stream)
        for _ in range(steps):
            p.timestep()
        e1.record(stream)
        stream.synchronize()
        total_ms += e0.elapsed_time(e1)
        total_steps += steps
        p.close()
    return total_steps / (total_ms / 1e3), total_ms / total_steps


def mixed_error(P, d, seed, nsteps=1000, energy=1e-3):
    """State rel-L2, kinetic-energy and friction errors of the mixed path
    against the FP64 device path (itself held to the oracle at 1e-12 after one
    step and 1e-9 after 100 by the parity tests) on the config-1 pipe N=40,
    K=24, M=16, after 1, 100 and 1000 steps (those not beyond nsteps)."""
    g64 = P.Pipe(P.PipeConfig(**d))
    gm = P.Pipe(P.PipeConfig(**d, precision=P.PF_PREC_MIXED))
    for g in (g64, gm):
        g.vel_matrices()
        P.seeded_state(g, seed, energy)
    marks = [s for s in (1, 100, 1000) if s <= nsteps] or [nsteps]
    rows = []
    done = 0
    for mark in marks:
        for g in (g64, gm):
            for _ in range(mark - done):
                g.timestep()
        done = mark
        num = den = 0.0
        for (ar, ai), (br, bi) in zip(gm.get_state(), g64.get_state()):
            num += float(np.sum((ar - br) ** 2 + (ai - bi) ** 2))
            den += float(np.sum(br ** 2 + bi ** 2))
        e64, em = g64.energy(), gm.energy()
        f64, fm = g64.friction()[2], gm.friction()[2]
        rows.append({"steps": mark, "state_rel_l2": math.sqrt(num / den), "energy_rel": abs(em - e64) / e64,
                     "friction_rel": abs(fm - f64) / f64})
    g64.close()
    gm.close()
    out = {"pipe": d, **rows[-1], "at_steps": rows}
    return out


def run_single(args, torch, P, dist, world, rank, local):
    """One large FP64 pipe per rank (cfg2 / cfg1)."""
    w = dict(SINGLE[args.workload])
    if args.spinup is not None:
        w["spinup"] = args.spinup
    pipe = P.Pipe(P.PipeConfig(**{k: w[k] for k in PHYS}), device=local)
    stream = torch.cuda.Stream()
    pipe.lib.pf_ctx_set_stream(pipe.ctx, stream.cuda_stream)
    pipe.vel_matrices()
    P.seeded_state(pipe, w["seed"] + rank, w["energy"])
    with torch.cuda.stream(stream):
        for _ in range(w["spinup"]):
            pipe.timestep()
        pipe.prof_enable(True)
        for _ in range(args.warmup):
            pipe.timestep()
        prof = pipe.prof_read()
        dom = max(prof, key=lambda k: prof[k][0])
        # time only the dominant category from here on; the step graphs are
        # re-captured (both pointer parities) with its event nodes, untimed
        pipe.prof_enable([dom])
        for _ in range(2):
            pipe.timestep()
        pipe.prof_enable([dom])
        stream.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        n0 = pipe.launches()
        ev0, ev1 = dev_timer(torch, stream)
        ncorr = 0
        with ClockSampler(local) as clk:
            ev0.record(stream)
            for _ in range(args.steps):
                ncorr += pipe.timestep()
            ev1.record(stream)
            stream.synchronize()
        launches = pipe.launches() - n0
        ms = ev0.elapsed_time(ev1)
        dom_ms, dom_n = pipe.prof_read()[dom]
        pipe.prof_enable(False)
        # end to end through the C ABI with pinned host buffers
        N, H = pipe.N, pipe.H
        host = [torch.empty((H, N), dtype=torch.float64, pin_memory=True) for _ in range(6)]
        ptrs = [P.api.C.cast(t.data_ptr(), P._lib.DP) for t in host]
        P.api._check(pipe.lib.pf_vel_get_state(pipe.ctx, *ptrs))
        ne = max(1, min(args.e2e_steps, args.steps))
        e0, e1 = dev_timer(torch, stream)
        e0.record(stream)
        for _ in range(ne):
            P.api._check(pipe.lib.pf_vel_set_state(pipe.ctx, *ptrs))
            pipe.timestep()
            P.api._check(pipe.lib.pf_vel_get_state(pipe.ctx, *ptrs))
        e1.record(stream)
        stream.synchronize()
        e2e_ms = e0.elapsed_time(e1)
    pipe.close()
    S = coll_bytes(w)
    nc = ncorr / args.steps
    per_launch = PER_LAUNCH_S[dom] * S
    res = dict(ms=ms, e2e_ms=e2e_ms, ne=ne, count=1, launches=launches, clk=clk.summary(),
               extra={"corrector_iterations_per_step": nc,
                      "algorithmic_bytes_per_step": S * (15 + 21 * nc),
                      "step_bandwidth_gbs": S * (15 + 21 * nc) / (ms / args.steps / 1e3) / 1e9},
               dom=dom, dom_ms=dom_ms, dom_n=dom_n, per_launch=per_launch,
               h2d=6 * N * H * 8, d2h=6 * N * H * 8, dtype="f64", config=config_of(args, w))
    return res


def run_batched(args, torch, P, dist, world, rank, local):
    """One batch of uneven mixed-precision pipes per rank."""
    cfgs = batched_configs(args.pipes)
    seeds = rank_seeds(rank, args.pipes)
    batch = P.Batch([P.PipeConfig(**d, precision=P.PF_PREC_MIXED) for d in cfgs], device=local)
    batch.matrices()
    for p, sd in zip(batch.pipes, seeds):
        P.seeded_state(p, sd, 1e-3)
    h = P.api.C.c_void_p()
    P.api._check(batch.lib.pf_batch_stream(batch.h, P.api.C.byref(h)))
    master = torch.cuda.ExternalStream(h.value)
    tuned = None
    if args.ld_solver != "auto" or args.nl_fused:  # one choice for every pipe (profiling)
        ld = {"auto": P.PF_LD_AUTO, "streamed": P.PF_LD_STREAMED, "rebuilt": P.PF_LD_REBUILT,
              "paired": P.PF_LD_PAIRED, "warpring": P.PF_LD_WARPRING}[args.ld_solver]
        for p in batch.pipes:
            p.set_tuning(ld_solver=ld, nl_fused=1 if args.nl_fused else 0)
    if args.worklist != "auto":  # the form of the transform stages, for every run below
        batch.set_worklist(args.worklist == "on")
    if args.tune:
        # the project's autotuner picks the launch choices per pipe shape by
        # timing whole batch steps (untimed here; states restored afterwards)
        t0 = time.perf_counter()
        tuner = P.Tuner(use_cache=False, steps=4, reps=2)
        choice = tuner.tune_batch(batch)
        if args.worklist != "auto":
            batch.set_worklist(args.worklist == "on")
        tuned = {"seconds": time.perf_counter() - t0, "timings": len(tuner.log), "choice": choice}
    batch.step(args.spinup if args.spinup is not None else 20)
    batch.prof_enable(True)
    batch.step(args.warmup)
    # the dominant kernel among the stage-batched launches, whose every span
    # covers all pipes (a pipe's own extra corrector pass is left out): the
    # categories timed as one kernel's launches (the transform categories
    # each span several launches, one per transform length, run side by
    # side; they are reported together as the transform chain below)
    staged0 = batch.staged()
    prof = batch.prof_read(staged_only=staged0)
    single = ("lusolve", "ppe", "infl")
    dom = max(single, key=lambda k: prof[k][0])
    nl_evals = max(prof["thfwd"][1], 1)
    chain_ms = (prof["zinv"][0] + prof["thfwd"][0] + prof["zfwd"][0]) / nl_evals
    chain_share = (prof["zinv"][0] + prof["thfwd"][0] + prof["zfwd"][0]) / max(sum(v[0] for v in prof.values()), 1e-30)
    batch.prof_enable([dom])
    batch.step(2)  # re-capture both parities with the dominant category's event nodes
    batch.prof_enable([dom])
    batch.sync()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    n0 = batch.launches()
    staged = batch.staged()
    ev0, ev1 = dev_timer(torch, master)
    with ClockSampler(local) as clk:
        ev0.record(master)
        passes = batch.step(args.steps)
        ev1.record(master)
        master.synchronize()
    launches = batch.launches() - n0
    ms = ev0.elapsed_time(ev1)
    dom_ms, dom_n = batch.prof_read(staged_only=staged)[dom]
    batch.prof_enable(False)
    # end to end through the C ABI: every step uploads a block with every
    # pipe's state from pinned host memory, steps, and downloads the stepped
    # states; the upload of the next block and the download of the last one
    # run on copy streams while the step in between computes
    nd = batch.io_bytes() // 8
    hin = [torch.empty(nd, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    hout = [torch.empty(nd, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    off = 0
    for p in batch.pipes:  # the block from the pipes' current states
        n = p.N * p.H
        ptrs = [P.api.C.cast(hin[0].data_ptr() + (off + k * n) * 8, P._lib.DP) for k in range(6)]
        P.api._check(p.lib.pf_vel_get_state(p.ctx, *ptrs))
        off += 6 * n
    hin[1].copy_(hin[0])
    batch.put_states(0, hin[0])  # first use: allocates the device staging
    batch.step_io(0, 1)
    batch.get_states(0, hout[0])
    batch.io_sync()
    ne = max(1, min(args.e2e_steps, args.steps))
    e0, e1 = dev_timer(torch, master)
    e0.record(master)
    batch.put_states(0, hin[0])
    for s in range(ne):
        if s + 1 < ne:
            batch.put_states((s + 1) % 2, hin[(s + 1) % 2])
        batch.step_io(s % 2, 1)
        batch.get_states(s % 2, hout[s % 2])
    batch.io_sync()
    e1.record(master)
    master.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    # the same copies with no step between them (both directions at once, on
    # the batch's copy streams): the PCIe rate the end-to-end figure meets
    t0 = time.perf_counter()
    for s in range(ne):
        batch.put_states(s % 2, hin[s % 2])
        batch.get_states(s % 2, hout[s % 2])
    batch.io_sync()
    copies_ms = (time.perf_counter() - t0) * 1e3 / ne
    worklist = batch.worklist
    batch.close()
    S = [coll_bytes(d) for d in cfgs]
    nc = passes / (args.steps * args.pipes)
    step_bytes = sum(s * (15 + 21 * nc) for s in S)
    # dominant category: algorithmic bytes per launch; a stage-batched launch
    # covers every pipe, a per-pipe launch one pipe (averaged over the pipes)
    per_launch = PER_LAUNCH_S[dom] * (sum(S) if staged else sum(S) / len(S))
    io = sum(6 * d["N"] * harmonics_count(d) * 8 for d in cfgs)
    chain_bytes = 6 * sum(S)   # u in, N out
    chain_flops = sum(transform_flops(d) for d in cfgs)
    extra = {"corrector_iterations_per_step": nc, "algorithmic_bytes_per_batch_step": step_bytes,
             "stage_batched": staged, "worklist_stages": worklist, "autotune": tuned,
             "transform_roofline": {
                 "scope": "one evaluation of the nonlinear terms of every pipe: FP64 mean-mode pass (and curl), "
                          "z inverse, theta pass with u x curl(u), z forward (all transform launches)",
                 "avg_evaluation_us": chain_ms * 1e3, "share_of_step_kernels": chain_share,
                 "algorithmic_bytes": chain_bytes, "achieved_gbs": chain_bytes / (chain_ms / 1e3) / 1e9,
                 "frac_of_measured_hbm": chain_bytes / (chain_ms / 1e3) / 1e9 / peaks()[0],
                 "fft_flops": chain_flops, "achieved_fp32_tflops": chain_flops / (chain_ms / 1e3) / 1e12,
                 "fp32_nominal_tflops": 74.4,
                 "note": "flops by the 5 L log2 L count per complex FFT of length L; the FP32 peak is the nominal "
                         "148 SMs x 128 lanes x 2 x 1.965 GHz (not measured)"},
             "batch_step_ms": ms / args.steps,
             # per-category stage spans of the warm-up steps (every category's event nodes on)
             "stage_spans_us": {k: 1e3 * v[0] / v[1] for k, v in prof.items() if v[1] > 0},
             "step_roofline": {"bound": "hbm", "scope": "whole batch step (all stages, all pipes)",
                               "achieved": step_bytes / (ms / args.steps / 1e3) / 1e9, "unit": "GB/s"}}
    if rank == 0:
        plain, plain_ms = plain_sequential(P, torch, cfgs[:args.plain_pipes], seeds[:args.plain_pipes])
        extra["plain"] = {"value": plain, "unit": "timesteps/s", "ms_per_pipe_step": plain_ms,
                          "what": f"the same pipes (first {args.plain_pipes}) in FP64, one pipe at a time "
                                  f"through pf_timestep"}
        extra["batched_over_plain"] = (args.pipes * args.steps / (ms / 1e3)) / plain
        extra["mixed_vs_fp64"] = mixed_error(P, {k: SINGLE["cfg1"][k] for k in PHYS}, SINGLE["cfg1"]["seed"],
                                             args.err_steps, SINGLE["cfg1"]["energy"])
        extra["util_plugins"] = util_plugin_timing(P, torch, local)
        if args.with_serve:
            extra["serve"] = run_serve(args, P, local, plain)
        if args.with_cfg2 and not args.no_cpu_baseline:
            # config-1: the plain FP64 drop-in on one pipe against the CPU
            # restatement of the reference step on every host thread
            sub = argparse.Namespace(**vars(args))
            sub.workload, sub.spinup, sub.steps = "cfg1", 0, 200
            r1 = run_single(sub, torch, P, None, 1, 0, local)
            gpu1 = sub.steps / (r1["ms"] / 1e3)
            cpu1 = cpu_baseline("cfg1", 10)
            extra["cfg1"] = {"gpu_plain": gpu1, "cpu": cpu1["value"], "cpu_cores": cpu1["cores"],
                             "unit": "timesteps/s", "gpu_over_cpu": gpu1 / cpu1["value"],
                             "what": "N=40 K=24 M=16 FP64, one pipe: pf_timestep (CUDA graph) vs the "
                                     "C++/OpenMP CPU restatement"}
        if args.with_cfg2:
            sub = argparse.Namespace(**vars(args))
            sub.workload, sub.spinup, sub.steps = "cfg2", args.cfg2_spinup, args.cfg2_steps
            r = run_single(sub, torch, P, None, 1, 0, local)
            extra["plain_cfg2"] = {"value": sub.steps / (r["ms"] / 1e3), "unit": "timesteps/s",
                                   "ms_per_step": r["ms"] / sub.steps, "workload": r["config"]["workload"],
                                   "dominant_kernel": r["dom"],
                                   "dominant_avg_launch_us": r["dom_ms"] * 1e3 / max(r["dom_n"], 1),
                                   **r["extra"]}
    return dict(ms=ms, e2e_ms=e2e_ms, ne=ne, count=args.pipes, launches=launches, clk=clk.summary(),
                e2e_path="pf_batch_put_states / pf_batch_step_io / pf_batch_get_states: one pinned state block "
                         "in and one out per step, copies on their own streams overlapping the step between",
                extra=extra, dom=dom, dom_ms=dom_ms, dom_n=dom_n, per_launch=per_launch, h2d=io, d2h=io,
                copies_ms=copies_ms,
                dtype="mixed: f32 transforms, f64 solves", config=config_of(args))


KRYLOV = dict(N=48, K=32, M=24, Mp=1, Re=2000.0, alpha=1.25)


def util_plugin_timing(P, torch, local, steps=100):
    """ms per main-loop step of the config-1 pipe (FP64) with each built-in
    plug-in of main.f90's var_null hook: Coriolis and Carreau-Yasuda run
    inside the step graphs, LES eagerly (its update_nu_r reads max nu_t back
    to the host)."""
    from pipeflow import _lib as L
    kinds = {"none": None, "coriolis": (L.PF_UTIL_CORIOLIS, (0.5, 0.3)),
             "carreau_yasuda": (L.PF_UTIL_CARREAU_YASUDA, (1000.0, 0.01, 0.05, 0.0035, 3.3, 0.36, 2.0)),
             "les_smagorinsky": (L.PF_UTIL_LES, (1.0, 0.025, 1.0, 25.0))}
    out = {}
    stream = torch.cuda.Stream()
    for name, k in kinds.items():
        p = P.Pipe(P.PipeConfig(**{q: SINGLE["cfg1"][q] for q in PHYS}), device=local)
        p.lib.pf_ctx_set_stream(p.ctx, stream.cuda_stream)
        p.vel_matrices()
        P.seeded_state(p, 1, 1e-3)
        if k:
            p.util_set(*k)
        for _ in range(3):
            p.timestep()
        e0, e1 = dev_timer(torch, stream)
        e0.record(stream)
        for _ in range(steps):
            p.timestep()
        e1.record(stream)
        stream.synchronize()
        out[name] = e0.elapsed_time(e1) / steps
        p.close()
    return {"ms_per_step": out, "what": "N=40 K=24 M=16 FP64 pf_timestep, 100 steps"}


def run_serve(args, P, local, plain_value):
    """Config-4 serving: Poisson arrivals of time-T-map requests (T uniform in
    [1, 20], dt = 0.01), 30% GMRES Krylov-vector evaluations at N=48 K=32 M=24
    (FP64, base state + 1e-7 seeded perturbation), the rest on the batched
    mix's sizes in mixed precision; 150 GB HBM admission budget; continuous
    batching.  The arrival window is bounded so the run takes seconds."""
    from pipeflow import serve as S
    reqs = S.make_stream(args.serve_rate, args.serve_window, 4, batched_configs(64), KRYLOV, device=local)
    srv = P.Server(hbm_budget=150 * 10**9, device=local)
    n0 = srv.launches()
    makespan = S.run_stream(srv, reqs)
    launches = srv.launches() - n0
    srv.close()
    out = S.latency_summary(reqs)
    if args.sustained:
        out["sustained"] = sustained_rate(args, P, S, local)
    out.update({"rate_req_per_s": args.serve_rate, "arrival_window_s": args.serve_window,
                "hbm_budget_bytes": 150 * 10**9, "makespan_s": makespan,
                "served_timesteps_per_s": out["pipe_steps"] / makespan,
                "served_over_plain": out["pipe_steps"] / makespan / plain_value,
                "gpu_launches": launches,
                "note": "latency from arrival to the result on the host; the offered load "
                        f"({args.serve_rate:.0f} req/s x ~1050 steps each) exceeds one GPU's throughput, so "
                        "every arrival joins a growing batch and latency grows with the number in flight"})
    return out


def sustained_rate(args, P, S, local):
    """The highest Poisson arrival rate (of those tried) that one GPU serves
    within a latency bound: for each rate about `sustained_requests`
    requests of the same mix arrive at that rate, and the rate is sustained
    while the median latency stays within twice the median at the lowest
    rate tried (the unloaded latency).  With continuous batching every
    arrival is admitted at once while memory lasts, so an overloaded server
    shows as every request slowing down together, not as a queue.  Returns
    the rate found and every trial's p50/p99 and throughput."""
    trials = []
    best = None
    base = None
    for rate in args.sustained_rates:
        window = args.sustained_requests / rate
        reqs = S.make_stream(rate, window, 40 + int(rate), batched_configs(64), KRYLOV, device=local)
        if len(reqs) < 4:
            continue
        srv = P.Server(hbm_budget=150 * 10**9, device=local)
        makespan = S.run_stream(srv, reqs)
        srv.close()
        lat = S.latency_summary(reqs)
        if base is None:
            base = lat["p50_s"]
        row = {"rate_req_per_s": rate, "arrival_window_s": window, "requests": lat["requests"],
               "p50_s": lat["p50_s"], "p99_s": lat["p99_s"],
               "offered_timesteps_per_s": lat["pipe_steps"] / window,
               "served_timesteps_per_s": lat["pipe_steps"] / makespan,
               "failed_requests": lat["failed_requests"]}
        row["within_bound"] = bool(lat["p50_s"] <= 2.0 * base)
        trials.append(row)
        if row["within_bound"]:
            best = rate
        else:
            break  # latency has left the bound: higher rates will not meet it either
    return {"sustained_rate_req_per_s": best,
            "criterion": "median latency within 2x the median at the lowest rate tried",
            "unloaded_p50_s": base, "requests_per_rate": args.sustained_requests, "trials": trials}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched", choices=["batched", "cfg2", "cfg1"])
    ap.add_argument("--pipes", type=int, default=64)
    ap.add_argument("--spinup", type=int, default=None)
    ap.add_argument("--ref-steps", type=int, default=64)
    ap.add_argument("--e2e-steps", type=int, default=100)
    ap.add_argument("--plain-pipes", type=int, default=64)
    ap.add_argument("--err-steps", type=int, default=1000)
    ap.add_argument("--cfg2-spinup", type=int, default=500)
    ap.add_argument("--cfg2-steps", type=int, default=1000)
    ap.add_argument("--no-cfg2", dest="with_cfg2", action="store_false")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-window", type=float, default=0.5)
    ap.add_argument("--no-serve", dest="with_serve", action="store_false")
    ap.add_argument("--no-sustained", dest="sustained", action="store_false")
    ap.add_argument("--sustained-rates", type=float, nargs="+", default=[4.0, 8.0, 12.0, 16.0, 24.0, 32.0])
    ap.add_argument("--sustained-requests", type=int, default=32)
    ap.add_argument("--no-tune", dest="tune", action="store_false")
    ap.add_argument("--ld-solver", default="auto", choices=["auto", "streamed", "rebuilt", "paired", "warpring"])
    ap.add_argument("--worklist", default="auto", choices=["auto", "on", "off"],
                    help="transform stages as one work-list launch each (auto: the autotuner decides)")
    ap.add_argument("--nl-fused", action="store_true",
                    help="transforms of a radial point in one block for every pipe where built")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    dist = None
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    import pipeflow as P

    run = run_batched if args.workload == "batched" else run_single
    r = run(args, torch, P, dist, world, rank, local)
    ms, e2e_ms = max_over_ranks(dist, torch, [r["ms"], r["e2e_ms"]], "cuda")
    value = world * r["count"] * args.steps / (ms / 1e3)
    e2e_value = world * r["count"] * r["ne"] / (e2e_ms / 1e3)

    if rank == 0:
        peak, src = peaks()
        avg_launch_s = (r["dom_ms"] / 1e3) / max(r["dom_n"], 1)
        achieved = r["per_launch"] / avg_launch_s / 1e9 if avg_launch_s > 0 else None
        line = {
            "metric": METRIC, "value": value, "unit": "timesteps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": r["dtype"], "data": "synthetic",
            "config": r["config"],
            "roofline": {"bound": "hbm", "kernel": r["dom"], "achieved": achieved, "peak": peak,
                         "peak_source": src, "unit": "GB/s", "frac": achieved / peak if achieved else None,
                         "algorithmic_bytes_per_launch": r["per_launch"],
                         "avg_launch_us": avg_launch_s * 1e6, "launches": r["dom_n"],
                         "traffic": read_traffic(r["dom"], args.workload)},
            "gpu_launches": r["launches"],
            "e2e": {"value": e2e_value, "unit": "timesteps/s", "steps": r["ne"],
                    "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"],
                    "path": r.get("e2e_path", "")},
            "clocks": r["clk"],
        }
        if r.get("copies_ms"):
            line["e2e"]["copies_only_ms_per_step"] = r["copies_ms"]
            line["e2e"]["copies_only_gbs_each_way"] = r["h2d"] / (r["copies_ms"] / 1e3) / 1e9
        if args.workload == "batched":
            if r["extra"].get("stage_batched"):
                line["roofline"]["note"] = (
                    "one launch covers every pipe; a category's launches of different transform lengths "
                    "run concurrently and are timed as one span; algorithmic bytes exclude the LU factors "
                    "and influence vectors that the solves stream (traffic includes them)")
            else:
                line["roofline"]["note"] = ("kernel spans of concurrent pipes overlap in time, so the per-launch "
                                            "duration includes GPU sharing and frac is a lower bound")
        line.update(r["extra"])
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args.workload, max(1, args.ref_steps))
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
