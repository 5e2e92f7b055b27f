"""Request streams for the continuous-batching server (``Server``).

A request is a time-T map: advance a state by round(T/dt) timesteps.  Two
kinds are built here:

* plain time-T maps on seeded states of the batched mix's sizes;
* Krylov-vector evaluations as GMRES makes them in the Newton-hookstep
  search: a base state plus a small seeded perturbation (newton.f90:439-445,
  where the perturbation is scaled by epsJ).

``run_stream`` replays a stream against wall-clock arrival times: requests
are submitted when their arrival time has passed, the server steps while any
request is queued or running, and each request's latency runs from its
arrival to the moment its result is back on the host.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from .api import Pipe, PipeConfig, PipeflowError, Server
from .ic import seeded_state


@dataclass
class Request:
    arrival: float                 # seconds after the stream starts
    cfg: PipeConfig
    nsteps: int
    state: list                    # (ur, ut, uz) as Pipe.set_state takes it
    kind: str = "tmap"
    rid: int | None = None
    done_at: float | None = None
    result: list | None = field(default=None, repr=False)
    error: str | None = None       # a failed request's message (the server reports it alone)

    @property
    def latency(self) -> float | None:
        return None if self.done_at is None else self.done_at - self.arrival


class StateMaker:
    """Seeded states on the device, one helper pipe per shape."""

    def __init__(self, device: int = -1):
        self.device = device
        self.pipes = {}

    def __call__(self, cfg: PipeConfig, seed: int, energy_frac: float):
        key = (cfg.N, cfg.K, cfg.M, cfg.Mp)
        want = PipeConfig(N=cfg.N, K=cfg.K, M=cfg.M, Mp=cfg.Mp, alpha=cfg.alpha)
        p = self.pipes.get(key)
        if p is None:
            p = self.pipes[key] = Pipe(want, device=self.device)
        elif p.cfg.alpha != cfg.alpha:  # the energy norm depends on alpha
            p.reconfigure(want)
        seeded_state(p, seed, energy_frac)
        return p.get_state()

    def close(self):
        for p in self.pipes.values():
            p.close()
        self.pipes.clear()


def make_stream(rate: float, window: float, seed: int, mix_cfgs, krylov_cfg: dict, krylov_frac: float = 0.3,
                t_range=(1.0, 20.0), dt: float = 0.01, mixed: bool = True, eps: float = 1e-3,
                eps_krylov: float = 1e-7, device: int = -1):
    """Poisson arrivals at `rate` per second for `window` seconds.  A fraction
    `krylov_frac` are Krylov-vector evaluations at `krylov_cfg` (FP64); the
    rest are time-T maps on sizes drawn from `mix_cfgs` (mixed precision when
    `mixed`).  T is uniform in `t_range`."""
    rng = np.random.default_rng(seed)
    maker = StateMaker(device)
    reqs = []
    t = rng.exponential(1.0 / rate)
    k = 0
    try:
        while t < window:
            T = rng.uniform(*t_range)
            nsteps = max(1, int(round(T / dt)))
            if rng.uniform() < krylov_frac:
                cfg = PipeConfig(**dict(krylov_cfg, dt=dt))
                base = maker(cfg, 5000, eps)
                pert = maker(cfg, 6000 + k, eps)
                state = [(b[0] + eps_krylov * q[0], b[1] + eps_krylov * q[1]) for b, q in zip(base, pert)]
                kind = "krylov"
            else:
                d = mix_cfgs[rng.integers(len(mix_cfgs))]
                cfg = PipeConfig(**dict(d, dt=dt), precision=1 if mixed else 0)
                state = maker(cfg, 7000 + k, eps)
                kind = "tmap"
            reqs.append(Request(arrival=t, cfg=cfg, nsteps=nsteps, state=state, kind=kind))
            k += 1
            t += rng.exponential(1.0 / rate)
    finally:
        maker.close()
    return reqs


def run_stream(server: Server, reqs, keep_results: bool = False):
    """Replay the stream in wall-clock time; returns the stream's makespan in
    seconds (first arrival to last result)."""
    pending = sorted(reqs, key=lambda r: r.arrival)
    by_id = {}
    i = 0
    t0 = time.perf_counter()
    done = 0
    while done < len(pending):
        now = time.perf_counter() - t0
        while i < len(pending) and pending[i].arrival <= now:
            r = pending[i]
            r.rid = server.submit(r.cfg, r.nsteps, r.state)
            by_id[r.rid] = r
            i += 1
        st = server.stats()
        if st["queued"] == 0 and st["active"] == 0:
            if i < len(pending):
                time.sleep(max(0.0, pending[i].arrival - (time.perf_counter() - t0)))
            continue
        server.step()
        fin = server.finished()
        if fin:
            now = time.perf_counter() - t0
            for rid in fin:
                r = by_id[rid]
                try:
                    res = server.result(rid)
                except PipeflowError as e:  # this request failed alone (e.g. its state went non-finite)
                    res, r.error = None, str(e)
                r.done_at = now
                if keep_results:
                    r.result = res
                done += 1
    return time.perf_counter() - t0 - (pending[0].arrival if pending else 0.0)


def latency_summary(reqs) -> dict:
    lat = np.array([r.latency for r in reqs if r.latency is not None])
    steps = sum(r.nsteps for r in reqs)
    return {"requests": len(reqs), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max()), "pipe_steps": int(steps),
            "krylov_requests": sum(r.kind == "krylov" for r in reqs),
            "failed_requests": sum(r.error is not None for r in reqs)}
