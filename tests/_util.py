"""Helpers shared by the test modules: paired oracle / device pipes and field
conversions."""
from __future__ import annotations

import math

import numpy as np

import pipeflow_oracle as O

# small cases the oracle finishes in well under a second per step
SMALL = [
    dict(N=16, K=4, M=4, Mp=1, Re=2000.0, alpha=1.25, dt=0.01),
    dict(N=24, K=6, M=5, Mp=2, Re=3000.0, alpha=0.8, dt=0.005),
    dict(N=20, K=5, M=6, Mp=1, Re=1800.0, alpha=1.6, dt=0.01, const_flux=False),
]
# the reference's CPU-runnable case: N=40, K=24, M=16, Re=2000, alpha=1.25, dt=0.01
CFG1 = dict(N=40, K=24, M=16, Mp=1, Re=2000.0, alpha=1.25, dt=0.01)


def oracle_pipe(cfgd):
    return O.Pipe(O.PipeConfig(**cfgd))


def device_pipe(cfgd, **extra):
    import pipeflow as P
    d = dict(cfgd)
    d.update(extra)
    return P.Pipe(P.PipeConfig(**d))


def rand_coll(N, H, rng, scale=1.0):
    return O.Coll(scale * rng.standard_normal((N, H)), scale * rng.standard_normal((N, H)))


def to_dev(pipe, c: O.Coll):
    return pipe.coll(c.re, c.im)


def from_dev(c) -> O.Coll:
    re, im = c.download()
    return O.Coll(re, im)


def rel(a, b) -> float:
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def rel_coll(a: O.Coll, b: O.Coll) -> float:
    num = np.sum((a.re - b.re) ** 2 + (a.im - b.im) ** 2)
    den = np.sum(b.re ** 2 + b.im ** 2)
    return float(math.sqrt(num / den)) if den > 0 else float(math.sqrt(num))


def state_from_dev(pipe):
    return [O.Coll(re, im) for re, im in pipe.get_state()]


def state_to_dev(pipe, st):
    pipe.set_state(*[(c.re, c.im) for c in st])
