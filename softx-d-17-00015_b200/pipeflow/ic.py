"""Seeded initial states (the reference's ic.f90 is an empty template).

State = Hagen-Poiseuille flow (stored as zero: vel_uz holds the deviation
from U = 1 - r^2, velocity.f90:53) plus a solenoidal perturbation u' = curl A.
A has one complex Gaussian coefficient per (component, mode) from
numpy.random.default_rng(seed), drawn as a single (3, 2, H) standard-normal
block (component, re/im, mode), scaled by exp(-(k^2+m^2)/16), with radial
envelopes that are regular on the axis and vanish with their slope at the
wall: r^(|m Mp|+1)(1-r^2)^2 for A_r, A_theta and r^(|m Mp|+2)(1-r^2)^2 for
A_z.  The curl is taken on the device (var_coll_curl), the k=m=0 symmetry is
imposed (var_imposesym(0)) and the state is scaled to a perturbation energy
of ``energy_frac`` * E_lam, E_lam = pi^2/(3 alpha) (io.f90:548).
"""
from __future__ import annotations

import math

import numpy as np

PI = 3.1415926535897931


def harmonics(K: int, M: int):
    """Mode order of the serial _loop_km macro (parallel.h:47-57)."""
    ks, ms = [], []
    for m in range(M):
        for k in range(-(K - 1), K):
            if m == 0 and k < 0:
                continue
            ks.append(k)
            ms.append(m)
    return np.array(ks), np.array(ms)


def vector_potential_host(K: int, M: int, Mp: int, r: np.ndarray, seed: int):
    """Host arrays [(re, im)] * 3 of shape (N, H) of the seeded potential on
    the radial mesh r."""
    H = (2 * K - 1) * M - (K - 1)
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((3, 2, H))
    kk, mm = harmonics(K, M)
    k = kk.astype(float)
    m = mm.astype(float)
    amp = np.exp(-(k * k + m * m) / 16.0)
    r = np.asarray(r, dtype=float)[:, None]
    am = np.abs(mm * Mp)[None, :]
    prof_rt = r ** (am + 1) * (1.0 - r * r) ** 2
    prof_z = r ** (am + 2) * (1.0 - r * r) ** 2
    profs = (prof_rt, prof_rt, prof_z)
    return [(g[c, 0][None, :] * amp[None, :] * profs[c], g[c, 1][None, :] * amp[None, :] * profs[c])
            for c in range(3)]


def seeded_state(pipe, seed: int, energy_frac: float) -> None:
    """Load the seeded perturbation into vel_ur, vel_ut, vel_uz of ``pipe``."""
    r = pipe.mes_D()["r"]
    A = [pipe.coll(re, im) for re, im in vector_potential_host(pipe.K, pipe.M, pipe.Mp, r, seed)]
    u = [pipe.vel_ur, pipe.vel_ut, pipe.vel_uz]
    pipe.var_coll_curl(A[0], A[1], A[2], u[0], u[1], u[2])
    pipe.var_imposesym(0, u[0], u[1], u[2])
    E = sum(pipe.var_coll_norm(f)[0] for f in u)
    s = math.sqrt(energy_frac * (PI * PI / (3.0 * pipe.cfg.alpha)) / E)
    for f in u:
        pipe.var_coll_dmult(s, f)
