"""State files of io.f90 (netCDF-3: state*.cdf.dat, state.cdf.in).

    Pipe.io_save_state(path)                      # io_save_state (io.f90:303-378)
    Pipe.io_load_state(path, time_from_file)      # io_load_state (io.f90:98-226)
    state_write(path, N, K, M, Mp, r, state, t=..., Re=..., alpha=..., dt=...)
    state_read(path, N, K, M, Mp, r) -> (state, scalars, changes)

The last two need no GPU.  A state is three (re, im) pairs of (N, H) float64
arrays indexed [n, nh] (ur, ut, uz), as Pipe.set_state takes them.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib as L
from .api import PipeflowError, _check, _dp

SCALARS = ("t", "Re", "alpha", "dt", "dtcor", "dtcfl")


def _harmonics(K: int, M: int) -> int:
    return (2 * K - 1) * M - (K - 1)


def state_write(path, N: int, K: int, M: int, Mp: int, r, state, t: float = 0.0, Re: float = 0.0,
                alpha: float = 0.0, dt: float = 0.0, dtcor: float = 0.0, dtcfl: float = 0.0) -> None:
    """Write a state file (pf_state_write)."""
    H = _harmonics(K, M)
    r = np.ascontiguousarray(r, dtype=np.float64)
    if r.shape != (N,):
        raise PipeflowError(L.PF_ERR_ARG, "state_write: r must have N points")
    arrs = []
    for re, im in state:
        for x in (re, im):
            x = np.asarray(x, dtype=np.float64)
            if x.shape != (N, H):
                raise PipeflowError(L.PF_ERR_ARG, f"state_write: fields must be (N, H) = ({N}, {H})")
            arrs.append(np.ascontiguousarray(x.T))
    sc = np.array([t, Re, alpha, dt, dtcor, dtcfl], dtype=np.float64)
    _check(L.load().pf_state_write(os.fsencode(path), N, K, M, Mp, _dp(r), *[_dp(a) for a in arrs], _dp(sc)))


def state_read(path, N: int, K: int, M: int, Mp: int, r):
    """Read a state file onto N radial points r and K, M harmonics
    (pf_state_read).  Returns (state, scalars, changes): scalars maps t, Re,
    alpha, dt, dtcor, dtcfl to values (NaN where absent); changes has bit 1
    if interpolated, 2 if K, 4 if M, 8 if Mp differed."""
    H = _harmonics(K, M)
    r = np.ascontiguousarray(r, dtype=np.float64)
    arrs = [np.empty((H, N)) for _ in range(6)]
    sc = np.empty(6)
    ch = C.c_int()
    _check(L.load().pf_state_read(os.fsencode(path), N, K, M, Mp, _dp(r), *[_dp(a) for a in arrs], _dp(sc),
                                  C.byref(ch)))
    a = [np.ascontiguousarray(x.T) for x in arrs]
    return [(a[0], a[1]), (a[2], a[3]), (a[4], a[5])], dict(zip(SCALARS, sc.tolist())), ch.value


def io_save_state(pipe, path) -> None:
    _check(pipe.lib.pf_io_save_state(pipe.ctx, os.fsencode(path)))


def io_load_state(pipe, path, time_from_file: bool = False) -> int:
    ch = C.c_int()
    _check(pipe.lib.pf_io_load_state(pipe.ctx, os.fsencode(path), L.PF_IO_TIME_FROM_FILE if time_from_file else 0,
                                      C.byref(ch)))
    return ch.value
