"""CPU oracle of the state-file path (io.f90:98-392).

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module.  It
reads and writes the files with scipy.io.netcdf_file (an implementation of
the netCDF-3 format independent of the product's) and restates
io_load_state's interpolation and re-truncation in numpy, so the product's
own writer and reader are checked against a second implementation of the
format and of the algorithm.

Parity status: **parity unpinned** -- no state file made by the reference is
available; the structure follows io_save_state (io.f90:303-378) and the
interpolation is pinned by exactness on polynomials (tests/test_statefile.py).
"""
from __future__ import annotations

import math

import numpy as np
import scipy.io

KL = 4


def harmonics(K: int, M: int) -> int:
    return (2 * K - 1) * M - (K - 1)


def write_like_reference(path, N, K, M, Mp, r, state, t=0.0, Re=0.0, alpha=0.0, dt=0.0, dtcor=0.0, dtcfl=0.0,
                         version=1):
    """A state file with io_save_state's definitions, in its order
    (io.f90:315-348); Fortran dims (r, H, ReIm) are (ReIm, H, r) in C order.
    version 1: classic format, 2: 64-bit offsets."""
    H = harmonics(K, M)
    f = scipy.io.netcdf_file(path, "w", version=version)
    f.t = np.float64(t)
    f.Re = np.float64(Re)
    f.alpha = np.float64(alpha)
    f.createDimension("r", N)
    f.createDimension("H", H)
    f.createDimension("ReIm", 2)
    vr = f.createVariable("r", "d", ("r",))
    vdt = f.createVariable("dt", "d", ())
    vc = f.createVariable("dtcor", "d", ())
    vf = f.createVariable("dtcfl", "d", ())
    fields = []
    for nm in ("Ur", "Ut", "Uz"):
        v = f.createVariable(nm, "d", ("ReIm", "H", "r"))
        v.K = np.int32(K)
        v.M = np.int32(M)
        v.Mp = np.int32(Mp)
        fields.append(v)
    vr[:] = r
    vdt[()] = dt
    vc[()] = dtcor
    vf[()] = dtcfl
    for v, (re, im) in zip(fields, state):
        v[0, :, :] = np.asarray(re).T
        v[1, :, :] = np.asarray(im).T
    f.close()


def read_raw(path):
    """Everything in the file, as numpy arrays and floats."""
    f = scipy.io.netcdf_file(path, "r", mmap=False)
    out = {"dims": dict(f.dimensions), "t": float(f.t), "Re": float(f.Re), "alpha": float(f.alpha),
           "r": np.array(f.variables["r"][:]), "dt": float(f.variables["dt"].getValue())}
    for nm in ("dtcor", "dtcfl"):
        out[nm] = float(f.variables[nm].getValue()) if nm in f.variables else math.nan
    for nm in ("Ur", "Ut", "Uz"):
        v = f.variables[nm]
        out[nm] = (np.array(v[:]), int(v.K), int(v.M), int(v.Mp), v.dimensions)
    f.close()
    return out


def interp_weights(xi: np.ndarray, xo: np.ndarray):
    """io_interp_wts (io.f90:232-262): per output point, the input range and
    the first row of the inverse Taylor matrix."""
    ni = xi.size
    rows = []
    for x in xo:
        j = 0
        while xi[j] < x - 1e-8 and j < ni - 1:
            j += 1
        lo, hi = max(0, j - KL), min(j + KL, ni - 1)
        pts = xi[lo:hi + 1]
        m = pts.size
        A = np.empty((m, m))
        A[:, 0] = 1.0
        for c in range(1, m):
            A[:, c] = A[:, c - 1] * (pts - x) / c
        rows.append((lo, np.linalg.inv(A)[0]))
    return rows


def load_state(path, N, K, M, Mp, r_target):
    """io_load_state + io_load_coll (io.f90:98-226) onto (N, K, M, Mp, r).
    Returns (state, scalars)."""
    raw = read_raw(path)
    r_ = raw["r"]
    N_ = r_.size
    xi = np.concatenate([-r_[KL - 1::-1], r_])
    interp = True if N_ != N else bool(np.max(np.abs(np.asarray(r_target) - r_)) > 1e-8)
    W = interp_weights(xi, np.asarray(r_target)) if interp else None
    H = harmonics(K, M)
    state = []
    for nm, S in (("Ur", 1), ("Ut", 1), ("Uz", 0)):
        data, K_, M_, Mp_, _ = raw[nm]
        if Mp_ != Mp and M_ > 2:
            raise ValueError("io_load_coll: Mp /= i_Mp")
        H_ = data.shape[1]
        out = [np.zeros((N, H)), np.zeros((N, H))]
        K1, M1 = max(K_, K) - 1, max(M_, M) - 1
        nhf = nh = -1
        for m in range(M1 + 1):
            for k in range(-K1, K1 + 1):
                if k < 0 and m == 0:
                    continue
                if abs(k) >= K or m >= M:
                    nhf += 1
                    continue
                nh += 1
                if abs(k) >= K_ or m >= M_:
                    continue
                nhf += 1
                if nhf >= H_:
                    continue
                for p in range(2):
                    fn = data[p, nhf, :]
                    if interp:
                        sg = -1.0 if (m * Mp + S) % 2 == 1 else 1.0
                        fe = np.concatenate([sg * fn[KL - 1::-1], fn])
                        out[p][:, nh] = [float(w @ fe[lo:lo + w.size]) for lo, w in W]
                    else:
                        out[p][:, nh] = fn
        state.append((out[0], out[1]))
    sc = {k: raw[k] for k in ("t", "Re", "alpha", "dt", "dtcor", "dtcfl")}
    return state, sc
