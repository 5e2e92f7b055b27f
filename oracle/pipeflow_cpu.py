"""C++/OpenMP CPU restatement of the timestep (oracle/pipeflow_cpu.cpp).

TEST INFRASTRUCTURE, not the product.  It serves as the CPU baseline that
``bench.py`` times on the host cores (the reference's own FFTW+MPI build
cannot be compiled here) and as a second, independent restatement that the
numpy oracle is checked against (tests/test_cpu_oracle.py).

``CpuPipe(oracle_pipe)`` takes the set-up an oracle ``Pipe`` made in
``vel_matrices`` (radial mesh, banded LU factors as scipy's dgbtrf left them,
explicit-side matrices, influence matrices) and then steps on its own.

    python oracle/pipeflow_cpu.py      # builds oracle/_build/libpipeflow_cpu.so
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "pipeflow_cpu.cpp"
LIB = HERE / "_build" / "libpipeflow_cpu.so"
KL = 4

_lib = None


def build(force: bool = False) -> Path:
    """Compile the shared library (g++, OpenMP, no FMA contraction so the
    arithmetic follows the numpy oracle's operation order; plain complex
    products, without the C99 infinity and NaN recovery)."""
    if LIB.exists() and not force and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    LIB.parent.mkdir(parents=True, exist_ok=True)
    cmd = ["g++", "-O3", "-march=native", "-fopenmp", "-ffp-contract=off", "-fcx-limited-range", "-std=c++17",
           "-fPIC", "-shared",
           "-o", str(LIB), str(SRC)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"building the CPU oracle failed:\n{r.stderr}")
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    build()
    lib = C.CDLL(str(LIB))
    D, I, P = C.POINTER(C.c_double), C.c_int, C.c_void_p
    lib.pfc_create.restype = P
    lib.pfc_create.argtypes = [I, I, I, I, C.c_double, C.c_double, C.c_double, I, C.c_double, C.c_double,
                               D, D, D, D, D, D]
    lib.pfc_destroy.argtypes = [P]
    lib.pfc_set_lu.argtypes = [P, I, D, C.POINTER(C.c_int)]
    lib.pfc_set_lt.argtypes = [P, I, D, D]
    lib.pfc_set_influence.argtypes = [P, D, D, D, C.c_double]
    lib.pfc_set_state.argtypes = [P, D, D, D, D, D, D, C.c_double, C.c_double]
    lib.pfc_get_state.argtypes = [P, D, D, D, D, D, D]
    lib.pfc_timestep.argtypes = [P, I]
    lib.pfc_timestep.restype = I
    lib.pfc_threads.restype = I
    lib.pfc_set_threads.argtypes = [I]
    _lib = lib
    return lib


def _d(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def threads() -> int:
    return load().pfc_threads()


def set_threads(n: int) -> None:
    load().pfc_set_threads(int(n))


class CpuPipe:
    """One pipe stepped by the C++ restatement, set up from an oracle Pipe
    on which vel_matrices has run (fixed dt, no symmetry flags beyond the
    mean-mode one)."""

    def __init__(self, op):
        cfg = op.cfg
        if cfg.mirrorsym or cfg.shiftrefl or cfg.shiftrott:
            raise ValueError("the CPU restatement covers the mean-mode symmetry only")
        lib = load()
        self.lib = lib
        self.N, self.H = op.N, op.H
        D = op.mes_D
        self._keep = []

        def arr(a, dtype=np.float64):
            a = np.ascontiguousarray(a, dtype=dtype)
            self._keep.append(a)
            return a

        drb = arr(D.dr[0])
        rm1 = arr(D.rp[-1])
        velU = arr(op.vel_U)
        velUp = arr(op.vel_Up)
        intrdr = arr(D.intrdr)
        dr1 = arr(D.dr1)
        self.h = lib.pfc_create(op.N, op.K, op.M, op.Mp, cfg.alpha, cfg.Re, cfg.implicit, int(cfg.const_flux),
                                cfg.dterr, cfg.courant, _d(drb), _d(rm1), _d(velU), _d(velUp), _d(intrdr), _d(dr1))
        for which, (AB, piv) in enumerate((op.LNp, op.LDp, op.LDm, op.LDz)):
            ab = np.ascontiguousarray(AB, dtype=np.float64)
            ip = np.ascontiguousarray(piv, dtype=np.int32) + 1  # LAPACK's 1-based pivots
            lib.pfc_set_lu(self.h, which, _d(ab), ip.ctypes.data_as(C.POINTER(C.c_int)))
        for which, (off, diag) in enumerate((op.Ltp, op.Ltm, op.Ltz)):
            lib.pfc_set_lt(self.h, which, _d(np.ascontiguousarray(off)), _d(np.ascontiguousarray(diag)))
        A = np.ascontiguousarray(op._A, dtype=np.float64)
        U = np.ascontiguousarray(op._U, dtype=np.float64)
        Ui = np.ascontiguousarray(getattr(op, "_Ui", np.zeros(op.N)), dtype=np.float64)
        lib.pfc_set_influence(self.h, _d(A), _d(U), _d(Ui), float(getattr(op, "_flux_d1", 1.0)))
        self.dt = op.tim_dt
        self.set_state(*op.state(), Pr0=op.vel_Pr0)

    def set_state(self, ur, ut, uz, Pr0: float = 0.0):
        a = [np.ascontiguousarray(x, dtype=np.float64) for f in (ur, ut, uz) for x in (f.re, f.im)]
        self.lib.pfc_set_state(self.h, *[_d(x) for x in a], float(self.dt), float(Pr0))

    def state(self):
        a = [np.empty((self.N, self.H)) for _ in range(6)]
        self.lib.pfc_get_state(self.h, *[_d(x) for x in a])
        return [(a[0], a[1]), (a[2], a[3]), (a[4], a[5])]

    def timestep(self, orbit: bool = False) -> int:
        n = self.lib.pfc_timestep(self.h, int(orbit))
        if n < 0:
            raise RuntimeError(f"tim_check_cgce failure {n}")
        return n

    def close(self):
        if self.h:
            self.lib.pfc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


if __name__ == "__main__":
    print(build(force=True), "threads:", os.cpu_count())
