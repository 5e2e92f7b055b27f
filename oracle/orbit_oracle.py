"""CPU FP64 oracle of the Newton-Krylov orbit search (newton.f90,
NewtonHook.f90, GMRESm.f90) on top of the timestep oracle.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module; the
tests use it as the checker of the device orbit vectors and of the host-side
Newton-hookstep driver.

Parity status: **parity unpinned** (as the timestep oracle: the reference
ships no golden vectors and cannot be built here).  Pinned by invariants the
reference's formulas imply (tests/test_orbit.py): vec2rtz inverts rtz2vec,
the shift directions are the derivatives of var_coll_shift, GMRES solves a
small dense system, and Newton converges on a problem with a known root.

Vectors are numpy arrays of n = 8 + 6*N*H doubles (newton.f90:36, one rank);
index [8 + (nh*N + n)*6 + c] holds component c of (ur Re, ur Im, ut Re, ut Im,
uz Re, uz Im) at mode nh, radial point n.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg

from pipeflow_oracle import Coll, Pipe


# ---------------------------------------------------------------------------
# state <-> vector (newton.f90:567-643)
# ---------------------------------------------------------------------------
def _multipliers(op: Pipe, scaleU):
    """(3, N, H) multipliers: d(n) w(nh) scaleU(c), and d(n) alone for u_z of
    the k = m = 0 mode (newton.f90:578-592)."""
    d = np.sqrt(np.abs(op.mes_D.intrdr))                               # (N,)
    w = 4.0 / (4.0 + (op.cfg.alpha * np.abs(op.kk)) + (op.Mp * np.abs(op.mm)).astype(float))
    s = np.empty((3, op.N, op.H))
    for c in range(3):
        s[c] = d[:, None] * w[None, :] * scaleU[c]
    mean = (op.kk == 0) & (op.mm == 0)
    s[2][:, mean] = d[:, None]
    return s


def vec_len(op: Pipe) -> int:
    return 8 + 6 * op.N * op.H


def rtz2vec(op: Pipe, r: Coll, t: Coll, z: Coll, scaleU, v: np.ndarray) -> None:
    """newton.f90:567-602: writes v[8:], leaves v[0:8]."""
    s = _multipliers(op, scaleU)
    out = np.empty((op.H, op.N, 6))
    for c, f in enumerate((r, t, z)):
        out[:, :, 2 * c] = (f.re * s[c]).T
        out[:, :, 2 * c + 1] = (f.im * s[c]).T
    v[8:] = out.reshape(-1)


def vec2rtz(op: Pipe, v: np.ndarray, scaleU):
    """newton.f90:608-643."""
    s = _multipliers(op, scaleU)
    a = v[8:].reshape(op.H, op.N, 6)
    return [Coll(a[:, :, 2 * c].T / s[c], a[:, :, 2 * c + 1].T / s[c]) for c in range(3)]


def dotprod(n_: int, a: np.ndarray, b: np.ndarray) -> float:
    """newton.f90:652-672 (one rank): n_ = -1 skips the first 8 entries."""
    n1 = 8 if n_ == -1 else 0
    return float(np.dot(a[n1:], b[n1:]))


def getshiftdir(op: Pipe, i: int, x: np.ndarray, scaleU) -> np.ndarray:
    """newton.f90:533-561: i*ds times every mode, ds = Mp m (i=1) or alpha k
    (i=2).  s[0:8] are zero here (the reference leaves them unset)."""
    r, t, z = vec2rtz(op, x, scaleU)
    ds = (op.Mp * op.mm).astype(float) if i == 1 else op.cfg.alpha * op.kk.astype(float)
    out = []
    for f in (r, t, z):
        out.append(Coll(-f.im * ds[None, :], f.re * ds[None, :]))
    s = np.zeros_like(x)
    rtz2vec(op, *out, scaleU, s)
    return s


# ---------------------------------------------------------------------------
# the orbit module (newton.f90:22-40, 272-305, 356-475, 721-860)
# ---------------------------------------------------------------------------
@dataclass
class Orbit:
    op: Pipe
    ndts: list
    T_fixed: bool = False
    epsJ: float = 1e-6
    scaleU: np.ndarray = field(default_factory=lambda: np.ones(3))
    scaleT: float = 1.0
    new_x: np.ndarray | None = None
    new_fx: np.ndarray | None = None

    @property
    def n(self) -> int:
        return vec_len(self.op)

    @property
    def ms(self) -> int:
        return len(self.ndts)

    def get_scales(self) -> None:
        """newton.f90:272-305 from the pipe's current state; new_x must hold
        the unscaled shifts and periods in x[p*n + 0..2]."""
        op, n = self.op, self.n
        Er = op.var_coll_norm(op.vel_ur)[0]
        Et = op.var_coll_norm(op.vel_ut)[0]
        Ez = op.var_coll_norm(op.vel_uz)[0]
        c1 = op.vel_uz.copy()
        c1.re[:, 0] = 0.0
        Ez00 = op.var_coll_norm(c1)[0]
        Ez00 = Ez - Ez00
        Ez = Ez - Ez00
        self.scaleU = np.array([math.sqrt(0.2 * Ez00 / Er), math.sqrt(0.2 * Ez00 / Et),
                                math.sqrt(0.5 * Ez00 / Ez)])
        x0 = self.new_x[:n]
        rtz2vec(op, op.vel_ur, op.vel_ut, op.vel_uz, self.scaleU, x0)
        d = dotprod(-1, x0, x0)
        self.scaleT = x0[2] / math.sqrt(d)
        for p in range(self.ms):
            self.new_x[p * n:p * n + 3] /= self.scaleT

    def steporbit(self, ndts: int, x: np.ndarray, y: np.ndarray) -> None:
        """newton.f90:721-831 without continuation or output; writes y[8:]."""
        op = self.op
        p = x[:3] * self.scaleT
        op.vel_ur, op.vel_ut, op.vel_uz = vec2rtz(op, x, self.scaleU)
        if ndts != 1:
            op.tim_dt = p[2] / float(ndts)
            op.vel_matrices()
        t0, step0 = op.tim_t, op.tim_step
        for _ in range(ndts):
            op.timestep(orbit=True)
        if ndts != 1:
            for name in ("vel_ur", "vel_ut", "vel_uz"):
                setattr(op, name, op.var_coll_shift(-p[0], -p[1], getattr(op, name)))
        else:
            op.tim_t, op.tim_step = t0, step0
        rtz2vec(op, op.vel_ur, op.vel_ut, op.vel_uz, self.scaleU, y)

    def dotprod_ms(self, n_: int, a, b) -> float:
        """newton.f90:678-689."""
        n = self.n
        return sum(dotprod(n_, a[p * n:(p + 1) * n], b[p * n:(p + 1) * n]) for p in range(self.ms))

    def getrhs(self, x: np.ndarray) -> np.ndarray:
        """newton.f90:399-419."""
        n, ms = self.n, self.ms
        y_ = np.zeros(n * ms)
        for p in range(ms):
            p1 = (p + 1) % ms
            self.steporbit(self.ndts[p], x[p * n:(p + 1) * n].copy(), y_[p1 * n:(p1 + 1) * n])
        y = y_ - x
        for p in range(ms):
            y[p * n:p * n + 8] = 0.0
        return y

    def multJ(self, x: np.ndarray) -> np.ndarray:
        """newton.f90:425-465 (no continuation)."""
        n, ms, op = self.n, self.ms, self.op
        eps = math.sqrt(self.dotprod_ms(1, x, x))
        if eps == 0.0:
            raise ZeroDivisionError("multJ: eps=0 (1)")
        eps = self.epsJ * math.sqrt(self.dotprod_ms(1, self.new_x, self.new_x)) / eps
        y = self.new_x + eps * x
        s = self.getrhs(y)
        y = (s - self.new_fx) / eps
        for p in range(ms):
            xp = x[p * n:(p + 1) * n]
            nx = self.new_x[p * n:(p + 1) * n]
            s = getshiftdir(op, 1, nx, self.scaleU)
            y[p * n] = dotprod(-1, s, xp)
            s = getshiftdir(op, 2, nx, self.scaleU)
            y[p * n + 1] = dotprod(-1, s, xp)
            s = np.zeros(n)
            self.steporbit(1, nx, s)
            s = (s - nx) / op.tim_dt
            y[p * n + 2] = dotprod(-1, s, xp)
            if op.cfg.mirrorsym or op.cfg.shiftrefl:
                y[p * n] = xp[0]
            if self.T_fixed:
                y[p * n + 2] = xp[2]
        return y

    def multA(self, x: np.ndarray, y0: np.ndarray, epsA: float) -> np.ndarray:
        """newton.f90:837-860."""
        n = self.n
        y = x.copy()
        for p in range(self.ms):
            nx = self.new_x[p * n:(p + 1) * n]
            eps = math.sqrt(dotprod(-1, y, y))
            if eps == 0.0:
                raise ZeroDivisionError("multA: eps=0 (1)")
            eps = epsA * math.sqrt(dotprod(-1, nx, nx)) / eps
            y = nx + eps * y
            y[:8] = nx[:8]
            self.steporbit(self.ndts[p], y.copy(), y)
            y = (y - y0[p * n:(p + 1) * n]) / eps
        return y


# ---------------------------------------------------------------------------
# GMRES with hookstep (GMRESm.f90) and Newton-hookstep (NewtonHook.f90)
# ---------------------------------------------------------------------------
def hookstep(j: int, h: np.ndarray, beta: float, delta: float):
    """GMRESm.f90:119-153.  Returns (y, predicted residual)."""
    a = h[:j + 1, :j].copy()
    u, s, vt = scipy.linalg.svd(a, full_matrices=True, lapack_driver="gesvd")
    p = beta * u[0, :j]
    mu = max(s[j - 1] * s[j - 1] * 1e-6, 1e-99)
    qn = 1e99
    while qn > delta:
        mu = mu * 1.1
        q = p * s / (mu + s * s)
        qn = math.sqrt(float(np.dot(q, q)))
    y = q @ vt
    pp = -(h[:j + 1, :j] @ y)
    pp[0] += beta
    return y, math.sqrt(float(np.dot(pp, pp)))


def _lsq(hj: np.ndarray, rhs: np.ndarray) -> np.ndarray:
    """dgelsy on the (j+1) x j Hessenberg system (GMRESm.f90:82-85)."""
    y, *_ = scipy.linalg.lstsq(hj, rhs, cond=1e-300, lapack_driver="gelsy")
    return y


class GMRES:
    """gmresm (GMRESm.f90:27-113) with its saved state (h, v, beta, j)."""

    def __init__(self, m: int, n: int):
        self.m, self.n = m, n
        self.h = np.zeros((m + 1, m))
        self.v = np.zeros((m + 1, n))
        self.beta = 0.0
        self.j = 0

    def solve(self, x, b, matvec, dot, res, delta, its, info):
        """Returns (x, res, delta, its, info) as the Fortran arguments on exit."""
        m = self.m
        if info == 2:
            y, delta = hookstep(self.j, self.h, self.beta, delta)
            x = y @ self.v[:self.j]
            return x, res, delta, its, 0
        tol = res
        imx = its
        its = 0
        self.v[:] = 0.0
        while True:  # label 1 (restart)
            res_ = 1e99
            stgn = 1.0 - 1e-14
            beta = math.sqrt(dot(x, x))
            w = np.zeros_like(b) if beta == 0.0 else matvec(x)
            w = b - w
            beta = math.sqrt(dot(w, w))
            self.beta = beta
            self.v[0] = w / beta
            self.h[:] = 0.0
            for j in range(1, m + 1):
                self.j = j
                its += 1
                z = self.v[j - 1].copy()
                w = matvec(z)
                for i in range(1, j + 1):
                    self.h[i - 1, j - 1] = dot(w, self.v[i - 1])
                    w = w - self.h[i - 1, j - 1] * self.v[i - 1]
                self.h[j, j - 1] = math.sqrt(dot(w, w))
                self.v[j] = w / self.h[j, j - 1]
                p = np.zeros(j + 1)
                p[0] = beta
                y = _lsq(self.h[:j + 1, :j], p)
                p = -(self.h[:j + 1, :j] @ y)
                p[0] += beta
                res = math.sqrt(float(np.dot(p, p)))
                done = res <= tol or its == imx or res > res_
                if done or j == m:
                    if delta > 0.0:
                        y, delta = hookstep(j, self.h, beta, delta)
                    z = y @ self.v[:j]
                    x = x + z
                    if its == imx:
                        info = 2
                    if res > res_:
                        info = 1
                    if res <= tol:
                        info = 0
                    if done:
                        return x, res, delta, its, info
                    break  # restart
                res_ = res * stgn


@dataclass
class NewtonResult:
    x: np.ndarray
    fx: np.ndarray
    tol: float
    delta: float
    nits: int
    gits: int
    info: int
    history: list


def newtonhook(f, df, dp, x0, m, gtol, tol, delta, mndl, mxdl, nits, state=None):
    """NewtonHook.f90:46-180.  f(x) and df(s) see the current iterate through
    ``state.new_x``/``state.new_fx`` when a state object is given."""
    n = x0.size
    st = state if state is not None else type("S", (), {})()
    st.new_x = x0.copy()
    new_nits = 0
    new_gits = 0
    new_del = delta
    mxdl_ = mxdl
    ginfo = 0
    gm = GMRES(m, n)
    st.new_fx = f(st.new_x)
    new_tol = math.sqrt(dp(st.new_fx, st.new_fx))
    if delta < 0.0:
        new_del = new_tol / 10.0
        mxdl_ = 1e99
    hist = [(new_nits, new_gits, new_tol, new_del)]
    x_, fx_, tol_ = st.new_x.copy(), st.new_fx.copy(), new_tol
    tol__ = 1e99
    x__ = fx__ = None
    del__ = 0.0
    if new_tol < tol:
        return NewtonResult(st.new_x, st.new_fx, new_tol, new_del, 0, 0, 0, hist)
    while True:
        if new_del < mndl:
            return NewtonResult(st.new_x, st.new_fx, new_tol, new_del, new_nits, new_gits, 3, hist)
        s = np.zeros(n)
        gres = gtol * new_tol
        gdel = new_del
        if ginfo != 2:
            new_gits = m
        s, gres, gdel, new_gits, ginfo = gm.solve(s, fx_, df, dp, gres, gdel, new_gits, ginfo)
        ginfo = 0
        st.new_x = x_ - s
        st.new_fx = f(st.new_x)
        new_tol = math.sqrt(dp(st.new_fx, st.new_fx))
        snrm = math.sqrt(dp(s, s))
        ared = tol_ - new_tol
        pred = tol_ - gdel
        if new_tol > tol__:
            st.new_x, st.new_fx, new_tol, new_del = x__, fx__, tol__, del__
        elif ared < 0.0:
            new_del = snrm * 0.5
            ginfo = 2
        elif ared / pred < 0.75:
            x__, fx__, tol__ = st.new_x.copy(), st.new_fx.copy(), new_tol
            del__ = snrm if ared / pred > 0.1 else snrm * 0.5
            new_del = snrm * 0.7
            ginfo = 2
        elif snrm < new_del * 0.9:
            new_del = min(mxdl_, snrm * 2.0)
        elif new_del < mxdl_ * 0.9:
            x__, fx__, tol__, del__ = st.new_x.copy(), st.new_fx.copy(), new_tol, new_del
            new_del = min(mxdl_, snrm * 2.0)
            ginfo = 2
        if ginfo == 2:
            continue
        new_nits += 1
        hist.append((new_nits, new_gits, new_tol, new_del))
        x_, fx_, tol_ = st.new_x.copy(), st.new_fx.copy(), new_tol
        tol__ = 1e99
        if new_tol < tol:
            return NewtonResult(st.new_x, st.new_fx, new_tol, new_del, new_nits, new_gits, 0, hist)
        if new_nits == nits:
            return NewtonResult(st.new_x, st.new_fx, new_tol, new_del, new_nits, new_gits, 2, hist)
