"""Newton-Krylov search for relative periodic orbits (newton.f90 with
NewtonHook.f90 and GMRESm.f90) over the device timestep.

The time-T map, the state <-> vector scaling, the shift directions and the
dot products run on the GPU through the C ABI (pf_orbit_*); the Krylov basis
and every Newton vector stay in device memory as float64 torch tensors.  The
small dense work -- the least-squares solve of the Hessenberg system (dgelsy)
and the hookstep's SVD (dgesvd) -- runs on the host through scipy's LAPACK,
as the reference keeps it in LAPACK.

Entry points, named after the reference's routines:

    orb = Orbit(pipe, ndts=[100], shifts=[(0.0, sz, T)])   # shifts.in
    orb.get_scales()                 # newton.f90:272-305 (after the state is set)
    orb.load_ms_states()             # newton.f90:311-350 (shooting points by stepping)
    orb.search_sz()                  # newton.f90:356-394
    res = orb.solve(m=150, nits=100, rel_err=3e-6, delta=-1.0, mndl=1e-7,
                    mxdl=1e7, gtol=1e-3)     # the main program's call of newtonhook

plus getrhs / multJ / multA / steporbit / dotprod / dotprod_ms / getshiftdir /
rtz2vec / vec2rtz on device vectors, and get_eigen (newton.f90:868-979, the
Arnoldi iteration of arnoldi.f on multA) for the Floquet spectrum of the
converged orbit, and parameter continuation in Re or alpha
(start_continuation / continuation_run, newton.f90:89-170).  The output files
are not included.
"""
from __future__ import annotations

import copy
import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg
import torch

from . import _lib as L
from .api import Pipe, PipeflowError, _check


def _ptr(t: torch.Tensor) -> int:
    return t.data_ptr()


# ---------------------------------------------------------------------------
# GMRES with hookstep (GMRESm.f90) on device vectors
# ---------------------------------------------------------------------------
def hookstep(j: int, h: np.ndarray, beta: float, delta: float):
    """GMRESm.f90:119-153: the y that gives the hookstep of size delta in the
    Krylov space of dimension j, and the residual that it predicts."""
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


def _least_squares(hj: np.ndarray, rhs: np.ndarray) -> np.ndarray:
    """dgelsy on the (j+1) x j Hessenberg system (GMRESm.f90:82-85), full
    rank unless a column is exactly dependent."""
    y, *_ = scipy.linalg.lstsq(hj, rhs, cond=1e-300, lapack_driver="gelsy")
    return y


class GMRES:
    """gmresm (GMRESm.f90:27-113).  The Krylov basis v (m+1 vectors) lives
    on the vectors' device; h, beta and j are kept between calls, so that
    info=2 recomputes the hookstep for a new trust region without new
    matrix-vector products."""

    def __init__(self, m: int, n: int, like: torch.Tensor):
        self.m, self.n = m, n
        self.h = np.zeros((m + 1, m))
        self.v = torch.zeros((m + 1, n), dtype=like.dtype, device=like.device)
        self.beta = 0.0
        self.j = 0

    def _combine(self, y: np.ndarray, j: int) -> torch.Tensor:
        yt = torch.as_tensor(y[:j], dtype=self.v.dtype).to(self.v.device, non_blocking=False)
        return yt @ self.v[:j]

    def solve(self, x, b, matvec, dot, res, delta, its, info):
        """Returns (x, res, delta, its, info) as gmresm leaves its arguments:
        x the solution (hookstep if delta > 0), res the residual reached,
        delta the residual the hookstep predicts, its the iterations taken,
        info 0 converged / 1 breakdown / 2 iteration limit."""
        m = self.m
        if info == 2:
            y, delta = hookstep(self.j, self.h, self.beta, delta)
            return self._combine(y, self.j), res, delta, its, 0
        tol = res
        imx = its
        its = 0
        self.v.zero_()
        while True:
            res_ = 1e99
            stgn = 1.0 - 1e-14
            beta = math.sqrt(dot(x, x))
            w = torch.zeros_like(b) if beta == 0.0 else matvec(x)
            w = b - w
            beta = math.sqrt(dot(w, w))
            self.beta = beta
            self.v[0] = w / beta
            self.h[:] = 0.0
            for j in range(1, m + 1):
                self.j = j
                its += 1
                w = matvec(self.v[j - 1].clone())
                for i in range(1, j + 1):
                    hij = dot(w, self.v[i - 1])
                    self.h[i - 1, j - 1] = hij
                    w = w - hij * self.v[i - 1]
                self.h[j, j - 1] = math.sqrt(dot(w, w))
                self.v[j] = w / self.h[j, j - 1]
                p = np.zeros(j + 1)
                p[0] = beta
                y = _least_squares(self.h[:j + 1, :j], p)
                p = -(self.h[:j + 1, :j] @ y)
                p[0] += beta
                res = math.sqrt(float(np.dot(p, p)))
                done = res <= tol or its == imx or res > res_
                if done or j == m:
                    if delta > 0.0:
                        y, delta = hookstep(j, self.h, beta, delta)
                    x = x + self._combine(y, j)
                    if its == imx:
                        info = 2
                    if res > res_:
                        info = 1
                    if res <= tol:
                        info = 0
                    if done:
                        return x, res, delta, its, info
                    break  # restart with the new x
                res_ = res * stgn


@dataclass
class NewtonResult:
    """newtonhook's exit state: the iterate, its residual vector and norm,
    the trust region, Newton and GMRES iteration counts, and info
    (0 converged, 2 iteration limit, 3 trust region below mndl)."""
    x: torch.Tensor
    fx: torch.Tensor
    tol: float
    delta: float
    nits: int
    gits: int
    info: int
    history: list = field(default_factory=list)


class NewtonState:
    """The newton module's variables (NewtonHook.f90:39-45)."""
    new_x = None
    new_fx = None
    new_tol = 0.0
    new_del = 0.0
    new_nits = 0
    new_gits = 0


def newtonhook(f, df, dp, x0, m, gtol, tol, delta, mndl, mxdl, nits, state: NewtonState | None = None, sub=None):
    """Newton iteration with GMRES hooksteps (NewtonHook.f90:46-180) for
    f(x) = 0.  f and df map vectors to vectors (df is the Jacobian with its
    constraint rows), dp is the dot product, sub() runs after every accepted
    iteration; state.new_x / state.new_fx hold the current iterate while f
    and df run."""
    n = x0.numel()
    st = state if state is not None else NewtonState()
    st.new_x = x0.clone()
    st.new_nits = 0
    st.new_gits = 0
    st.new_del = delta
    mxdl_ = mxdl
    ginfo = 0
    gm = GMRES(m, n, x0)
    st.new_fx = f(st.new_x)
    st.new_tol = math.sqrt(dp(st.new_fx, st.new_fx))
    if delta < 0.0:
        st.new_del = st.new_tol / 10.0
        mxdl_ = 1e99
    hist = [(st.new_nits, st.new_gits, st.new_tol, st.new_del)]
    if sub:
        sub()
    x_, fx_, tol_ = st.new_x.clone(), st.new_fx.clone(), st.new_tol
    tol__ = 1e99
    x__ = fx__ = None
    del__ = 0.0

    def result(info):
        return NewtonResult(st.new_x, st.new_fx, st.new_tol, st.new_del, st.new_nits, st.new_gits, info, hist)

    if st.new_tol < tol:
        return result(0)
    while True:
        if st.new_del < mndl:
            return result(3)
        s = torch.zeros_like(x0)
        gres = gtol * st.new_tol
        gdel = st.new_del
        if ginfo != 2:
            st.new_gits = m
        s, gres, gdel, st.new_gits, ginfo = gm.solve(s, fx_, df, dp, gres, gdel, st.new_gits, ginfo)
        ginfo = 0
        st.new_x = x_ - s
        st.new_fx = f(st.new_x)
        st.new_tol = math.sqrt(dp(st.new_fx, st.new_fx))
        snrm = math.sqrt(dp(s, s))
        ared = tol_ - st.new_tol
        pred = tol_ - gdel
        if st.new_tol > tol__:  # accept the previous, better step
            st.new_x, st.new_fx, st.new_tol, st.new_del = x__, fx__, tol__, del__
        elif ared < 0.0:  # norm increased: smaller step
            st.new_del = snrm * 0.5
            ginfo = 2
        elif ared / pred < 0.75:  # step ok: try a smaller one
            x__, fx__, tol__ = st.new_x.clone(), st.new_fx.clone(), st.new_tol
            del__ = snrm if ared / pred > 0.1 else snrm * 0.5
            st.new_del = snrm * 0.7
            ginfo = 2
        elif snrm < st.new_del * 0.9:  # full Newton step taken
            st.new_del = min(mxdl_, snrm * 2.0)
        elif st.new_del < mxdl_ * 0.9:  # good step: try a larger one
            x__, fx__, tol__, del__ = st.new_x.clone(), st.new_fx.clone(), st.new_tol, st.new_del
            st.new_del = min(mxdl_, snrm * 2.0)
            ginfo = 2
        if ginfo == 2:
            continue
        st.new_nits += 1
        hist.append((st.new_nits, st.new_gits, st.new_tol, st.new_del))
        if sub:
            sub()
        x_, fx_, tol_ = st.new_x.clone(), st.new_fx.clone(), st.new_tol
        tol__ = 1e99
        if st.new_tol < tol:
            return result(0)
        if st.new_nits == nits:
            return result(2)


# ---------------------------------------------------------------------------
# Arnoldi iteration (arnoldi.f) on device vectors
# ---------------------------------------------------------------------------
SMALL = 1e-80


class Arnoldi:
    """arnold (arnoldi.f:22-254): one call per new vector A.q_k.  The Krylov
    basis q (kmax vectors) lives on the vectors' device, the Hessenberg
    matrix h on the host; the eigenvalues of the k x k Hessenberg matrix come
    from LAPACK's dgeev (balance, Hessenberg reduction, QR), which runs the
    same dgebal / dgehrd / dhseqr sequence as the reference, and the
    eigenvectors of the converged ones from the same decomposition (the
    reference uses inverse iteration, dhsein; an eigenvector is defined up
    to a scalar either way)."""

    def __init__(self, n: int, kmax: int, ncgd: int, dp, tol: float, like: torch.Tensor):
        self.n, self.kmax, self.ncgd, self.dp, self.tol = n, kmax, ncgd, dp, tol
        self.q = torch.zeros((kmax, n), dtype=like.dtype, device=like.device)
        self.h = np.zeros((kmax, kmax))
        self.wr2 = np.zeros(ncgd)
        self.wi2 = np.zeros(ncgd)
        self.k = 0
        self.b = None  # converged eigenvectors, columns as rows: (<= 2 ncgd, n)

    def step(self, sv: torch.Tensor):
        """Returns (ifail, sv): ifail -1 converged, 0 continue with sv <- A.sv,
        1 reached kmax, 2 invariant subspace."""
        k, h, q = self.k, self.h, self.q
        if k >= self.kmax:
            return 1, sv
        q[k] = sv
        for j in range(1, k + 1):  # modified Gram-Schmidt
            h[j - 1, k - 1] = self.dp(q[k], q[j - 1])
            q[k] -= h[j - 1, k - 1] * q[j - 1]
        for j in range(1, k + 1):  # reorthogonalise
            norm = self.dp(q[k], q[j - 1])
            q[k] -= norm * q[j - 1]
            h[j - 1, k - 1] += norm
        norm = math.sqrt(self.dp(q[k], q[k]))
        if norm < SMALL:
            return 2, sv
        q[k] /= norm
        sv = q[k].clone()
        ifail = 0
        if k == 0:
            h[:] = 0.0
        else:
            h[k, k - 1] = norm
            if k >= self.ncgd:
                ifail = self._eigen(k)
        self.k = k + 1
        return ifail, sv

    def _eigen(self, k: int) -> int:
        w, vr = scipy.linalg.eig(self.h[:k, :k], right=True)
        wr, wi = w.real.copy(), w.imag.copy()
        select = [False] * k
        p = 0
        for i in range(self.ncgd):  # largest magnitude first; compare with the last call's
            norm, m = -1.0, 0
            for j in range(k):
                if not select[j]:
                    nm = wr[j] * wr[j] + wi[j] * wi[j]
                    if nm > norm:
                        norm, m = nm, j
            select[m] = True
            if abs(wi[m]) > SMALL and m + 1 < k:
                select[m + 1] = True
            if math.hypot(wr[m] - self.wr2[i], wi[m] - self.wi2[i]) < self.tol:
                p += 1
            self.wr2[i], self.wi2[i] = wr[m], wi[m]
        if p < self.ncgd:
            return 0
        # eigenvectors of h for the converged values, in wr2 order: one
        # column for a real value, (Re, Im) for a complex pair
        cols = []
        for i in range(self.ncgd):
            j = int(np.argmin(np.abs(w - complex(self.wr2[i], self.wi2[i]))))
            v = vr[:, j]
            v = v / np.max(np.abs(v.real) + np.abs(v.imag))  # dhsein's normalisation
            cols.append(v.real)
            if abs(self.wi2[i]) > SMALL:
                cols.append(v.imag)
        V = torch.as_tensor(np.array(cols), dtype=self.q.dtype).to(self.q.device)
        self.b = V @ self.q[:k]
        return -1


def logeig(wr: np.ndarray, wi: np.ndarray, t: float):
    """logeig (arnoldi.f:264-312): Floquet multipliers w = wr + i wi of the
    period-t map to exponents sigma with w = exp(sigma t)."""
    sr, si = np.empty_like(wr), np.empty_like(wi)
    for i, (re, im) in enumerate(zip(wr, wi)):
        if abs(re) < SMALL:
            if abs(im) < SMALL:
                raise PipeflowError(L.PF_ERR_ARG, f"logeig: zero multiplier {i + 1}")
            th = 0.5 * math.pi if im > 0.0 else -0.5 * math.pi
        elif re > 0.0:
            th = math.atan(im / re)
        else:
            th = math.pi + math.atan(im / re) if im > 0.0 else -math.pi + math.atan(im / re)
        sr[i] = math.log(math.sqrt(re * re + im * im)) / t
        si[i] = th / t
    return sr, si


# ---------------------------------------------------------------------------
# parameter continuation (the main program of newton.f90)
# ---------------------------------------------------------------------------
def continuation_start(new_x, x_second, n: int, ms: int, ctdp0: float, param: float, d: float):
    """newton.f90:102-117: from the first solution new_x and the second
    x_second (entry 3 of each block the parameter they were found at), the
    branch direction ctstp = x_second - new_x (a unit step in the parameter
    if they are equal), the last point ctx_ = x_second, the first guess
    x_second + ctdp0 ctstp, and the parameter entries divided by
    ctpsc = param / sqrt(d).  Returns (new_x, ctstp, ctx_, ctpsc)."""
    ctx_ = new_x.clone()
    nx = x_second.clone()
    ctstp = nx - ctx_
    if float(ctstp.abs().max()) == 0.0:
        ctstp.view(ms, n)[:, 3] += 1.0
    ctx_ = nx.clone()
    nx = nx + ctstp * ctdp0
    ctpsc = param / math.sqrt(d)
    for v in (nx, ctstp, ctx_):
        v.view(ms, n)[:, 3] /= ctpsc
    return nx, ctstp, ctx_, ctpsc


def continuation_next(new_x, ctx_, nits: int, gits: int, ctntmn: int, ctntmx: int, n: int, ms: int, ndts,
                      T_fixed: bool, m: int):
    """newton.f90:155-170: the next guess along the branch after a point
    found in nits Newton iterations: the last step scaled by 1.1, by 0.5
    above ctntmx iterations or by 2 below ctntmn; with a fixed period the
    steps per period and the shifts and periods of new_x and ctx_ scaled by
    2 (more than 2m/3 GMRES iterations) or 0.5 (fewer than 10).  Returns
    (new_x, ctstp, ctx_, ndts)."""
    d = 1.1
    if nits > ctntmx:
        d = 0.5
    if nits < ctntmn:
        d = 2.0
    ctstp = new_x - ctx_
    ctx_ = new_x.clone()
    nx = new_x + ctstp * d
    ndts = list(ndts)
    if T_fixed:
        d = 1.0
        if gits > (2 * m) // 3:
            d = 2.0
        if gits < 10:
            d = 0.5
        ndts = [int(nd * d + 0.5) for nd in ndts]
        for v in (nx, ctx_):
            v.view(ms, n)[:, :3] *= d
    return nx, ctstp, ctx_, ndts


# ---------------------------------------------------------------------------
# the orbit module (newton.f90)
# ---------------------------------------------------------------------------
class Orbit(NewtonState):
    """newton.f90's orbit module for one pipe: ms = len(ndts) shooting
    points, ndts[p] timesteps from point p to p+1, shifts[p] = (theta shift,
    z shift, period) as read from shifts.in.  All vectors are float64 CUDA
    tensors of ms*n entries, n = 8 + 6*N*H.  The pipe's work is moved onto a
    stream of its own that the vector arithmetic shares."""

    def __init__(self, pipe: Pipe, ndts, shifts, T_fixed: bool = False, epsJ: float = 1e-6, continuation=None):
        if not torch.cuda.is_available():
            raise PipeflowError(L.PF_ERR_NODEVICE, "Orbit: no CUDA device")
        self.pipe = pipe
        self.lib = pipe.lib
        self.ctx = pipe.ctx
        dev = pipe.device if pipe.device >= 0 else torch.cuda.current_device()
        self.dev = torch.device("cuda", dev)
        self.stream = torch.cuda.Stream(device=self.dev)
        _check(self.lib.pf_ctx_set_stream(self.ctx, C.c_void_p(self.stream.cuda_stream)))
        nn = C.c_longlong()
        _check(self.lib.pf_orbit_vec_len(self.ctx, C.byref(nn)))
        self.n = nn.value
        self.ndts = [int(d) for d in ndts]
        self.ms = len(self.ndts)
        if self.ms < 1 or len(shifts) != self.ms:
            raise PipeflowError(L.PF_ERR_ARG, "Orbit: one (theta shift, z shift, period) per shooting point")
        self.T_fixed = T_fixed
        self.epsJ = epsJ
        # parameter continuation (params_ct.in): param "Re" (ctp 1) or
        # "alpha" (ctp 2), first step ctdp0, Newton-count window ctntmn..ctntmx
        self.Ctnu = continuation is not None
        if self.Ctnu:
            c = dict(continuation)
            if c.get("param") not in ("Re", "alpha"):
                raise PipeflowError(L.PF_ERR_ARG, "Orbit: continuation param must be 'Re' or 'alpha'")
            self.ctp = 1 if c["param"] == "Re" else 2
            self.ctdp0 = float(c.get("ctdp0", 0.01))
            self.ctntmn = int(c.get("ctntmn", 3))
            self.ctntmx = int(c.get("ctntmx", 8))
            self.ctpsc = 1.0
            self.ctstp = None
            self.ctx_ = None
            self._d0 = None
            self._m = 150
            self.cti = 0
        self.scaleU = np.ones(3)
        self.scaleT = 1.0
        with torch.cuda.stream(self.stream):
            self.new_x = torch.zeros(self.ms * self.n, dtype=torch.float64, device=self.dev)
            hdr = torch.tensor(np.asarray(shifts, dtype=np.float64).reshape(self.ms, 3), device=self.dev)
            self.new_x.view(self.ms, self.n)[:, :3] = hdr
            if self.Ctnu:  # x(4::n) = the parameter (newton.f90:318-326)
                self.new_x.view(self.ms, self.n)[:, 3] = self._parameter()
            self.new_fx = torch.zeros_like(self.new_x)
        self.history = []

    # -- vector maps -------------------------------------------------------
    def _part(self, v: torch.Tensor, p: int) -> torch.Tensor:
        return v[p * self.n:(p + 1) * self.n]

    def set_scales(self, scaleU, scaleT: float) -> None:
        self.scaleU = np.asarray(scaleU, dtype=np.float64).copy()
        self.scaleT = float(scaleT)
        _check(self.lib.pf_orbit_set_scales(self.ctx, self.scaleU.ctypes.data_as(L.DP), self.scaleT))

    def rtz2vec(self, v: torch.Tensor) -> None:
        """vel_ur, vel_ut, vel_uz -> v[8:n] (newton.f90:567-602)."""
        _check(self.lib.pf_orbit_rtz2vec(self.ctx, C.c_void_p(_ptr(v))))

    def vec2rtz(self, v: torch.Tensor) -> None:
        """v -> vel_ur, vel_ut, vel_uz (newton.f90:608-643)."""
        _check(self.lib.pf_orbit_vec2rtz(self.ctx, C.c_void_p(_ptr(v))))

    def dotprod(self, n_: int, a: torch.Tensor, b: torch.Tensor) -> float:
        """newton.f90:652-672: n_ = -1 leaves out the 8 header entries."""
        out = C.c_double()
        _check(self.lib.pf_orbit_dotprod(self.ctx, int(n_), C.c_void_p(_ptr(a)), C.c_void_p(_ptr(b)),
                                         C.byref(out)))
        return out.value

    def dotprod_ms(self, n_: int, a: torch.Tensor, b: torch.Tensor) -> float:
        """newton.f90:678-689."""
        return sum(self.dotprod(n_, self._part(a, p), self._part(b, p)) for p in range(self.ms))

    def getshiftdir(self, i: int, x: torch.Tensor) -> torch.Tensor:
        """newton.f90:533-561: direction of a theta (i=1) or z (i=2) shift."""
        with torch.cuda.stream(self.stream):
            s = torch.zeros(self.n, dtype=torch.float64, device=self.dev)
        _check(self.lib.pf_orbit_shiftdir(self.ctx, int(i), C.c_void_p(_ptr(x)), C.c_void_p(_ptr(s))))
        return s

    def _parameter(self) -> float:
        return float(self.pipe.cfg.Re if self.ctp == 1 else self.pipe.cfg.alpha)

    def _set_parameter(self, v: float) -> None:
        """d_Re or d_alpha = v and var_precompute (newton.f90:730-735),
        through pf_ctx_reconfigure; steporbit then recomputes the matrices."""
        if v == self._parameter():
            return
        if not (math.isfinite(v) and v > 0.0):
            raise PipeflowError(L.PF_ERR_ARG, f"continuation parameter {v} out of range")
        cfg = copy.copy(self.pipe.cfg)
        if self.ctp == 1:
            cfg.Re = v
        else:
            cfg.alpha = v
        self.pipe.reconfigure(cfg)

    def steporbit(self, ndts: int, x: torch.Tensor, y: torch.Tensor) -> None:
        """newton.f90:721-831 (no output): y[8:] = the state ndts steps
        from x, shifted back for ndts != 1; with continuation the parameter
        x[3]*ctpsc is set first."""
        if self.Ctnu and ndts != 1:
            self._set_parameter(float(x[3].item()) * self.ctpsc)
        s = self.lib.pf_orbit_step(self.ctx, int(ndts), C.c_void_p(_ptr(x)), C.c_void_p(_ptr(y)))
        if s not in (L.PF_OK, L.PF_ERR_CONVERGE):
            _check(s)

    # -- set-up (newton.f90:272-394) ----------------------------------------
    def get_scales(self) -> None:
        """newton.f90:272-305 from the pipe's current state: scaleU from the
        energies of ur, ut and of uz without and with its mean mode, scaleT
        from the first period and the size of the state vector."""
        p = self.pipe
        Er = p.var_coll_norm(p.vel_ur)[0]
        Et = p.var_coll_norm(p.vel_ut)[0]
        Ez = p.var_coll_norm(p.vel_uz)[0]
        c1 = p.coll()
        p.var_coll_copy(p.vel_uz, c1)
        re, im = c1.download()
        re[:, 0] = 0.0
        c1.upload(re, im)
        Ez00 = p.var_coll_norm(c1)[0]
        Ez00 = Ez - Ez00
        Ez = Ez - Ez00
        self.set_scales([math.sqrt(0.2 * Ez00 / Er), math.sqrt(0.2 * Ez00 / Et), math.sqrt(0.5 * Ez00 / Ez)],
                        1.0)
        x0 = self._part(self.new_x, 0)
        self.rtz2vec(x0)
        d = self.dotprod(-1, x0, x0)
        with torch.cuda.stream(self.stream):
            scaleT = float(x0[2].item()) / math.sqrt(d)
            self.new_x.view(self.ms, self.n)[:, :3] /= scaleT
        self.set_scales(self.scaleU, scaleT)

    def load_ms_states(self) -> None:
        """newton.f90:311-350 without state files: shooting point p >= 1
        is the state ndts[p-1] steps on from point p-1; point 0 is the
        pipe's current state."""
        self.rtz2vec(self._part(self.new_x, 0))
        for p in range(1, self.ms):
            x = self._part(self.new_x, p - 1).clone()
            with torch.cuda.stream(self.stream):
                y = torch.zeros(self.n, dtype=torch.float64, device=self.dev)
            self.steporbit(self.ndts[p - 1], x, y)
            with torch.cuda.stream(self.stream):
                self._part(self.new_x, p)[8:] = y[8:]

    def search_sz(self) -> None:
        """newton.f90:356-394: for every shooting point whose shifts are
        (0, -1), the z shift in [0, 2 pi/alpha) on a 0.01 grid that brings
        the end state closest to the next point."""
        p_ = self.pipe
        n = self.n
        for p1 in range(self.ms):
            p = (p1 + 1) % self.ms
            hdr = self._part(self.new_x, p1)[:2].cpu().numpy() * self.scaleT
            st, sz = float(hdr[0]), float(hdr[1])
            if abs(st) > 1e-8 or abs(sz + 1.0) > 1e-8:
                continue
            with torch.cuda.stream(self.stream):
                x = self._part(self.new_x, p).clone()
                y = self._part(self.new_x, p1).clone()
                y[1] = 0.0
            self.steporbit(self.ndts[p1], y, y)
            self.vec2rtz(y)
            r, t, z = p_.coll(), p_.coll(), p_.coll()
            for i, c in enumerate((r, t, z)):
                p_.var_coll_copy(p_.vel_field(i), c)
            d1 = 1e99
            sz = 0.0
            sz_ = 0.0
            alpha = p_.cfg.alpha
            while sz < 2.0 * math.pi / alpha:
                for i, c in enumerate((r, t, z)):
                    p_.var_coll_shift(0.0, -sz, c, p_.vel_field(i))
                self.rtz2vec(y)
                with torch.cuda.stream(self.stream):
                    dlt = y - x
                d2 = self.dotprod(-1, dlt, dlt)
                if d2 < d1:
                    sz_ = sz
                    d1 = d2
                sz = sz + 0.01
            with torch.cuda.stream(self.stream):
                self.new_x[p1 * n + 1] = sz_ / self.scaleT

    # -- the Newton operators (newton.f90:399-475, 837-860) -------------------
    def getrhs(self, x: torch.Tensor) -> torch.Tensor:
        """newton.f90:399-419: y = F(x) - x, header entries 0."""
        n, ms = self.n, self.ms
        with torch.cuda.stream(self.stream):
            y_ = torch.zeros(n * ms, dtype=torch.float64, device=self.dev)
        for p in range(ms):
            p1 = (p + 1) % ms
            self.steporbit(self.ndts[p], self._part(x, p), self._part(y_, p1))
        with torch.cuda.stream(self.stream):
            y = y_ - x
            y.view(ms, n)[:, :8] = 0.0
        return y

    def multJ(self, x: torch.Tensor) -> torch.Tensor:
        """newton.f90:425-465 (no continuation): finite-difference Jacobian
        times x, with the constraint rows (no update along the shifts or
        the trajectory; fixed period if T_fixed)."""
        n, ms = self.n, self.ms
        eps = math.sqrt(self.dotprod_ms(1, x, x))
        if eps == 0.0:
            raise PipeflowError(L.PF_ERR_ARG, "multJ: eps=0 (1)")
        eps = self.epsJ * math.sqrt(self.dotprod_ms(1, self.new_x, self.new_x)) / eps
        if eps == 0.0:
            raise PipeflowError(L.PF_ERR_ARG, "multJ: eps=0 (2)")
        with torch.cuda.stream(self.stream):
            y = self.new_x + eps * x
        s = self.getrhs(y)
        with torch.cuda.stream(self.stream):
            y = (s - self.new_fx) / eps
        cfg = self.pipe.cfg
        for p in range(ms):
            xp = self._part(x, p)
            nx = self._part(self.new_x, p)
            vals = [0.0, 0.0, 0.0]
            s = self.getshiftdir(1, nx)
            vals[0] = self.dotprod(-1, s, xp)
            s = self.getshiftdir(2, nx)
            vals[1] = self.dotprod(-1, s, xp)
            with torch.cuda.stream(self.stream):
                s = torch.zeros(n, dtype=torch.float64, device=self.dev)
            self.steporbit(1, nx, s)
            dt = self.pipe.tim.dt
            with torch.cuda.stream(self.stream):
                s = (s - nx) / dt
            vals[2] = self.dotprod(-1, s, xp)
            if cfg.mirrorsym or cfg.shiftrefl or self.T_fixed:
                xh = xp[:3].cpu().numpy()
                if cfg.mirrorsym or cfg.shiftrefl:
                    vals[0] = float(xh[0])
                if self.T_fixed:
                    vals[2] = float(xh[2])
            with torch.cuda.stream(self.stream):
                y[p * n:p * n + 3] = torch.tensor(vals, dtype=torch.float64, device=self.dev)
        if self.Ctnu:  # the parameter row (newton.f90:462)
            if self.ctstp is None:
                raise PipeflowError(L.PF_ERR_STATE, "multJ: call start_continuation first")
            v = self.dotprod_ms(1, self.ctstp, x)
            with torch.cuda.stream(self.stream):
                y.view(ms, n)[:, 3] = v
        return y

    def multA(self, x: torch.Tensor, y0: torch.Tensor, epsA: float) -> torch.Tensor:
        """newton.f90:837-860: the linearised time-T map about new_x applied
        to x (for the Arnoldi eigenvalue step), y0 = F(new_x)."""
        n = self.n
        with torch.cuda.stream(self.stream):
            y = x.clone()
        for p in range(self.ms):
            nx = self._part(self.new_x, p)
            eps = math.sqrt(self.dotprod(-1, y, y))
            if eps == 0.0:
                raise PipeflowError(L.PF_ERR_ARG, "multA: eps=0 (1)")
            eps = epsA * math.sqrt(self.dotprod(-1, nx, nx)) / eps
            if eps == 0.0:
                raise PipeflowError(L.PF_ERR_ARG, "multA: eps=0 (2)")
            with torch.cuda.stream(self.stream):
                y = nx + eps * y
                y[:8] = nx[:8]
            self.steporbit(self.ndts[p], y, y)
            with torch.cuda.stream(self.stream):
                y = (y - self._part(y0, p)) / eps
        return y

    # -- Floquet analysis of the converged orbit (newton.f90:868-979) ---------
    def get_eigen(self, m: int = 150, ncgd: int = 5, rel_err: float = 3e-6, gtol: float = 1e-3) -> dict:
        """getEigen without the output files: Arnoldi on the linearised
        period map about new_x (multA), started from new_x shifted by 0.3 of
        the periods in theta and z with (1 - r^2) r^2 added to ur and ut of
        modes (k,m) = (1,0) and (0,1).  Returns the Floquet multipliers, their
        magnitude and angle, the Floquet exponents and the eigenvectors
        scaled to the energy of the orbit (rows of a device tensor)."""
        n, ms = self.n, self.ms
        epsA = self.epsJ
        rerr = min(rel_err, gtol)
        t = float(self.new_x.view(ms, n)[:, 2].sum().item()) * self.scaleT
        with torch.cuda.stream(self.stream):
            y0 = torch.zeros_like(self.new_x)
        for p in range(ms):
            self.steporbit(self.ndts[p], self._part(self.new_x, p), self._part(y0, p))
        pp = self.pipe
        self.vec2rtz(self._part(self.new_x, 0))
        st, sz = 0.3 * 2.0 * math.pi, 0.3 * 2.0 * math.pi / pp.cfg.alpha
        for i in range(3):
            pp.var_coll_shift(st, sz, pp.vel_field(i), pp.vel_field(i))
        r2 = pp.mes_D()["r"] ** 2
        prof = (1.0 - r2) * r2
        for i in range(2):
            f = pp.vel_field(i)
            re, im = f.download()
            for nh in (1, 2 * pp.K - 1):  # var_harmonic(1,0), var_harmonic(0,1)
                if nh < pp.H:
                    re[:, nh] = prof
            f.upload(re, im)
        pp.vel_imposesym()
        with torch.cuda.stream(self.stream):
            sv = torch.zeros(n, dtype=torch.float64, device=self.dev)
        self.rtz2vec(sv)
        ar = Arnoldi(n, m, ncgd, lambda a, b: self.dotprod(-1, a, b), rerr, sv)
        status = "converged"
        with torch.cuda.stream(self.stream):
            while True:
                sv[:8] = 0.0
                ifail, sv = ar.step(sv)
                if ifail == -1:
                    break
                if ifail == 0:
                    sv = self.multA(sv, y0, epsA)
                elif ifail == 1:
                    status = "reached max iterations"
                    break
                else:
                    raise PipeflowError(L.PF_ERR_CONVERGE, "getEigen: arnoldi error (invariant subspace)")
        wr, wi = ar.wr2.copy(), ar.wi2.copy()
        mag, ang = np.hypot(wr, wi), np.arctan2(wi, wr)
        sr, si = logeig(wr, wi, t)
        out = dict(its=ar.k, epsA=epsA, T=t, status=status, multipliers=(wr, wi), magnitude=mag, angle=ang,
                   exponents=(sr, si), eigvecs=None)
        if ar.b is not None:
            # eigenvectors scaled to the energy of the orbit
            def energy(v):
                self.vec2rtz(v)
                return sum(pp.var_coll_norm(pp.vel_field(c))[0] for c in range(3))
            E0 = energy(self._part(self.new_x, 0))
            b = ar.b
            j = 0
            for i in range(ncgd):
                npart = 2 if wi[i] != 0.0 else 1
                E = sum(energy(b[j + q]) for q in range(npart))
                if E > 0.0:
                    with torch.cuda.stream(self.stream):
                        b[j:j + npart] *= math.sqrt(E0 / E)
                j += npart
            out["eigvecs"] = b
        self.stream.synchronize()
        return out

    # -- the main program's search (newton.f90:102-128) -----------------------
    def solve(self, m: int = 150, nits: int = 100, rel_err: float = 3e-6, delta: float = -1.0,
              mndl: float = 1e-7, mxdl: float = 1e7, gtol: float = 1e-3, d: float | None = None) -> NewtonResult:
        """newtonhook from new_x with the tolerances of newton_params.in
        (rel_err, del, mndl, mxdl relative to |x|, |x|^2 = d, by default
        that of new_x now)."""
        if d is None:
            d = self.dotprod_ms(-1, self.new_x, self.new_x)
        sd = math.sqrt(d)
        tol = rel_err * sd

        def f(v):
            return self.getrhs(v)

        def dp(a, b):
            return self.dotprod_ms(1, a, b)

        def sub():
            nx = math.sqrt(self.dotprod_ms(-1, self.new_x, self.new_x))
            hdr = self.new_x.view(self.ms, self.n)[:, :3].cpu().numpy() * self.scaleT
            self.history.append(dict(nits=self.new_nits, gits=self.new_gits, tol=self.new_tol,
                                     delta=self.new_del, rel=self.new_tol / nx, norm_x=nx,
                                     shifts=hdr.tolist()))

        with torch.cuda.stream(self.stream):
            res = newtonhook(f, self.multJ, dp, self.new_x, m, gtol, tol, delta * sd, mndl * sd, mxdl * sd, nits,
                             state=self, sub=sub)
        self.stream.synchronize()
        return res

    # -- parameter continuation (newton.f90:89-101, 102-170) -----------------
    def start_continuation(self, x_second: torch.Tensor) -> None:
        """The main program's set-up of a continuation (newton.f90:102-117):
        x_second is the second solution (what load_ms_states(1) reads from
        state10.cdf.in), its x[3] the parameter it was found at; the first
        guess becomes new_x + ctdp0 (x_second - new_x), and the parameter
        entries are scaled by ctpsc = parameter / |x|."""
        if not self.Ctnu:
            raise PipeflowError(L.PF_ERR_STATE, "start_continuation: the Orbit has no continuation")
        d = self.dotprod_ms(-1, self.new_x, self.new_x)
        self._d0 = d
        with torch.cuda.stream(self.stream):
            self.new_x, self.ctstp, self.ctx_, self.ctpsc = continuation_start(
                self.new_x, x_second.to(self.dev, torch.float64), self.n, self.ms, self.ctdp0, self._parameter(), d)

    def continue_step(self, res: NewtonResult) -> dict:
        """After a converged point (newton.f90:128-170): the record of
        newton.dat_ct (point, Newton its, Re, alpha, phase speed sum(x2)/sum(x3))
        and the next guess along the branch, with the step grown by 1.1,
        halved above ctntmx Newton iterations or doubled below ctntmn (and
        ndts and the times rescaled as there when T is fixed)."""
        n, ms = self.n, self.ms
        self.cti += 1
        hdr = self.new_x.view(ms, n)[:, :3].cpu().numpy()
        rec = dict(cti=self.cti, nits=res.nits, Re=self.pipe.cfg.Re, alpha=self.pipe.cfg.alpha,
                   c=float(hdr[:, 1].sum() / hdr[:, 2].sum()), info=res.info)
        with torch.cuda.stream(self.stream):
            self.new_x, self.ctstp, self.ctx_, self.ndts = continuation_next(
                self.new_x, self.ctx_, res.nits, res.gits, self.ctntmn, self.ctntmx, n, ms, self.ndts, self.T_fixed,
                self._m)
        return rec

    def continuation_run(self, npoints: int, m: int = 150, **solve_kwargs) -> list:
        """newtonhook at npoints successive points of the branch, stopping at
        the first that does not converge; returns their records."""
        if self.ctstp is None:
            raise PipeflowError(L.PF_ERR_STATE, "continuation_run: call start_continuation first")
        self._m = m
        out = []
        for _ in range(npoints):
            res = self.solve(m=m, d=self._d0, **solve_kwargs)
            rec = self.continue_step(res)
            out.append(rec)
            if res.info != 0:
                break
        return out

    def close(self) -> None:
        """Give the pipe back its own stream (the orbit's stream is freed
        with the Orbit, so the pipe must not keep using it)."""
        if self.ctx:
            self.stream.synchronize()
            _check(self.lib.pf_ctx_set_stream(self.ctx, None))
            self.ctx = None

    def __del__(self):
        try:
            if self.ctx and self.pipe.ctx:
                self.close()
        except Exception:
            pass
