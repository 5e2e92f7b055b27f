"""CPU FP64 oracle of the openpipeflow timestep hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module; only the
test-suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
use it, and only as the checker / the timed CPU restatement.

What it is
    A numpy/scipy restatement, in FP64, of the reference's (openpipeflow 1.12,
    Fortran 90) radial mesh, spectral field algebra, dealiased transforms,
    banded Helmholtz / pressure-Poisson solves, influence-matrix boundary
    correction and predictor-corrector step.  Every routine cites the reference
    file:line it restates.  The banded LU uses scipy's LAPACK ``dgbtrf`` /
    ``dgbtrs`` -- the same LAPACK routines the reference calls
    (timestep.f90:92,115,118).  The FFTs use numpy's pocketfft with FFTW's sign
    and scaling conventions (transform.fftw3.f90:35-147); the c2r transform
    discards the imaginary part of the DC bin exactly as FFTW's c2r does.

Parity status: **parity unpinned.**
    The reference ships no tests, no golden vectors and no state files, and it
    cannot be compiled in this image (no Fortran compiler, FFTW, LAPACK, netCDF
    or MPI).  The oracle is instead pinned by known-answer invariants derived
    from the reference code (tests/test_oracle.py): FD weights exact on
    polynomials (meshs.f90:149-159), FFT round trip (transform.fftw3.f90),
    Hagen-Poiseuille preservation (velocity.f90:338-361), no-slip and
    divergence-free after a step (velocity.f90:183-298), zero perturbation
    mean flux (velocity.f90:152-177) and the linear decay rate of a single
    Fourier mode (dense linearised one-step map).

Layout conventions (identical to the reference's types, variables.f90:32-44)
    coll : ``Coll`` with ``re``/``im`` arrays of shape (N, H); array index
           [n, nh] == Fortran ``%Re(n+1, nh)``.
    phys : array of shape (N, Th, Z) in C order == Fortran ``%Re(0:Z-1,0:Th-1,N)``.
    mesh : band array (2KL+1, N), ``M[KL+n-j, j] = A[n, j]`` (meshs.f90:13).
    lumesh: band array (3KL+1, N) in LAPACK dgbtrf storage plus 0-based pivots.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
from scipy.linalg import lapack

KL = 4                      # parameters.f90:43  i_KL
PI = 3.1415926535897931     # parameters.f90:51  d_PI


# ---------------------------------------------------------------------------
# configuration (parameters.f90:17-51)
# ---------------------------------------------------------------------------
@dataclass
class PipeConfig:
    N: int
    K: int
    M: int
    Mp: int = 1
    Re: float = 2500.0
    alpha: float = 1.25
    dt: float = 0.01            # d_timestep (>0 fixed; <0 adaptive)
    implicit: float = 0.51      # d_implicit
    dterr: float = 1e-5         # d_dterr
    courant: float = 0.5        # d_courant
    maxdt: float = 1e99         # d_maxdt
    const_flux: bool = True     # b_const_flux
    mirrorsym: bool = False
    shiftrefl: bool = False
    shiftrott: bool = False
    r: np.ndarray | None = None  # custom mesh (mesh.in, meshs.f90:76-88)

    @property
    def H(self) -> int:         # parameters.f90:48  i_H1+1
        return (2 * self.K - 1) * self.M - (self.K - 1)

    @property
    def Z(self) -> int:
        return 3 * self.K

    @property
    def Th(self) -> int:
        return 3 * self.M


def harmonics(K: int, M: int):
    """Mode enumeration of the serial ``_loop_km_begin`` (parallel.h:47-57)."""
    ks, ms = [], []
    for m in range(M):
        for k in range(-(K - 1), K):
            if m == 0 and k < 0:
                continue
            ks.append(k)
            ms.append(m)
    return np.array(ks, dtype=np.int64), np.array(ms, dtype=np.int64)


def mode_index(K: int, k: int, m: int) -> int:
    """var_harmonic (variables.f90:94-104), serial: nh = m*(2K-1)+k."""
    return m * (2 * K - 1) + k


# ---------------------------------------------------------------------------
# Chebyshev helpers (cheby.f:2-108) and FD weights (meshs.f90:200-225)
# ---------------------------------------------------------------------------
def _deriv2(a: np.ndarray) -> np.ndarray:
    """Coefficients of d/dx of a shifted-Chebyshev series on [0,1] (cheby.f:69-108)."""
    M = len(a)
    ax = np.zeros(M)
    if M == 1:
        return ax
    if M == 2:
        ax[0] = 2.0 * a[1]
        return ax
    if M == 3:
        ax[0] = 2.0 * a[1]
        ax[1] = 8.0 * a[2]
        return ax
    if M == 4:
        ax[0] = 2.0 * a[1] + 6.0 * a[3]
        ax[1] = 8.0 * a[2]
        ax[2] = 12.0 * a[3]
        return ax
    ax[M - 2] = -4.0 * (1.0 - M) * a[M - 1]
    ax[M - 3] = -4.0 * (2.0 - M) * a[M - 2]
    for J in range(M - 3, 1, -1):
        ax[J - 1] = 4.0 * J * a[J] + ax[J + 1]
    ax[0] = 2.0 * a[1] + ax[2] / 2.0
    return ax


def _eval2(a: np.ndarray, x) -> np.ndarray:
    """Clenshaw sum of a shifted-Chebyshev series at x (cheby.f:38-67)."""
    x = np.asarray(x, dtype=float)
    M = len(a)
    xa = 2.0 * x - 1.0
    xb = 2.0 * xa
    b = [np.zeros_like(xa) for _ in range(M + 3)]
    for J in range(M - 1, -1, -1):
        b[J + 1] = xb * b[J + 2] - b[J + 3] + a[J]
    return b[1] - xa * b[2]


def cheby(m: int, nd: int, x) -> np.ndarray:
    """nd-th derivative of T_m(2x-1) at points x (cheby.f:2-36)."""
    x = np.asarray(x, dtype=float)
    if m == 0:
        return np.ones_like(x) if nd == 0 else np.zeros_like(x)
    a = np.zeros(m + 1)
    a[m] = 1.0
    for _ in range(nd):
        a = _deriv2(a)
    return _eval2(a, x)


def mes_weights(i: int, x: np.ndarray, x0: float) -> np.ndarray:
    """Weights w with sum_j w_j f(x_j) = f^(i)(x0) (meshs.f90:200-225)."""
    n = len(x)
    xl = min(x0, float(np.min(x)))
    xr = max(x0, float(np.max(x)))
    x_ = (x - xl) / (xr - xl)
    x0_ = (x0 - xl) / (xr - xl)
    A = np.empty((n, n))
    d = np.empty(n)
    for j in range(n):
        A[:, j] = cheby(j, 0, x_)
        d[j] = cheby(j, i, np.array([x0_]))[0]
    Ainv = np.linalg.inv(A)        # mes_mat_invert: dgetrf+dgetri (meshs.f90:231-243)
    return (d @ Ainv) / ((xr - xl) ** i)


def default_mesh(N: int) -> np.ndarray:
    """Wall-clustered default radial mesh (meshs.f90:90-99)."""
    N_ = N + int(math.sqrt(float(N)))
    r = np.empty(N)
    for n in range(N_ - N + 1, N_ + 1):
        r[n - N_ + N - 1] = 0.5 * (1.0 + math.cos(PI * (N_ - n) / float(N_)))
    for _ in range(10):
        dr = 1.5 * r[0] - 0.5 * r[1]
        r = r * (1.0 + dr) - dr
    return r


@dataclass
class RadialMesh:
    """type rdom (meshs.f90:48-55) filled by mes_rdom_init (meshs.f90:110-194)."""
    N: int
    r: np.ndarray                 # r(:,1)
    rp: dict = field(default_factory=dict)   # r(:,j) for j=-3..3
    dr: list = field(default_factory=list)   # dr[i-1] = band (2KL+1, N) of d^i/dr^i
    radLap: np.ndarray | None = None
    dr0: np.ndarray | None = None  # (KL+1, KL+1): dr0[j, i] = weight of point j for i-th deriv at r=0
    dr1: np.ndarray | None = None  # (KL+1, KL+1): at r=1 using points N-KL..N
    intrdr: np.ndarray | None = None


def mes_rdom_init(r: np.ndarray) -> RadialMesh:
    N = len(r)
    D = RadialMesh(N=N, r=r.copy())
    D.rp = {1: r.copy(), 0: np.ones(N), 2: r * r, 3: r * r * r,
            -1: 1.0 / r, -2: 1.0 / (r * r), -3: 1.0 / (r * r * r)}
    r_ = np.concatenate([[0.0], r])          # r_(0:N), r_(0)=0
    D.dr = [np.zeros((2 * KL + 1, N)) for _ in range(KL)]
    for n in range(1, N + 1):
        l = max(1, n - KL)
        rr = min(n + KL, N)
        for i in range(1, KL + 1):
            w = mes_weights(i, r_[l:rr + 1], r_[n])
            for j in range(l, rr + 1):
                D.dr[i - 1][KL + n - j, j - 1] = w[j - l]
    D.dr0 = np.zeros((KL + 1, KL + 1))
    D.dr1 = np.zeros((KL + 1, KL + 1))
    for i in range(0, KL + 1):
        D.dr0[:, i] = mes_weights(i, r_[1:KL + 2], r_[0])
        D.dr1[:, i] = mes_weights(i, r_[N - KL:N + 1], r_[N])
    D.radLap = np.zeros((2 * KL + 1, N))
    for j in range(1, N + 1):
        l = max(1, j - KL)
        rr = min(j + KL, N)
        for n in range(l, rr + 1):
            D.radLap[KL + n - j, j - 1] = (D.dr[1][KL + n - j, j - 1]
                                           + D.dr[0][KL + n - j, j - 1] / r_[n])
    D.intrdr = np.zeros(N)
    A = np.zeros((2 * KL + 1, 2 * KL + 1))
    for n in range(1, N + 1):
        l = max(1, n - KL)
        rr = min(n + KL, N)
        nn = rr - l + 1
        for i in range(1, nn + 1):
            A[i - 1, :nn] = mes_weights(i - 1, r_[l:rr + 1], r_[n])
        c = 1.0
        e = 1.0
        for i in range(1, nn + 1):
            c = c * (r_[min(n + 1, N)] - r_[n]) / float(i)
            e = e * (r_[max(0, n - 1)] - r_[n]) / float(i)
            D.intrdr[l - 1:l - 1 + nn] = (D.intrdr[l - 1:l - 1 + nn]
                                          + 0.5 * (c - e) * A[i - 1, :nn] * r_[n])
    return D


# ---------------------------------------------------------------------------
# fields
# ---------------------------------------------------------------------------
class Coll:
    """type coll (variables.f90:37-40): re/im of shape (N, H)."""
    __slots__ = ("re", "im")

    def __init__(self, re, im):
        self.re = re
        self.im = im

    @staticmethod
    def zeros(N, H):
        return Coll(np.zeros((N, H)), np.zeros((N, H)))

    def copy(self):
        return Coll(self.re.copy(), self.im.copy())

    def as_complex(self):
        return self.re + 1j * self.im


def band_matvec(Aband_offdiag, diag, b: Coll, c: Coll | None):
    """d = A b + c, column-ordered accumulation of tim_meshmult / var_coll_meshmult
    (timestep.f90:130-154, variables.f90:378-402).  ``Aband_offdiag`` is a
    (2KL+1, N) band shared by all modes; ``diag`` (N, H) overrides its main
    diagonal per mode (or is None to use the band's own diagonal)."""
    N, H = b.re.shape
    re = np.zeros((N, H)) if c is None else c.re.copy()
    im = np.zeros((N, H)) if c is None else c.im.copy()
    for j in range(N):
        for n in range(max(0, j - KL), min(j + KL, N - 1) + 1):
            if n == j and diag is not None:
                a = diag[j]
            else:
                a = Aband_offdiag[KL + n - j, j]
            re[n] = re[n] + a * b.re[j]
            im[n] = im[n] + a * b.im[j]
    return Coll(re, im)


# ---------------------------------------------------------------------------
# the pipe: variables + transform + timestep + velocity modules
# ---------------------------------------------------------------------------
class Pipe:
    """Module state of variables/transform/timestep/velocity for one pipe."""

    def __init__(self, cfg: PipeConfig):
        self.cfg = cfg
        N, K, M, Mp = cfg.N, cfg.K, cfg.M, cfg.Mp
        self.N, self.K, self.M, self.Mp = N, K, M, Mp
        self.H = cfg.H
        r = default_mesh(N) if cfg.r is None else np.asarray(cfg.r, dtype=float)
        self.mes_D = mes_rdom_init(r)
        D = self.mes_D
        # var_precompute tables (variables.f90:79-86)
        self.kk, self.mm = harmonics(K, M)
        self.ad_m1r1 = np.empty((N, M))
        self.ad_m2r2 = np.empty((N, M))
        for n in range(M):
            self.ad_m1r1[:, n] = D.rp[-1] * Mp * n
            self.ad_m2r2[:, n] = D.rp[-2] * Mp * n * Mp * n
        self.ad_k1a1 = {k: cfg.alpha * k for k in range(-(K - 1), K)}
        self.m1r1_h = self.ad_m1r1[:, self.mm]                  # (N,H)
        self.k1a1_h = cfg.alpha * self.kk.astype(float)         # (H,)
        # tim_precompute (timestep.f90:29-40)
        self.tim_t = 0.0
        self.tim_dt = cfg.dt
        self.tim_dterr = 0.0
        self.tim_it = 0
        self.tim_step = 0
        self.tim_corr_dt = 0.0
        self.tim_cfl_dt = 0.0
        self.tim_cfl_dir = 0
        self.tim_new_dt = False
        self.tim_pcn = -1
        self._lasterr = 1e99
        self._newdt_i = 0
        self.failed = None
        # vel_precompute (velocity.f90:47-55)
        z = lambda: Coll.zeros(N, self.H)
        self.vel_ur, self.vel_ut, self.vel_uz = z(), z(), z()
        self.vel_Nr, self.vel_Nt, self.vel_Nz = z(), z(), z()
        self.ur_, self.ut_, self.uz_ = z(), z(), z()
        self.Nr_, self.Nt_, self.Nz_ = z(), z(), z()
        self.vel_nu = 1.0
        self.vel_Pr0 = 0.0
        self.vel_U = 1.0 - D.rp[2]
        self.vel_Up = -2.0 * D.rp[1]
        self.phys = {}
        self._LNp = None
        self._matrices_dt = None

    # ---------------- variables.f90 ----------------
    def var_coll_meshmult(self, A, inp: Coll) -> Coll:
        """variables.f90:378-402 (shared band matrix, e.g. mes_D%dr(1))."""
        return band_matvec(A, None, inp, None)

    def var_coll_curl(self, r: Coll, t: Coll, z: Coll):
        """variables.f90:408-436."""
        c1, c2, c3 = r.copy(), t.copy(), z.copy()
        m1r1, k1a1, rm1 = self.m1r1_h, self.k1a1_h, self.mes_D.rp[-1][:, None]
        orr = Coll(-c3.im * m1r1 + c2.im * k1a1, c3.re * m1r1 - c2.re * k1a1)
        ot = self.var_coll_meshmult(self.mes_D.dr[0], c3)
        ot = Coll(-c1.im * k1a1 - ot.re, c1.re * k1a1 - ot.im)
        oz = self.var_coll_meshmult(self.mes_D.dr[0], c2)
        oz = Coll(c2.re * rm1 + oz.re + c1.im * m1r1, c2.im * rm1 + oz.im - c1.re * m1r1)
        return orr, ot, oz

    def var_coll_grad(self, p: Coll):
        """variables.f90:442-459."""
        c1 = p.copy()
        r = self.var_coll_meshmult(self.mes_D.dr[0], c1)
        t = Coll(-c1.im * self.m1r1_h, c1.re * self.m1r1_h)
        z = Coll(-c1.im * self.k1a1_h, c1.re * self.k1a1_h)
        return r, t, z

    def var_coll_div(self, r: Coll, t: Coll, z: Coll) -> Coll:
        """variables.f90:465-481."""
        c1 = self.var_coll_meshmult(self.mes_D.dr[0], r)
        rm1 = self.mes_D.rp[-1][:, None]
        m1r1, k1a1 = self.m1r1_h, self.k1a1_h
        re = r.re * rm1 + c1.re - t.im * m1r1 - z.im * k1a1
        im = r.im * rm1 + c1.im + t.re * m1r1 + z.re * k1a1
        return Coll(re, im)

    def var_coll_shift(self, dt: float, dz: float, a: Coll) -> Coll:
        """variables.f90:487-528."""
        b = a.copy()
        if dz != 0.0:
            ang = dz * self.kk * self.cfg.alpha
            sk, ck = np.sin(ang), np.cos(ang)
            dRe = b.re.copy()
            b.re = dRe * ck + b.im * sk
            b.im = b.im * ck - dRe * sk
        if dt != 0.0:
            ang = dt * self.mm * self.Mp
            sm, cm = np.sin(ang), np.cos(ang)
            dRe = b.re.copy()
            b.re = dRe * cm + b.im * sm
            b.im = b.im * cm - dRe * sm
        return b

    def var_imposesym(self, i: int, r: Coll, t: Coll, z: Coll):
        """variables.f90:538-618 (serial).  Modifies r,t,z in place."""
        K = self.K
        if i in (1, 2):
            c = [Coll.zeros(self.N, self.H) for _ in range(3)]
            for nh in range(self.H):
                k, m = int(self.kk[nh]), int(self.mm[nh])
                nh_ = nh if m == 0 else mode_index(K, -k, m)
                b = -1.0
                a = 1.0
                if i == 2 and (k % 2) != 0:
                    a = -1.0
                if m == 0:
                    b = 1.0
                c[0].re[:, nh_] = r.re[:, nh] * a
                c[0].im[:, nh_] = r.im[:, nh] * a * b
                c[1].re[:, nh_] = -t.re[:, nh] * a
                c[1].im[:, nh_] = -t.im[:, nh] * a * b
                c[2].re[:, nh_] = z.re[:, nh] * a
                c[2].im[:, nh_] = z.im[:, nh] * a * b
            for f, cc in zip((r, t, z), c):
                f.re[:] = (f.re + cc.re) / 2.0
                f.im[:] = (f.im + cc.im) / 2.0
        if i == 3:
            odd = ((self.kk + self.mm) % 2) != 0
            for f in (r, t, z):
                f.re[:, odd] = 0.0
                f.im[:, odd] = 0.0
        r.re[:, 0] = 0.0
        r.im[:, 0] = 0.0
        t.im[:, 0] = 0.0
        z.im[:, 0] = 0.0

    def var_coll_norm(self, a: Coll):
        """(1/2)int a.a dV per mode (variables.f90:718-751) -> E, Ek, Em."""
        w = 4.0 * PI * PI / self.cfg.alpha
        f = w * (a.re * a.re + a.im * a.im)
        b = self.mes_D.intrdr @ f                      # dot_product(f, intrdr) per mode
        b = b.copy()
        b[0] = 0.5 * b[0]                              # k==0 .and. m==0
        Ek = np.zeros(self.K)
        Em = np.zeros(self.M)
        np.add.at(Em, self.mm, b)
        np.add.at(Ek, np.abs(self.kk), b)
        return float(np.sum(Em)), Ek, Em

    # ---------------- transform.fftw3.f90 ----------------
    def tra_spec2phys(self, c: Coll) -> np.ndarray:
        """coll -> phys: var_coll2spec (variables.f90:184-197) + tra_spec2phys
        (transform.fftw3.f90:65-102).  Returns (N, Th, Z)."""
        N, K, M = self.N, self.K, self.M
        Z, Th = 3 * K, 3 * M
        s = c.re + 1j * c.im
        X = np.zeros((N, M, Z), dtype=complex)
        X[:, 0, 0:K] = s[:, 0:K]
        X[:, 0, 2 * K + 1:] = np.conj(s[:, K - 1:0:-1])
        for m in range(1, M):
            base = m * (2 * K - 1)
            X[:, m, 0:K] = s[:, base:base + K]
            X[:, m, 2 * K + 1:] = s[:, base - (K - 1):base]
        Y = np.fft.ifft(X, axis=2, norm="forward")            # c2c, sign +1, unscaled
        Xs = np.zeros((N, Z, Th // 2 + 1), dtype=complex)
        Xs[:, :, 0:M] = Y.transpose(0, 2, 1)
        p = np.fft.irfft(Xs, n=Th, axis=2, norm="forward")    # c2r, unscaled
        return np.ascontiguousarray(p.transpose(0, 2, 1))

    def tra_phys2spec(self, p: np.ndarray) -> Coll:
        """phys -> coll: tra_phys2spec (transform.fftw3.f90:108-147) +
        var_spec2coll (variables.f90:281-294)."""
        N, K, M = self.N, self.K, self.M
        Z, Th = 3 * K, 3 * M
        scale_ = 1.0 / float(Z * Th)
        Ys = scale_ * p                                       # (N, Th, Z)
        Xs = np.fft.rfft(Ys.transpose(0, 2, 1), axis=2)       # r2c, sign -1
        Y = Xs[:, :, 0:M].transpose(0, 2, 1)                  # (N, M, Z)
        X = np.fft.fft(Y, axis=2)                             # c2c, sign -1
        s = np.zeros((N, self.H), dtype=complex)
        s[:, 0:K] = X[:, 0, 0:K]
        for m in range(1, M):
            base = m * (2 * K - 1)
            s[:, base:base + K] = X[:, m, 0:K]
            s[:, base - (K - 1):base] = X[:, m, 2 * K + 1:]
        return Coll(np.ascontiguousarray(s.real), np.ascontiguousarray(s.imag))

    # ---------------- timestep.f90 ----------------
    def _dvec(self, PM: int):
        """The diagonal term d(n, nh) of tim_mesh_init / tim_lumesh_init
        (timestep.f90:54-55, 76-77)."""
        r2 = self.mes_D.rp[-2][:, None]
        Mp = self.Mp
        m = self.mm[None, :].astype(float)
        k = self.kk[None, :].astype(float)
        al = self.cfg.alpha
        d = -(r2 * Mp * m * Mp * m) - al * k * al * k
        if PM != 0:
            d = d - r2 - 2.0 * PM * Mp * m * r2
        return d

    def tim_mesh_init(self, PM: int, c1: float, c2: float):
        """A = c1 I + c2 Lap (timestep.f90:46-60).  Returned as (offdiag band,
        per-mode diagonal) -- the same numbers as the per-mode band arrays."""
        off = c2 * self.mes_D.radLap
        diag = (c2 * self.mes_D.radLap[KL][:, None] + c2 * self._dvec(PM)) + c1
        return (off, diag)

    def tim_lumesh_init(self, PM: int, BC: int, c1: float, c2: float):
        """Banded matrix with axis-parity and wall rows, LU-factored per mode
        by LAPACK dgbtrf (timestep.f90:67-96)."""
        N, H, Mp = self.N, self.H, self.Mp
        D = self.mes_D
        d = self._dvec(PM)
        AB = np.zeros((H, 3 * KL + 1, N))
        AB[:, KL:, :] = c2 * D.radLap[None, :, :]
        AB[:, 2 * KL, :] = AB[:, 2 * KL, :] + (c2 * d).T + c1
        ipiv = np.zeros((H, N), dtype=np.int32)
        for nh in range(H):
            k, m = int(self.kk[nh]), int(self.mm[nh])
            S = (m * Mp + abs(PM)) % 2
            for j in range(1, KL + 2):
                AB[nh, 2 * KL + 1 - j, j - 1] = D.dr0[j - 1, 1 - S]
            for j in range(N - KL, N + 1):
                AB[nh, 2 * KL + N - j, j - 1] = D.dr1[KL - N + j, BC]
            if BC == 1 and k == 0 and m == 0:
                continue
            lu, piv, info = lapack.dgbtrf(AB[nh], KL, KL)
            if info != 0:
                raise RuntimeError("tim_lumesh_init")
            AB[nh] = lu
            ipiv[nh] = piv
        return (AB, ipiv)

    def tim_lumesh_invert(self, BC: int, A, b: Coll) -> None:
        """Solve A x = b per mode with dgbtrs, Re and Im as two right-hand
        sides (timestep.f90:102-123).  In place."""
        AB, ipiv = A
        for nh in range(self.H):
            if BC == 1 and self.kk[nh] == 0 and self.mm[nh] == 0:
                b.re[:, nh] = 0.0
                b.im[:, nh] = 0.0
                continue
            rhs = np.stack([b.re[:, nh], b.im[:, nh]], axis=1)
            x, info = lapack.dgbtrs(AB[nh], KL, KL, rhs, ipiv[nh])
            if info != 0:
                raise RuntimeError("mes_lumesh_invert")
            b.re[:, nh] = x[:, 0]
            b.im[:, nh] = x[:, 1]

    def tim_meshmult(self, A, b: Coll, c: Coll) -> Coll:
        """d = A b + c (timestep.f90:130-154)."""
        off, diag = A
        return band_matvec(off, diag, b, c)

    @staticmethod
    def tim_zerobc(a: Coll) -> None:
        """timestep.f90:160-169."""
        a.re[0, :] = 0.0
        a.re[-1, :] = 0.0
        a.im[0, :] = 0.0
        a.im[-1, :] = 0.0

    def tim_nlincorr(self, N_: Coll, Nn: Coll) -> None:
        """N = c N + (1-c) N_ (timestep.f90:174-184).  In place on Nn."""
        d1 = self.cfg.implicit
        d2 = 1.0 - self.cfg.implicit
        Nn.re[:] = d1 * Nn.re + d2 * N_.re
        Nn.im[:] = d1 * Nn.im + d2 * N_.im

    def tim_measurecorr(self, c1: Coll, c2: Coll, c3: Coll) -> None:
        """max |correction|^2 over modes and points (timestep.f90:190-207)."""
        dterr = 0.0
        for c in (c1, c2, c3):
            dterr = max(dterr, float(np.max(c.re * c.re + c.im * c.im)))
        self.tim_dterr = max(self.tim_dterr, math.sqrt(dterr))

    def tim_check_cgce(self) -> None:
        """Corrector control (timestep.f90:214-253).  Failures set
        ``self.failed`` instead of forcing the step counter."""
        cfg = self.cfg
        if self.tim_it == 1:
            # d_dterr/0 is +Inf in the reference's IEEE arithmetic
            self.tim_corr_dt = (self.tim_dt * math.sqrt(cfg.dterr / self.tim_dterr)
                                if self.tim_dterr > 0 else math.inf)
            self._lasterr = 1e99
        if self.tim_dt < 1e-9 and self.tim_step > 30:
            self.failed = "tim_check_cgce: dt --> 0 !!!?"
            self.tim_it = 0
        elif self.tim_it == self.tim_pcn:
            self.tim_it = 0
        elif self.tim_it > 10:
            self.failed = "tim_check_cgce: too many its!!!"
            self.tim_it = 0
        elif self.tim_dterr > self._lasterr:
            if self.tim_dterr > 2.0 * cfg.dterr:
                self.failed = "tim_check_cgce: increasing error!!!"
            if self.tim_dterr < 2.0 * cfg.dterr:
                self.tim_corr_dt = self.tim_dt / (10.0 * cfg.courant)
            self.tim_it = 0
        elif self.tim_dterr > cfg.dterr:
            self._lasterr = self.tim_dterr
            self.tim_it = self.tim_it + 1
        else:
            self.tim_it = 0
        self.tim_dterr = 0.0

    def tim_new_tstep(self) -> None:
        """Adaptive dt (timestep.f90:259-278)."""
        cfg = self.cfg
        dt = min(self.tim_dt * 1.11, cfg.maxdt)
        if self.tim_step == 0 and self.tim_corr_dt == 0.0:
            dt = min(dt, self.tim_cfl_dt * 0.1)
        if self.tim_cfl_dt > 0.0:
            dt = min(dt, self.tim_cfl_dt * cfg.courant)
        if self.tim_corr_dt > 0.0:
            dt = min(dt, self.tim_corr_dt * 0.95)
        self._newdt_i -= 1
        i = self._newdt_i
        self.tim_new_dt = (dt < self.tim_dt * 0.95
                           or (dt > self.tim_dt * 1.10 and i < 0)
                           or (dt == cfg.maxdt and self.tim_dt < dt and i < 0))
        if self.tim_new_dt:
            if dt >= self.tim_dt:
                self._newdt_i = 99
            self.tim_dt = dt

    # ---------------- velocity.f90 ----------------
    def vel_imposesym(self) -> None:
        """velocity.f90:61-74."""
        cfg = self.cfg
        self.var_imposesym(0, self.vel_ur, self.vel_ut, self.vel_uz)
        if cfg.mirrorsym:
            self.var_imposesym(1, self.vel_ur, self.vel_ut, self.vel_uz)
        if cfg.shiftrefl:
            self.var_imposesym(2, self.vel_ur, self.vel_ut, self.vel_uz)
        if cfg.shiftrott:
            self.var_imposesym(3, self.vel_ur, self.vel_ut, self.vel_uz)

    @staticmethod
    def vel_rt2pm(r: Coll, t: Coll):
        """u+- = u_r +- i u_theta (velocity.f90:80-95)."""
        up = Coll(r.re - t.im, r.im + t.re)
        um = Coll(r.re + t.im, r.im - t.re)
        return up, um

    @staticmethod
    def vel_pm2rt(up: Coll, um: Coll):
        """velocity.f90:98-114."""
        r = Coll(0.5 * (up.re + um.re), 0.5 * (up.im + um.im))
        t = Coll(0.5 * (up.im - um.im), -0.5 * (up.re - um.re))
        return r, t

    def vel_matrices(self) -> None:
        """velocity.f90:120-146."""
        cfg = self.cfg
        if self._LNp is None:
            self._LNp = self.tim_lumesh_init(0, 1, 0.0, 1.0)
        d1 = 1.0 / self.tim_dt
        d2 = -cfg.implicit * self.vel_nu / cfg.Re
        self.LDp = self.tim_lumesh_init(1, 0, d1, d2)
        self.LDm = self.tim_lumesh_init(-1, 0, d1, d2)
        self.LDz = self.tim_lumesh_init(0, 0, d1, d2)
        d1 = 1.0 / self.tim_dt
        d2 = (1.0 - cfg.implicit) * self.vel_nu / cfg.Re
        self.Ltp = self.tim_mesh_init(1, d1, d2)
        self.Ltm = self.tim_mesh_init(-1, d1, d2)
        self.Ltz = self.tim_mesh_init(0, d1, d2)
        self.vel_adjustFlux(0)
        self.vel_adjPPE(0)
        self._matrices_dt = self.tim_dt

    @property
    def LNp(self):
        return self._LNp

    def vel_adjustFlux(self, F: int) -> None:
        """Constant mass flux (velocity.f90:152-177)."""
        if not self.cfg.const_flux:
            return
        D = self.mes_D
        N = self.N
        if F == 0:
            Ui = np.ones(N)
            Ui[0] = 0.0
            Ui[N - 1] = 0.0
            AB, ipiv = self.LDz
            x, info = lapack.dgbtrs(AB[0], KL, KL, Ui[:, None].copy(), ipiv[0])
            if info != 0:
                raise RuntimeError("vel_adjustFlux: err 1")
            self._Ui = x[:, 0].copy()
            self._flux_d1 = 2.0 * float(np.dot(self._Ui, D.intrdr))
            if self._flux_d1 == 0.0:
                raise RuntimeError("vel_adjustFlux: err 2")
        elif F == 1:
            d2 = 2.0 * float(np.dot(self.vel_uz.re[:, 0], D.intrdr))
            d3 = -d2 / self._flux_d1
            self.vel_uz.re[:, 0] = self.vel_uz.re[:, 0] + d3 * self._Ui
            self.vel_Pr0 = self.vel_Pr0 + d3 * self.cfg.Re / 4.0

    def vel_evalBC(self, up: Coll, um: Coll, uz: Coll):
        """Boundary residuals at r=1 (velocity.f90:262-298) -> BRe, BIm (4, H)."""
        D = self.mes_D
        N = self.N
        n = N - 1
        m_ = (self.mm * self.Mp).astype(float)
        a_ = self.cfg.alpha * self.kk.astype(float)
        urRe = 0.5 * (up.re[n] + um.re[n])
        urIm = 0.5 * (up.im[n] + um.im[n])
        utRe = 0.5 * (up.im[n] - um.im[n])
        utIm = -0.5 * (up.re[n] - um.re[n])
        uzRe = uz.re[n]
        uzIm = uz.im[n]
        drRe = 0.5 * (D.dr1[:, 1] @ (up.re[N - KL - 1:N] + um.re[N - KL - 1:N]))
        drIm = 0.5 * (D.dr1[:, 1] @ (up.im[N - KL - 1:N] + um.im[N - KL - 1:N]))
        BRe = np.zeros((4, self.H))
        BIm = np.zeros((4, self.H))
        BRe[0] = up.re[n]
        BIm[0] = up.im[n]
        BRe[1] = um.re[n]
        BIm[1] = um.im[n]
        BRe[2] = -uzIm
        BIm[2] = uzRe
        d = D.rp[-1][n]
        BRe[3] = urRe * d + drRe - d * m_ * utIm - a_ * uzIm
        BIm[3] = urIm * d + drIm + d * m_ * utRe + a_ * uzRe
        BRe[:, 0] = 0.0
        BIm[:, 0] = 0.0
        return BRe, BIm

    def vel_adjPPE(self, F: int) -> None:
        """Pressure projection and influence-matrix correction
        (velocity.f90:183-259)."""
        N, H = self.N, self.H
        if F == 0:
            A = np.zeros((H, 4, 4))
            U = np.zeros((6, N, H))
            for j in range(1, 5):
                c1, c2, c3 = Coll.zeros(N, H), Coll.zeros(N, H), Coll.zeros(N, H)
                if j == 1:
                    c1.re[N - 1, :] = 1.0
                    self.tim_lumesh_invert(0, self.LDp, c1)
                    U[0] = c1.re
                elif j == 2:
                    c2.re[N - 1, :] = 1.0
                    self.tim_lumesh_invert(0, self.LDm, c2)
                    U[1] = c2.re
                elif j == 3:
                    c3.im[N - 1, :] = 1.0
                    self.tim_lumesh_invert(0, self.LDz, c3)
                    U[2] = c3.im
                else:
                    c1.re[N - 1, :] = -1.0
                    self.tim_lumesh_invert(1, self.LNp, c1)
                    c1, c2, c3 = self.var_coll_grad(c1)
                    c1, c2 = self.vel_rt2pm(c1, c2)
                    U[3] = c1.re
                    U[4] = c2.re
                    U[5] = c3.im
                BRe, BIm = self.vel_evalBC(c1, c2, c3)
                A[:, :, j - 1] = BRe.T
            for nh in range(1, H):
                A[nh] = np.linalg.inv(A[nh])
            self._A = A
            self._U = U
        elif F == 1:
            c1, c2 = self.vel_pm2rt(self.vel_ur, self.vel_ut)
            c1 = self.var_coll_div(c1, c2, self.vel_uz)
            self.tim_zerobc(c1)
            self.tim_lumesh_invert(1, self.LNp, c1)
            c1, c2, c3 = self.var_coll_grad(c1)
            c1, c2 = self.vel_rt2pm(c1, c2)
            for f, c in ((self.vel_ur, c1), (self.vel_ut, c2), (self.vel_uz, c3)):
                f.re = f.re - c.re
                f.im = f.im - c.im
        elif F == 2:
            BRe, BIm = self.vel_evalBC(self.vel_ur, self.vel_ut, self.vel_uz)
            A, U = self._A, self._U
            aR = -np.einsum("hij,jh->ih", A, BRe)
            aI = -np.einsum("hij,jh->ih", A, BIm)
            aR[:, 0] = 0.0
            aI[:, 0] = 0.0
            ur, ut, uz = self.vel_ur, self.vel_ut, self.vel_uz
            ur.re = ur.re + aR[0] * U[0]
            ur.im = ur.im + aI[0] * U[0]
            ut.re = ut.re + aR[1] * U[1]
            ut.im = ut.im + aI[1] * U[1]
            uz.re = uz.re - aI[2] * U[2]
            uz.im = uz.im + aR[2] * U[2]
            ur.re = ur.re + aR[3] * U[3]
            ur.im = ur.im + aI[3] * U[3]
            ut.re = ut.re + aR[3] * U[4]
            ut.im = ut.im + aI[3] * U[4]
            uz.re = uz.re - aI[3] * U[5]
            uz.im = uz.im + aR[3] * U[5]

    def vel_transform(self) -> None:
        """u and curl(u) in physical space (velocity.f90:304-317)."""
        P = self.phys
        P["r"] = self.tra_spec2phys(self.vel_ur)
        P["t"] = self.tra_spec2phys(self.vel_ut)
        P["z"] = self.tra_spec2phys(self.vel_uz)
        c1, c2, c3 = self.var_coll_curl(self.vel_ur, self.vel_ut, self.vel_uz)
        P["curlr"] = self.tra_spec2phys(c1)
        P["curlt"] = self.tra_spec2phys(c2)
        P["curlz"] = self.tra_spec2phys(c3)

    def vel_nonlinear(self) -> None:
        """u x curl(u), forward transforms, background-flow terms
        (velocity.f90:323-335)."""
        P = self.phys
        p = P["t"] * P["curlz"] - P["z"] * P["curlt"]
        self.vel_Nr = self.tra_phys2spec(p)
        p = P["z"] * P["curlr"] - P["r"] * P["curlz"]
        self.vel_Nt = self.tra_phys2spec(p)
        p = P["r"] * P["curlt"] - P["t"] * P["curlr"]
        self.vel_Nz = self.tra_phys2spec(p)
        self.vel_addHPF()

    def vel_addHPF(self) -> None:
        """Hagen-Poiseuille advection and constant-flux pressure
        (velocity.f90:338-361)."""
        b = (-self.vel_Up)[:, None]
        a = self.k1a1_h[None, :] * self.vel_U[:, None]
        Nr, Nt, Nz = self.vel_Nr, self.vel_Nt, self.vel_Nz
        ur, ut, uz = self.vel_ur, self.vel_ut, self.vel_uz
        Nr.re = Nr.re + a * ur.im
        Nr.im = Nr.im - a * ur.re
        Nt.re = Nt.re + a * ut.im
        Nt.im = Nt.im - a * ut.re
        Nz.re = Nz.re + a * uz.im + b * ur.re
        Nz.im = Nz.im - a * uz.re + b * ur.im
        if self.cfg.const_flux:
            D = self.mes_D
            self.vel_Pr0 = float(np.dot(uz.re[self.N - KL - 1:, 0], D.dr1[:, 1]))
            self.vel_Pr0 = self.vel_Pr0 / (-2.0)
            Nz.re[:, 0] = Nz.re[:, 0] + 4.0 * self.vel_Pr0 / self.cfg.Re

    def vel_step(self) -> None:
        """Advance one (predictor or corrector) step (velocity.f90:367-394)."""
        c1, c2 = self.vel_rt2pm(self.vel_Nr, self.vel_Nt)
        self.vel_ur, self.vel_ut = self.vel_rt2pm(self.ur_, self.ut_)
        self.vel_ur = self.tim_meshmult(self.Ltp, self.vel_ur, c1)
        self.vel_ut = self.tim_meshmult(self.Ltm, self.vel_ut, c2)
        self.vel_uz = self.tim_meshmult(self.Ltz, self.uz_, self.vel_Nz)
        self.vel_adjPPE(1)
        for f in (self.vel_ur, self.vel_ut, self.vel_uz):
            self.tim_zerobc(f)
        self.tim_lumesh_invert(0, self.LDp, self.vel_ur)
        self.tim_lumesh_invert(0, self.LDm, self.vel_ut)
        self.tim_lumesh_invert(0, self.LDz, self.vel_uz)
        self.vel_adjPPE(2)
        self.vel_ur, self.vel_ut = self.vel_pm2rt(self.vel_ur, self.vel_ut)
        self.vel_adjustFlux(1)
        self.vel_ur.re[:, 0] = 0.0
        self.vel_ur.im[:, 0] = 0.0
        self.vel_ut.im[:, 0] = 0.0
        self.vel_uz.im[:, 0] = 0.0

    def vel_predictor(self) -> None:
        """velocity.f90:400-410."""
        self.ur_, self.ut_, self.uz_ = self.vel_ur.copy(), self.vel_ut.copy(), self.vel_uz.copy()
        self.Nr_, self.Nt_, self.Nz_ = self.vel_Nr.copy(), self.vel_Nt.copy(), self.vel_Nz.copy()
        self.vel_step()

    def vel_corrector(self) -> None:
        """velocity.f90:416-432."""
        r, t, z = self.vel_ur.copy(), self.vel_ut.copy(), self.vel_uz.copy()
        self.tim_nlincorr(self.Nr_, self.vel_Nr)
        self.tim_nlincorr(self.Nt_, self.vel_Nt)
        self.tim_nlincorr(self.Nz_, self.vel_Nz)
        self.vel_step()
        for a, f in ((r, self.vel_ur), (t, self.vel_ut), (z, self.vel_uz)):
            a.re = a.re - f.re
            a.im = a.im - f.im
        self.tim_measurecorr(r, t, z)

    def vel_maxtstep(self) -> None:
        """CFL limit from the physical velocity (velocity.f90:438-481);
        needs ``vel_transform`` to have filled the physical fields."""
        P = self.phys
        r_ = self.mes_D.r
        N = self.N
        dt = [1e99, 1e99, 1e99]
        for n in range(N):
            if n == 0:
                d = r_[1] - r_[0]
            elif n == N - 1:
                d = r_[N - 1] - r_[N - 2]
            else:
                d = min(r_[n] - r_[n - 1], r_[n + 1] - r_[n])
            mx = float(np.max(np.abs(P["r"][n])))
            if mx != 0.0:
                dt[0] = min(dt[0], d / mx)
            d = 2.0 * PI / float(self.cfg.Th * self.Mp)
            mx = float(np.max(np.abs(P["t"][n])))
            if mx != 0.0:
                dt[1] = min(dt[1], d / mx)
            d = 2.0 * PI / (self.cfg.alpha * self.cfg.Z)
            mx = float(np.max(np.abs(P["z"][n] + (1.0 - r_[n] * r_[n]))))
            if mx != 0.0:
                dt[2] = min(dt[2], d / mx)
        self.tim_cfl_dt = min(dt)
        for i in range(3):
            if self.tim_cfl_dt == dt[i]:
                self.tim_cfl_dir = i + 1
        return tuple(dt)

    # ---------------- drivers ----------------
    def timestep(self, orbit: bool = False) -> int:
        """One pass of the main.f90 loop body (main.f90:20-44) -- corrector
        iterated to convergence -- or, with ``orbit=True``, of steporbit's
        body with exactly one corrector (newton.f90:740-762).  Returns the
        number of corrector iterations taken."""
        cfg = self.cfg
        self.vel_imposesym()
        self.vel_transform()
        self.vel_nonlinear()
        if cfg.dt < 0.0 and not orbit:
            self.vel_maxtstep()
            self.tim_new_tstep()
            if self.tim_new_dt:
                self.vel_matrices()
        self.vel_predictor()
        ncorr = 0
        if orbit:
            self.vel_transform()
            self.vel_nonlinear()
            self.vel_corrector()
            self.vel_imposesym()
            self.tim_it = 1
            self.tim_check_cgce()
            ncorr = 1
        else:
            self.tim_it = 1
            while self.tim_it != 0:
                self.vel_transform()
                self.vel_nonlinear()
                self.vel_corrector()
                self.tim_check_cgce()
                ncorr += 1
        self.tim_t = self.tim_t + self.tim_dt
        self.tim_step = self.tim_step + 1
        return ncorr

    def state(self):
        return (self.vel_ur.copy(), self.vel_ut.copy(), self.vel_uz.copy())

    def set_state(self, ur: Coll, ut: Coll, uz: Coll) -> None:
        self.vel_ur, self.vel_ut, self.vel_uz = ur.copy(), ut.copy(), uz.copy()

    def energy(self) -> float:
        """Perturbation kinetic energy as io_write_energy sums it (io.f90:501-514)."""
        return sum(self.var_coll_norm(f)[0] for f in (self.vel_ur, self.vel_ut, self.vel_uz))

    def friction(self):
        """Ub, Uc, u_tau of io_write_friction (io.f90:627-639)."""
        D = self.mes_D
        uz0 = self.vel_uz.re[:, 0]
        Ub = 0.5 + 2.0 * float(np.dot(uz0, D.intrdr))
        if self.cfg.const_flux:
            Ub = self.vel_Pr0
        Uc = 1.0 + float(np.dot(uz0[0:1 + KL], D.dr0[:, 0]))
        Ufr = float(np.dot(uz0[self.N - KL - 1:], D.dr1[:, 1]))
        Ufr = math.sqrt(abs((Ufr - 2.0) / self.cfg.Re))
        return Ub, Uc, Ufr


# ---------------------------------------------------------------------------
# seeded initial condition (the reference's ic.f90 is an empty template)
# ---------------------------------------------------------------------------
def vector_potential(pipe: Pipe, seed: int):
    """Seeded solenoidal-perturbation potential: complex Gaussian coefficient
    per (component, mode) from numpy default_rng(seed), drawn as one
    (3, 2, H) standard-normal block (component, re/im, mode), scaled by
    exp(-(k^2+m^2)/16) and given the radial envelope r^(|m Mp|+1) (1-r^2)^2."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((3, 2, pipe.H))
    k = pipe.kk.astype(float)
    m = pipe.mm.astype(float)
    amp = np.exp(-(k * k + m * m) / 16.0)
    r = pipe.mes_D.r[:, None]
    am = np.abs(pipe.mm * pipe.Mp)[None, :]
    prof_rt = r ** (am + 1) * (1.0 - r * r) ** 2
    prof_z = r ** (am + 2) * (1.0 - r * r) ** 2
    profs = (prof_rt, prof_rt, prof_z)
    return [Coll(g[c, 0][None, :] * amp[None, :] * profs[c],
                 g[c, 1][None, :] * amp[None, :] * profs[c]) for c in range(3)]


def seeded_state(pipe: Pipe, seed: int, energy_frac: float):
    """u' = curl(A), imposesym(0), scaled so that the perturbation energy
    equals energy_frac * E_lam with E_lam = pi^2/(3 alpha) (io.f90:548)."""
    A = vector_potential(pipe, seed)
    ur, ut, uz = pipe.var_coll_curl(*A)
    pipe.var_imposesym(0, ur, ut, uz)
    E = sum(pipe.var_coll_norm(f)[0] for f in (ur, ut, uz))
    E_lam = PI * PI / (3.0 * pipe.cfg.alpha)
    s = math.sqrt(energy_frac * E_lam / E)
    out = []
    for f in (ur, ut, uz):
        out.append(Coll(f.re * s, f.im * s))
    return out


def rel_l2(a_fields, b_fields) -> float:
    """Relative L2 distance over a list of Coll fields."""
    num = 0.0
    den = 0.0
    for a, b in zip(a_fields, b_fields):
        num += float(np.sum((a.re - b.re) ** 2 + (a.im - b.im) ** 2))
        den += float(np.sum(b.re ** 2 + b.im ** 2))
    return math.sqrt(num / den) if den > 0 else math.sqrt(num)
