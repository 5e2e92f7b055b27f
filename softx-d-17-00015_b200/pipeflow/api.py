"""Python mirror of the reference's Fortran module API for the timestep path.

One ``Pipe`` holds what the reference keeps in module state for one run
(parameters, mes_D, var_H, tim_*, vel_*, the LU factor sets).  Method names
are the reference's routine names (variables.f90, transform.fftw3.f90,
timestep.f90, velocity.f90) and keep their argument meaning; every non-zero
status of the C ABI raises ``PipeflowError`` with the library's message --
the reference's ``stop 'msg'``.

Host arrays use the reference's indexing: a coll component is a pair of
float64 arrays (re, im) of shape (N, H) indexed [n, nh] (== %Re(n+1, nh));
a phys field is a float64 array of shape (N, Th, Z) (== %Re(z, t, n+1)).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L


class PipeflowError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


def _check(status: int) -> int:
    if status != L.PF_OK:
        msg = L.load().pf_last_error()
        raise PipeflowError(status, msg.decode() if msg else "")
    return status


def _dp(a: np.ndarray):
    return a.ctypes.data_as(L.DP)


@dataclass
class PipeConfig:
    """parameters.f90:15-51 as a runtime record."""
    N: int
    K: int
    M: int
    Mp: int = 1
    Re: float = 2500.0
    alpha: float = 1.25
    dt: float = 0.01
    implicit: float = 0.51
    dterr: float = 1e-5
    courant: float = 0.5
    maxdt: float = 1e99
    const_flux: bool = True
    mirrorsym: bool = False
    shiftrefl: bool = False
    shiftrott: bool = False
    r: np.ndarray | None = None
    precision: int = L.PF_PREC_FP64

    @property
    def H(self) -> int:
        return (2 * self.K - 1) * self.M - (self.K - 1)

    @property
    def Z(self) -> int:
        return 3 * self.K

    @property
    def Th(self) -> int:
        return 3 * self.M


def cfg_struct(cfg: PipeConfig) -> L.pf_config:
    """The C ABI configuration record of a PipeConfig (keeps a custom mesh alive)."""
    c = L.pf_config()
    for f in ("N", "K", "M", "Mp", "Re", "alpha", "dt", "implicit", "dterr", "courant", "maxdt"):
        setattr(c, f, getattr(cfg, f))
    c.const_flux = int(cfg.const_flux)
    c.mirrorsym = int(cfg.mirrorsym)
    c.shiftrefl = int(cfg.shiftrefl)
    c.shiftrott = int(cfg.shiftrott)
    c.precision = int(cfg.precision)
    c._r = None
    if cfg.r is not None:
        c._r = np.ascontiguousarray(cfg.r, dtype=np.float64)
        c.r = _dp(c._r)
    return c


class Coll:
    """A device `type (coll)` field (variables.f90:37-40)."""

    def __init__(self, pipe: "Pipe", handle=None, owned: bool = True):
        self.pipe = pipe
        self.owned = owned
        if handle is None:
            h = C.c_void_p()
            _check(pipe.lib.pf_coll_create(pipe.ctx, C.byref(h)))
            handle = h
        self.h = handle

    def upload(self, re: np.ndarray, im: np.ndarray) -> "Coll":
        N, H = self.pipe.N, self.pipe.H
        re = np.ascontiguousarray(np.asarray(re, dtype=np.float64).reshape(N, H).T)
        im = np.ascontiguousarray(np.asarray(im, dtype=np.float64).reshape(N, H).T)
        _check(self.pipe.lib.pf_coll_upload(self.h, _dp(re), _dp(im)))
        return self

    def download(self):
        N, H = self.pipe.N, self.pipe.H
        re = np.empty((H, N))
        im = np.empty((H, N))
        _check(self.pipe.lib.pf_coll_download(self.h, _dp(re), _dp(im)))
        return np.ascontiguousarray(re.T), np.ascontiguousarray(im.T)

    def __del__(self):
        try:
            if self.owned and self.h and self.pipe.ctx:
                self.pipe.lib.pf_coll_destroy(self.h)
        except Exception:
            pass


class Phys:
    """A device `type (phys)` field (variables.f90:42-44)."""

    def __init__(self, pipe: "Pipe", handle=None, owned: bool = True):
        self.pipe = pipe
        self.owned = owned
        if handle is None:
            h = C.c_void_p()
            _check(pipe.lib.pf_phys_create(pipe.ctx, C.byref(h)))
            handle = h
        self.h = handle

    def upload(self, p: np.ndarray) -> "Phys":
        p = np.ascontiguousarray(p, dtype=np.float64)
        assert p.shape == (self.pipe.N, self.pipe.Th, self.pipe.Z)
        _check(self.pipe.lib.pf_phys_upload(self.h, _dp(p)))
        return self

    def download(self) -> np.ndarray:
        out = np.empty((self.pipe.N, self.pipe.Th, self.pipe.Z))
        _check(self.pipe.lib.pf_phys_download(self.h, _dp(out)))
        return out

    def __del__(self):
        try:
            if self.owned and self.h and self.pipe.ctx:
                self.pipe.lib.pf_phys_destroy(self.h)
        except Exception:
            pass


class Mesh:
    """A set of per-mode `type (mesh)` band matrices (meshs.f90:37-39)."""

    def __init__(self, pipe, h):
        self.pipe, self.h = pipe, h

    def download(self) -> np.ndarray:
        """(H, N, 2KL+1) array: [nh, j, row] == A(nh)%M(row+1, j+1)."""
        out = np.empty((self.pipe.H, self.pipe.N, 2 * L.KL + 1))
        _check(self.pipe.lib.pf_mesh_download(self.h, _dp(out)))
        return out

    def __del__(self):
        try:
            self.pipe.lib.pf_mesh_destroy(self.h)
        except Exception:
            pass


class LUMesh:
    """A set of per-mode `type (lumesh)` LU factors (meshs.f90:42-45)."""

    def __init__(self, pipe, h):
        self.pipe, self.h = pipe, h

    def download(self):
        """(M, ipiv): M (H, N, 3KL+1) == A(nh)%M(row+1, j+1); ipiv (H, N) 1-based."""
        H, N = self.pipe.H, self.pipe.N
        M = np.empty((H, N, 3 * L.KL + 1))
        piv = np.empty((H, N), dtype=np.int32)
        _check(self.pipe.lib.pf_lumesh_download(self.h, _dp(M), piv.ctypes.data_as(L.IP)))
        return M, piv

    def __del__(self):
        try:
            self.pipe.lib.pf_lumesh_destroy(self.h)
        except Exception:
            pass


class Pipe:
    """Module state of one pipe on one GPU."""

    def __init__(self, cfg: PipeConfig, device: int = -1, _handle=None):
        self.lib = L.load()
        self.cfg = cfg
        self.device = device  # -1: the device current at creation
        self._owned = _handle is None
        self.ctx = None
        if _handle is None:
            c = cfg_struct(cfg)
            self._r = c._r
            h = C.c_void_p()
            _check(self.lib.pf_ctx_create(C.byref(c), device, C.byref(h)))
            self.ctx = h
        else:
            self.ctx = _handle
        N, H, Z, Th = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _check(self.lib.pf_ctx_dims(self.ctx, C.byref(N), C.byref(H), C.byref(Z), C.byref(Th)))
        self.N, self.H, self.Z, self.Th = N.value, H.value, Z.value, Th.value
        self.K, self.M, self.Mp = cfg.K, cfg.M, cfg.Mp

    def reconfigure(self, cfg: PipeConfig):
        """New physics for the same shape (pf_ctx_reconfigure): a fresh run
        reusing this pipe's device memory; call vel_matrices again."""
        c = cfg_struct(cfg)
        _check(self.lib.pf_ctx_reconfigure(self.ctx, C.byref(c)))
        self.cfg = cfg

    def close(self):
        if self.ctx and self._owned:
            self.lib.pf_ctx_destroy(self.ctx)
        self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------- launch choices ----------------
    def set_tuning(self, ld_solver: int = L.PF_LD_AUTO, nl_mc: int = 0, nl_zc: int = 0, nl_fused: int = 0):
        """Launch choices of the fused step (pf_ctx_set_tuning); every choice
        gives the same numbers bit for bit, only the speed differs."""
        t = L.pf_tuning(int(ld_solver), int(nl_mc), int(nl_zc), int(nl_fused))
        _check(self.lib.pf_ctx_set_tuning(self.ctx, C.byref(t)))

    def get_tuning(self) -> dict:
        t = L.pf_tuning()
        _check(self.lib.pf_ctx_get_tuning(self.ctx, C.byref(t)))
        return {"ld_solver": t.ld_solver, "nl_mc": t.nl_mc, "nl_zc": t.nl_zc, "nl_fused": t.nl_fused}

    @property
    def nl_passes(self) -> int:
        """1 when the nonlinear terms run as one block per radial point, 3
        when they take the three-pass transforms (pf_nl_passes)."""
        v = C.c_int()
        _check(self.lib.pf_nl_passes(self.ctx, C.byref(v)))
        return v.value

    # ---------------- fields ----------------
    def coll(self, re=None, im=None) -> Coll:
        c = Coll(self)
        if re is not None:
            c.upload(re, im if im is not None else np.zeros_like(re))
        return c

    def phys(self, p=None) -> Phys:
        q = Phys(self)
        if p is not None:
            q.upload(p)
        return q

    def vel_field(self, which: int) -> Coll:
        h = C.c_void_p()
        _check(self.lib.pf_vel_coll(self.ctx, which, C.byref(h)))
        return Coll(self, h, owned=False)

    def vel_physfield(self, which: int) -> Phys:
        h = C.c_void_p()
        _check(self.lib.pf_vel_phys(self.ctx, which, C.byref(h)))
        return Phys(self, h, owned=False)

    @property
    def vel_ur(self):
        return self.vel_field(0)

    @property
    def vel_ut(self):
        return self.vel_field(1)

    @property
    def vel_uz(self):
        return self.vel_field(2)

    @property
    def vel_Nr(self):
        return self.vel_field(3)

    @property
    def vel_Nt(self):
        return self.vel_field(4)

    @property
    def vel_Nz(self):
        return self.vel_field(5)

    def set_state(self, ur, ut, uz):
        """ur, ut, uz: (re, im) pairs of (N, H) arrays."""
        arrs = []
        for re, im in (ur, ut, uz):
            arrs.append(np.ascontiguousarray(np.asarray(re, dtype=np.float64).T))
            arrs.append(np.ascontiguousarray(np.asarray(im, dtype=np.float64).T))
        _check(self.lib.pf_vel_set_state(self.ctx, *[_dp(a) for a in arrs]))

    def get_state(self):
        arrs = [np.empty((self.H, self.N)) for _ in range(6)]
        _check(self.lib.pf_vel_get_state(self.ctx, *[_dp(a) for a in arrs]))
        a = [np.ascontiguousarray(x.T) for x in arrs]
        return [(a[0], a[1]), (a[2], a[3]), (a[4], a[5])]

    def mes_D(self):
        """Radial mesh: dict of r, dr (KL, N, 2KL+1), radLap (N, 2KL+1), dr0/dr1 (KL+1, KL+1) [i, j], intrdr."""
        N, KL = self.N, L.KL
        r = np.empty(N)
        dr = np.empty((KL, N, 2 * KL + 1))
        rl = np.empty((N, 2 * KL + 1))
        d0 = np.empty((KL + 1, KL + 1))
        d1 = np.empty((KL + 1, KL + 1))
        w = np.empty(N)
        _check(self.lib.pf_mes_get(self.ctx, _dp(r), _dp(dr), _dp(rl), _dp(d0), _dp(d1), _dp(w)))
        return dict(r=r, dr=dr, radLap=rl, dr0=d0, dr1=d1, intrdr=w)

    def sync(self):
        _check(self.lib.pf_ctx_sync(self.ctx))

    def device_bytes(self) -> int:
        b = C.c_ulonglong()
        _check(self.lib.pf_ctx_device_bytes(self.ctx, C.byref(b)))
        return b.value

    # ---------------- variables.f90 ----------------
    def var_coll_init(self, a: Coll):
        _check(self.lib.pf_var_coll_init(a.h))

    def var_coll_copy(self, inp: Coll, out: Coll):
        _check(self.lib.pf_var_coll_copy(inp.h, out.h))

    def var_coll_add(self, ac: Coll, a: Coll):
        _check(self.lib.pf_var_coll_add(ac.h, a.h))

    def var_coll_sub(self, ac: Coll, a: Coll):
        _check(self.lib.pf_var_coll_sub(ac.h, a.h))

    def var_coll_dmult(self, d: float, a: Coll):
        _check(self.lib.pf_var_coll_dmult(d, a.h))

    def var_coll_neg(self, ac: Coll, a: Coll):
        _check(self.lib.pf_var_coll_neg(ac.h, a.h))

    def var_coll_meshmult(self, p: int, inp: Coll, out: Coll):
        _check(self.lib.pf_var_coll_meshmult(p, inp.h, out.h))

    def var_coll_curl(self, r: Coll, t: Coll, z: Coll, o_r: Coll, o_t: Coll, o_z: Coll):
        _check(self.lib.pf_var_coll_curl(r.h, t.h, z.h, o_r.h, o_t.h, o_z.h))

    def var_coll_grad(self, p: Coll, r: Coll, t: Coll, z: Coll):
        _check(self.lib.pf_var_coll_grad(p.h, r.h, t.h, z.h))

    def var_coll_div(self, r: Coll, t: Coll, z: Coll, dv: Coll):
        _check(self.lib.pf_var_coll_div(r.h, t.h, z.h, dv.h))

    def var_coll_shift(self, dt: float, dz: float, a: Coll, b: Coll):
        _check(self.lib.pf_var_coll_shift(dt, dz, a.h, b.h))

    def var_imposesym(self, i: int, r: Coll, t: Coll, z: Coll):
        _check(self.lib.pf_var_imposesym(i, r.h, t.h, z.h))

    def var_coll_norm(self, a: Coll):
        E = C.c_double()
        Ek = np.empty(self.K)
        Em = np.empty(self.M)
        _check(self.lib.pf_var_coll_norm(a.h, C.byref(E), _dp(Ek), _dp(Em)))
        return E.value, Ek, Em

    # ---------------- transform.fftw3.f90 ----------------
    def tra_coll2phys(self, c: Coll, p: Phys):
        _check(self.lib.pf_tra_coll2phys(c.h, p.h))

    def tra_phys2coll(self, p: Phys, c: Coll):
        _check(self.lib.pf_tra_phys2coll(p.h, c.h))

    tra_spec2phys = tra_coll2phys
    tra_phys2spec = tra_phys2coll

    # ---------------- timestep.f90 ----------------
    @property
    def tim(self) -> L.pf_tim_state:
        s = L.pf_tim_state()
        _check(self.lib.pf_tim_get(self.ctx, C.byref(s)))
        return s

    def set_tim(self, s: L.pf_tim_state):
        _check(self.lib.pf_tim_set(self.ctx, C.byref(s)))

    def tim_mesh_init(self, PM: int, c1: float, c2: float) -> Mesh:
        h = C.c_void_p()
        _check(self.lib.pf_tim_mesh_init(self.ctx, PM, c1, c2, C.byref(h)))
        return Mesh(self, h)

    def tim_lumesh_init(self, PM: int, BC: int, c1: float, c2: float) -> LUMesh:
        h = C.c_void_p()
        _check(self.lib.pf_tim_lumesh_init(self.ctx, PM, BC, c1, c2, C.byref(h)))
        return LUMesh(self, h)

    def tim_lumesh_invert(self, BC: int, A: LUMesh, b: Coll):
        _check(self.lib.pf_tim_lumesh_invert(BC, A.h, b.h))

    def tim_meshmult(self, S: int, A: Mesh, b: Coll, c: Coll, d: Coll):
        _check(self.lib.pf_tim_meshmult(S, A.h, b.h, c.h, d.h))

    def tim_zerobc(self, a: Coll):
        _check(self.lib.pf_tim_zerobc(a.h))

    def tim_nlincorr(self, N_: Coll, Nn: Coll):
        _check(self.lib.pf_tim_nlincorr(N_.h, Nn.h))

    def tim_measurecorr(self, c1: Coll, c2: Coll, c3: Coll):
        _check(self.lib.pf_tim_measurecorr(c1.h, c2.h, c3.h))

    def tim_check_cgce(self):
        _check(self.lib.pf_tim_check_cgce(self.ctx))

    def tim_new_tstep(self):
        _check(self.lib.pf_tim_new_tstep(self.ctx))

    # ---------------- velocity.f90 ----------------
    def vel_imposesym(self):
        _check(self.lib.pf_vel_imposesym(self.ctx))

    def vel_matrices(self):
        _check(self.lib.pf_vel_matrices(self.ctx))

    def vel_transform(self):
        _check(self.lib.pf_vel_transform(self.ctx))

    def vel_nonlinear(self):
        _check(self.lib.pf_vel_nonlinear(self.ctx))

    def vel_transform_nonlinear(self):
        """vel_transform + vel_nonlinear fused; vel_r..vel_curlz are not updated."""
        _check(self.lib.pf_vel_transform_nonlinear(self.ctx))

    def vel_predictor(self):
        _check(self.lib.pf_vel_predictor(self.ctx))

    def vel_corrector(self):
        _check(self.lib.pf_vel_corrector(self.ctx))

    def vel_maxtstep(self):
        _check(self.lib.pf_vel_maxtstep(self.ctx))

    @property
    def vel_Pr0(self) -> float:
        p = C.c_double()
        _check(self.lib.pf_vel_get_scalars(self.ctx, C.byref(p), None))
        return p.value

    @property
    def vel_nu(self) -> float:
        """The reference viscosity of the implicit operator (velocity.f90:26)."""
        p = C.c_double()
        _check(self.lib.pf_vel_get_scalars(self.ctx, None, C.byref(p)))
        return p.value

    def influence(self):
        """U (6, H, N) and the inverted A (H, 4, 4) of vel_adjPPE(0)."""
        U = np.empty((6, self.H, self.N))
        A = np.empty((self.H, 4, 4))  # memory [nh][j][i] -> transpose below
        _check(self.lib.pf_vel_influence_download(self.ctx, _dp(U), _dp(A)))
        return U, np.ascontiguousarray(A.transpose(0, 2, 1))

    # ---------------- drivers ----------------
    def timestep(self) -> int:
        n = C.c_int()
        _check(self.lib.pf_timestep(self.ctx, C.byref(n)))
        return n.value

    def steporbit(self, nsteps: int):
        _check(self.lib.pf_steporbit(self.ctx, nsteps))

    # ---------------- util plug-ins (main.f90's var_null hook) ----------------
    def util_set(self, kind: int, params=()):
        """Built-in plug-in: PF_UTIL_CORIOLIS (Ek0, phi) or PF_UTIL_CARREAU_YASUDA
        (rho, radius, mu_0, mu_inf, lam_CY, n_CY, a_CY); PF_UTIL_NONE clears."""
        p = np.ascontiguousarray(params, dtype=np.float64)
        _check(self.lib.pf_util_set(self.ctx, int(kind), _dp(p) if p.size else None, int(p.size)))

    def util_set_callback(self, fn):
        """fn(flag) runs at var_null(flag) inside pf_timestep (None clears)."""
        if fn is None:
            self._util_cb = None
            _check(self.lib.pf_util_set_callback(self.ctx, None, None))
            return
        self._util_cb = L.UTIL_FN(lambda ctx, flag, user: fn(flag))
        _check(self.lib.pf_util_set_callback(self.ctx, C.cast(self._util_cb, C.c_void_p), None))

    def util(self, flag: int):
        _check(self.lib.pf_util(self.ctx, int(flag)))

    def util_nu_stats(self):
        """(nu_wall, nu_min, nu_max) of the last Carreau-Yasuda evaluation."""
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        _check(self.lib.pf_util_nu_stats(self.ctx, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    # ---------------- io.f90 state files ----------------
    def io_save_state(self, path):
        """io_save_state (io.f90:303-378): this pipe's state to a netCDF file."""
        from .statefile import io_save_state
        io_save_state(self, path)

    def io_load_state(self, path, time_from_file: bool = False) -> int:
        """io_load_state (io.f90:98-226): interpolated and re-truncated onto
        this pipe; returns the change bits (1 mesh, 2 K, 4 M, 8 Mp)."""
        from .statefile import io_load_state
        return io_load_state(self, path, time_from_file)

    def energy(self) -> float:
        E = C.c_double()
        _check(self.lib.pf_diag_energy(self.ctx, C.byref(E)))
        return E.value

    def friction(self):
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        _check(self.lib.pf_diag_friction(self.ctx, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    # ---------------- instrumentation ----------------
    KERNEL_CATEGORIES = ("zinv", "thinv", "thfwd", "zfwd", "lusolve", "stencil", "ew", "infl",
                         "factor", "step", "ppe")

    def launches(self) -> int:
        n = C.c_ulonglong()
        _check(self.lib.pf_ctx_launches(self.ctx, C.byref(n)))
        return n.value

    def prof_enable(self, on=True):
        """on: True (all categories), False, or a list of category names."""
        if on is True:
            mask = (1 << len(self.KERNEL_CATEGORIES)) - 1
        elif not on:
            mask = 0
        else:
            mask = 0
            for name in on:
                mask |= 1 << self.KERNEL_CATEGORIES.index(name)
        _check(self.lib.pf_prof_enable(self.ctx, mask))

    def prof_read(self):
        """{category: (total ms, launches)} since prof_enable."""
        out = {}
        for i, name in enumerate(self.KERNEL_CATEGORIES):
            ms, n = C.c_double(), C.c_ulonglong()
            _check(self.lib.pf_prof_read(self.ctx, i, C.byref(ms), C.byref(n)))
            out[name] = (ms.value, n.value)
        return out


class Batch:
    """Independent pipes of uneven size advanced together (pf_batch_*): one
    CUDA graph per batch timestep, each stage launched once over all pipes
    where the pipes allow it, else one kernel chain per pipe."""

    def __init__(self, cfgs=(), device: int = -1):
        self.lib = L.load()
        cfgs = list(cfgs)
        arr = (L.pf_config * max(1, len(cfgs)))()
        keep = []
        for i, cfg in enumerate(cfgs):
            c = cfg_struct(cfg)
            keep.append(c._r)
            arr[i] = c
        h = C.c_void_p()
        self.h = None
        _check(self.lib.pf_batch_create(len(cfgs), arr, device, C.byref(h)))
        self.h = h
        self.pipes = []
        for i, cfg in enumerate(cfgs):
            ph = C.c_void_p()
            _check(self.lib.pf_batch_pipe(self.h, i, C.byref(ph)))
            self.pipes.append(Pipe(cfg, _handle=ph))

    def attach(self, pipe: "Pipe"):
        """Add a pipe the caller owns (it must stay open while attached)."""
        _check(self.lib.pf_batch_attach(self.h, pipe.ctx))
        self.pipes.append(pipe)

    def detach(self, pipe: "Pipe"):
        _check(self.lib.pf_batch_detach(self.h, pipe.ctx))
        self.pipes = [p for p in self.pipes if p is not pipe]

    def set_graphs(self, on: bool):
        """False: launch every step directly (membership changing every step)."""
        _check(self.lib.pf_batch_set_graphs(self.h, int(bool(on))))

    @property
    def worklist(self) -> bool:
        """Whether each transform stage runs as one persistent launch over a
        work list of every pipe's tiles (else one launch per transform length)."""
        v = C.c_int()
        _check(self.lib.pf_batch_get_worklist(self.h, C.byref(v)))
        return bool(v.value)

    def set_worklist(self, on: bool):
        """Choose the form of the transform stages (bitwise the same results)."""
        _check(self.lib.pf_batch_set_worklist(self.h, int(bool(on))))

    def matrices(self):
        _check(self.lib.pf_batch_matrices(self.h))

    def step(self, nsteps: int = 1, orbit: bool = False) -> int:
        """Advance every pipe; returns the corrector passes summed over pipes and steps."""
        n = C.c_longlong()
        _check(self.lib.pf_batch_step(self.h, nsteps, int(orbit), C.byref(n)))
        return n.value

    def sync(self):
        _check(self.lib.pf_batch_sync(self.h))

    # ---- pipelined state I/O (pf_batch_put_states / step_io / get_states)
    def io_bytes(self) -> int:
        """Bytes of one state block: every pipe's (ur, ut, uz) Re/Im, pipe
        after pipe, each (H, N) with n fastest."""
        b = C.c_ulonglong()
        _check(self.lib.pf_batch_io_bytes(self.h, C.byref(b)))
        return b.value

    @staticmethod
    def _host_ptr(buf) -> C.c_void_p:
        if isinstance(buf, np.ndarray):
            if buf.dtype != np.float64 or not buf.flags.c_contiguous:
                raise PipeflowError(L.PF_ERR_ARG, "state block: contiguous float64 array required")
            return C.c_void_p(buf.ctypes.data)
        return C.c_void_p(buf.data_ptr())  # a torch tensor (page-locked for overlap)

    def put_states(self, slot: int, host):
        _check(self.lib.pf_batch_put_states(self.h, slot, self._host_ptr(host)))

    def step_io(self, slot: int, nsteps: int = 1, orbit: bool = False) -> int:
        n = C.c_longlong()
        _check(self.lib.pf_batch_step_io(self.h, slot, nsteps, int(orbit), C.byref(n)))
        return n.value

    def get_states(self, slot: int, host):
        _check(self.lib.pf_batch_get_states(self.h, slot, self._host_ptr(host)))

    def io_wait(self, slot: int):
        _check(self.lib.pf_batch_io_wait(self.h, slot))

    def io_sync(self):
        _check(self.lib.pf_batch_io_sync(self.h))

    def prof_enable(self, on=True):
        """on: True (all kernel categories), False, or a list of category names."""
        cats = Pipe.KERNEL_CATEGORIES
        if on is True:
            mask = (1 << len(cats)) - 1
        elif not on:
            mask = 0
        else:
            mask = sum(1 << cats.index(n) for n in on)
        _check(self.lib.pf_batch_prof_enable(self.h, mask))

    def prof_read(self, staged_only=False):
        """{category: (total ms, launches)} summed over the pipes; with
        staged_only, the spans of the stage-batched launches alone (each
        covers every pipe), without per-pipe launches."""
        fn = self.lib.pf_batch_prof_read_staged if staged_only else self.lib.pf_batch_prof_read
        out = {}
        for i, name in enumerate(Pipe.KERNEL_CATEGORIES):
            ms, n = C.c_double(), C.c_ulonglong()
            _check(fn(self.h, i, C.byref(ms), C.byref(n)))
            out[name] = (ms.value, n.value)
        return out

    def launches(self) -> int:
        """Kernels launched so far by the batch (the pipes' and the batched ones)."""
        n = C.c_ulonglong()
        _check(self.lib.pf_batch_launches(self.h, C.byref(n)))
        return n.value

    def staged(self) -> bool:
        """True when each stage of a step is one launch over every pipe."""
        v = C.c_int()
        _check(self.lib.pf_batch_staged(self.h, C.byref(v)))
        return bool(v.value)

    def close(self):
        if self.h:
            for p in self.pipes:
                if not p._owned:  # the batch's own pipes die with it; attached ones stay open
                    p.ctx = None
            self.lib.pf_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching request server (pf_serve_*): each request advances
    a state by nsteps timesteps; admitted requests share one batch."""

    def __init__(self, hbm_budget: int = 150 * 10**9, max_active: int = 4096, orbit: bool = True,
                 device: int = -1):
        self.lib = L.load()
        h = C.c_void_p()
        self.h = None
        _check(self.lib.pf_serve_create(device, int(hbm_budget), int(max_active), int(orbit), C.byref(h)))
        self.h = h
        self._shape = {}

    def submit(self, cfg: PipeConfig, nsteps: int, state) -> int:
        """state: (ur, ut, uz), each an (re, im) pair of (N, H) arrays, as
        Pipe.set_state takes it."""
        c = cfg_struct(cfg)
        arrs = []
        for re, im in state:
            arrs.append(np.ascontiguousarray(np.asarray(re, dtype=np.float64).T))
            arrs.append(np.ascontiguousarray(np.asarray(im, dtype=np.float64).T))
        ptrs = [_dp(a) for a in arrs]
        rid = C.c_longlong()
        _check(self.lib.pf_serve_submit(self.h, C.byref(c), int(nsteps), *ptrs, C.byref(rid)))
        self._shape[rid.value] = (cfg.H, cfg.N)
        return rid.value

    def step(self):
        """Admit, advance one timestep, retire; returns (admitted, finished)."""
        a, f = C.c_int(), C.c_int()
        _check(self.lib.pf_serve_step(self.h, C.byref(a), C.byref(f)))
        return a.value, f.value

    def finished(self, cap: int = 4096):
        ids = (C.c_longlong * cap)()
        n = C.c_int()
        _check(self.lib.pf_serve_finished(self.h, ids, cap, C.byref(n)))
        return [ids[i] for i in range(n.value)]

    def cancel(self, rid: int):
        """Withdraw a queued or running request (pf_serve_cancel); it is
        reported finished and its result() raises PF_ERR_CANCELLED."""
        _check(self.lib.pf_serve_cancel(self.h, int(rid)))

    def result(self, rid: int):
        """Final state as Pipe.get_state returns it; the request is forgotten.
        A request that failed (corrector abort, non-finite state, admission)
        or was cancelled raises PipeflowError with its own status."""
        H, N = self._shape.pop(rid)
        out = [np.empty((H, N), dtype=np.float64) for _ in range(6)]
        _check(self.lib.pf_serve_result(self.h, int(rid), *[_dp(a) for a in out]))
        a = [np.ascontiguousarray(x.T) for x in out]
        return [(a[0], a[1]), (a[2], a[3]), (a[4], a[5])]

    def stats(self) -> dict:
        q, a, p = C.c_int(), C.c_int(), C.c_int()
        b, s = C.c_ulonglong(), C.c_longlong()
        _check(self.lib.pf_serve_stats(self.h, C.byref(q), C.byref(a), C.byref(p), C.byref(b), C.byref(s)))
        return dict(queued=q.value, active=a.value, pooled=p.value, bytes=b.value, steps=s.value)

    def launches(self) -> int:
        bh = C.c_void_p()
        _check(self.lib.pf_serve_batch(self.h, C.byref(bh)))
        n = C.c_ulonglong()
        _check(self.lib.pf_batch_launches(bh, C.byref(n)))
        return n.value

    def close(self):
        if self.h:
            self.lib.pf_serve_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
