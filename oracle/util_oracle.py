"""CPU oracle of the util plug-ins (Coriolis.f90, nonnewtonian.f90, LES.f90) and of
main.f90's loop with its var_null hook.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module.  It is
a numpy restatement on top of the timestep oracle (pipeflow_oracle.Pipe).

Parity status: **parity unpinned** (as the timestep oracle); the plug-ins are
additionally pinned by invariants in tests/test_util.py (a Coriolis force
about the pipe axis acts on the azimuthal and radial velocity only, and on
laminar flow it is the analytic m = 1 force; a
Newtonian limit of the Carreau-Yasuda law, mu_inf = mu_0, adds nothing; on
laminar flow the Carreau-Yasuda term equals the analytic divergence of the
extra viscous stress).
"""
from __future__ import annotations

import math

import numpy as np

from pipeflow_oracle import Coll, Pipe

PI = 3.1415926535897931


def coriolis(op: Pipe, Ek0: float, phi: float) -> None:
    """util(2) of Coriolis.f90:40-68: N += -1/(4 Ro) Omega x (U + u'),
    Ro = Re Ek0, from the physical fields vel_transform made."""
    P = op.phys
    Th = 3 * op.M
    d1 = 2.0 * PI / Th
    th = d1 * np.arange(Th)
    Or = math.sin(phi) * np.cos(th)
    Ot = -math.sin(phi) * np.sin(th)
    Oz = math.cos(phi)
    U = op.vel_U[:, None, None]
    Ro = op.cfg.Re * Ek0
    f = -1.0 / (4.0 * Ro)
    vr, vt, vz = P["r"], P["t"], P["z"]  # (N, Th, Z)
    w = vz + U
    Nr = f * (Ot[None, :, None] * w - Oz * vt)
    Nt = f * (Oz * vr - Or[None, :, None] * w)
    Nz = f * (Or[None, :, None] * vt - Ot[None, :, None] * vr)
    for name, p in (("vel_Nr", Nr), ("vel_Nt", Nt), ("vel_Nz", Nz)):
        c = op.tra_phys2spec(p)
        old = getattr(op, name)
        setattr(op, name, Coll(old.re + c.re, old.im + c.im))


def carreau_yasuda(op: Pipe, rho, radius, mu_0, mu_inf, lam_CY, n_CY, a_CY):
    """util(2) of nonnewtonian.f90: get_nu (:111-207) then
    update_nonlin_terms (:213-246).  Returns (nu_wall, nu_min, nu_max)."""
    D = op.mes_D
    lam = op.cfg.Re * lam_CY * mu_0 / (rho * radius ** 2)
    ur, ut, uz = op.vel_ur.copy(), op.vel_ut.copy(), op.vel_uz.copy()
    uz.re[:, 0] = uz.re[:, 0] + op.vel_U
    A = [[None] * 3 for _ in range(3)]
    for j, f in enumerate((ur, ut, uz)):
        A[0][j] = op.tra_spec2phys(op.var_coll_meshmult(D.dr[0], f))
    m_ = (op.mm * op.Mp).astype(float)[None, :]
    rm1 = D.rp[-1][:, None]
    c1 = Coll(rm1 * (-ur.im * m_ - ut.re), rm1 * (ur.re * m_ - ut.im))
    c2 = Coll(rm1 * (-ut.im * m_ + ur.re), rm1 * (ut.re * m_ + ur.im))
    c3 = Coll(rm1 * (-uz.im * m_), rm1 * (uz.re * m_))
    for j, c in enumerate((c1, c2, c3)):
        A[1][j] = op.tra_spec2phys(c)
    d1 = (op.cfg.alpha * op.kk.astype(float))[None, :]
    for j, f in enumerate((ur, ut, uz)):
        A[2][j] = op.tra_spec2phys(Coll(-f.im * d1, f.re * d1))
    S = A
    for (i, j) in ((0, 1), (0, 2), (1, 2)):
        s = 0.5 * (S[i][j] + S[j][i])
        S[i][j] = s
        S[j][i] = s
    sr = S[0][0] ** 2 + S[1][1] ** 2 + S[2][2] ** 2 + 2.0 * (S[0][1] ** 2 + S[0][2] ** 2 + S[1][2] ** 2)
    sr = np.sqrt(2.0 * sr)
    e1 = mu_inf / mu_0
    e2 = -n_CY / a_CY
    nu = e1 + (1.0 - e1) * (1.0 + (lam * sr) ** a_CY) ** e2
    nuc = op.tra_phys2spec(nu)
    stats = (float(nuc.re[-1, 0]), float(nu.min()), float(nu.max()))
    # update_nonlin_terms
    g = [op.tra_spec2phys(c) for c in op.var_coll_grad(nuc)]
    w = op.var_coll_curl(ur, ut, uz)
    q = [op.tra_spec2phys(c) for c in op.var_coll_curl(*w)]
    nu_ = nu - op.vel_nu
    for i in range(3):
        v = nu_ * (-q[i])
        for j in range(3):
            v = v + g[j] * S[j][i] * 2.0
        if i == 2:
            v = v + (op.vel_nu - 1.0) * (-4.0)
        q[i] = v / op.cfg.Re
    for name, p in zip(("vel_Nr", "vel_Nt", "vel_Nz"), q):
        c = op.tra_phys2spec(p)
        old = getattr(op, name)
        setattr(op, name, Coll(old.re + c.re, old.im + c.im))
    return stats


def velocity_gradient(op: Pipe):
    """The total velocity (u' plus the laminar U on the mean mode) and its
    gradient tensor A(i, j) on the physical grid, rows d/dr, (1/r)(d/dth ..),
    d/dz (LES.f90:109-150; nonnewtonian.f90:119-157)."""
    D = op.mes_D
    ur, ut, uz = op.vel_ur.copy(), op.vel_ut.copy(), op.vel_uz.copy()
    uz.re[:, 0] = uz.re[:, 0] + op.vel_U
    A = [[None] * 3 for _ in range(3)]
    for j, f in enumerate((ur, ut, uz)):
        A[0][j] = op.tra_spec2phys(op.var_coll_meshmult(D.dr[0], f))
    m_ = (op.mm * op.Mp).astype(float)[None, :]
    rm1 = D.rp[-1][:, None]
    c1 = Coll(rm1 * (-ur.im * m_ - ut.re), rm1 * (ur.re * m_ - ut.im))
    c2 = Coll(rm1 * (-ut.im * m_ + ur.re), rm1 * (ut.re * m_ + ur.im))
    c3 = Coll(rm1 * (-uz.im * m_), rm1 * (uz.re * m_))
    for j, c in enumerate((c1, c2, c3)):
        A[1][j] = op.tra_spec2phys(c)
    d1 = (op.cfg.alpha * op.kk.astype(float))[None, :]
    for j, f in enumerate((ur, ut, uz)):
        A[2][j] = op.tra_spec2phys(Coll(-f.im * d1, f.re * d1))
    return (ur, ut, uz), A


class LES:
    """The LES plug-in of LES.f90 (FLAG == 2: get_nu, update_nu_r,
    update_nonlin_terms; LES.f90:102-339): Smagorinsky (model 1) or Vreman
    (model 2) eddy viscosity nu_t from the resolved strain, with the van
    Driest wall damping, and the extra nonlinear terms of a variable
    viscosity.  The FLAG == 1 outputs (bisect, profiles, vel_Retau.dat) are
    not part of it.  Holds the per-run state the reference keeps in its les
    module: Re_tau, u_tau, nu_max and the filter widths."""

    def __init__(self, op: Pipe, model: int, C_s: float, filter_: int, A_plus: float):
        # init_params_model (LES.f90:68-96)
        self.model, self.C_s, self.filter, self.A_plus = int(model), float(C_s), int(filter_), float(A_plus)
        op.tim_pcn = 1
        op.tim_it = 0
        N = op.N
        r = op.mes_D.rp[1]
        self.Rdth = (2.0 * PI / float(op.Mp * 3 * op.M)) * (3.0 / 2.0)
        self.dz = (2.0 * PI / (op.cfg.alpha * 3 * op.K)) * (3.0 / 2.0)
        Dr = np.empty(N)
        Dr[0] = (r[1] - 0.0) / 2.0
        for n in range(1, N - 1):
            Dr[n] = (r[n + 1] - r[n - 1]) / 2.0
        Dr[N - 1] = 1.0 - r[N - 2]
        self.Delta_r = Dr
        self.r = r
        self.Re_tau = self.u_tau = self.nu_max = 0.0

    def get_nu(self, op: Pipe):
        """LES.f90:102-189: A, S, the strain rate, u_tau, nu_t, nu_max."""
        (u, A) = velocity_gradient(op)
        S = [[None] * 3 for _ in range(3)]
        for i in range(3):
            S[i][i] = A[i][i]
        for (i, j) in ((0, 1), (0, 2), (1, 2)):
            S[i][j] = 0.5 * (A[i][j] + A[j][i])
            S[j][i] = S[i][j]
        sr = S[0][0] ** 2 + S[1][1] ** 2 + S[2][2] ** 2 + 2.0 * (S[0][1] ** 2 + S[0][2] ** 2 + S[1][2] ** 2)
        sr = np.sqrt(2.0 * sr)
        D = op.mes_D
        N = op.N
        d1 = float(np.dot(op.vel_uz.re[N - 1 - 4:N, 0], D.dr1[:, 1]))
        self.u_tau = math.sqrt(abs((d1 - 2.0) / op.cfg.Re))
        self.Re_tau = op.cfg.Re * self.u_tau
        y_plus = self.Re_tau * (1.0 - self.r)
        if self.model == 1:
            nu = self._smagorinsky(sr, y_plus)
        else:
            nu = self._vreman(A, y_plus)
        self.nu = nu
        self.nuc = op.tra_phys2spec(nu)
        self.nu_max = float(nu.max())
        return u, S

    def _smagorinsky(self, sr, y_plus):
        """LES.f90:195-223"""
        Dr, r = self.Delta_r, self.r
        if self.filter == 1:
            Delta = (Dr * self.Rdth * self.dz) ** (1.0 / 3.0)
        elif self.filter == 2:
            Delta = (Dr * r * self.Rdth * self.dz) ** (1.0 / 3.0)
        else:
            Delta = np.sqrt((Dr ** 2 + (r * self.Rdth) ** 2 + self.dz ** 2) / 3.0)
        vanDr = 1.0 - np.exp(-(y_plus / self.A_plus) ** 2)
        d1 = vanDr * (self.C_s * Delta) ** 2
        return d1[:, None, None] * sr

    def _vreman(self, A, y_plus):
        """LES.f90:229-274.  For filter 3 the reference assigns no width to
        the azimuthal direction, so its d1 keeps the last radial width,
        Delta_r(i_N); that is restated."""
        Dr, r = self.Delta_r, self.r
        N = len(r)
        AA = np.zeros_like(A[0][0])
        for i in range(3):
            for j in range(3):
                AA = AA + A[i][j] ** 2
        dm = [Dr, None, np.full(N, self.dz)]
        if self.filter == 1:
            dm[1] = np.full(N, self.Rdth)
        elif self.filter == 2:
            dm[1] = r * self.Rdth
        else:
            dm[1] = np.full(N, Dr[N - 1])
        B = [[None] * 3 for _ in range(3)]
        for i in range(3):
            for j in range(3):
                b = np.zeros_like(AA)
                for m in range(3):
                    b = b + (dm[m] ** 2)[:, None, None] * A[m][i] * A[m][j]
                B[i][j] = b
        P = (B[0][0] * B[1][1] - B[0][1] ** 2 + B[0][0] * B[2][2] - B[0][2] ** 2
             + B[1][1] * B[2][2] - B[1][2] ** 2)
        P = np.where(AA < 1e-12, 0.0, P)
        P = np.maximum(P, 0.0)
        AA = np.maximum(AA, 1e-12)
        nu = self.C_s * np.sqrt(P / AA)
        if self.A_plus <= 0.0:
            return nu
        vanDr = 1.0 - np.exp(-(y_plus / self.A_plus) ** 2)
        d1 = 0.03 / self.C_s
        d1 = d1 + (1.0 - d1) * vanDr
        return d1[:, None, None] * nu

    def update_nu_r(self, op: Pipe) -> bool:
        """LES.f90:280-290: a new reference viscosity (and matrices) when
        nu_r strays from 1.1 (1 + Re nu_max) by more than 7%."""
        d1 = 1.0 + op.cfg.Re * self.nu_max
        d1 = 1.10 * d1
        if op.vel_nu < 0.93 * d1 or op.vel_nu > 1.07 * d1:
            op.vel_nu = d1
            op.vel_matrices()
            return True
        return False

    def update_nonlin_terms(self, op: Pipe, u, S):
        """LES.f90:296-339"""
        g = [op.tra_spec2phys(c) for c in op.var_coll_grad(self.nuc)]
        w = op.var_coll_curl(*u)
        q = [op.tra_spec2phys(c) for c in op.var_coll_curl(*w)]
        Re = op.cfg.Re
        nu = self.nu
        nu_ = Re * nu + (1.0 - op.vel_nu)
        for i in range(3):
            v = (1.0 / Re) * nu_ * (-q[i])
            if i == 2:
                v = v + nu * (-4.0)
            for j in range(3):
                v = v + g[j] * S[j][i] * 2.0
            q[i] = v
        for name, p in zip(("vel_Nr", "vel_Nt", "vel_Nz"), q):
            c = op.tra_phys2spec(p)
            old = getattr(op, name)
            setattr(op, name, Coll(old.re + c.re, old.im + c.im))

    def __call__(self, op: Pipe):
        """util(2) of LES.f90:58-62"""
        u, S = self.get_nu(op)
        if op.tim_it == 0:
            self.update_nu_r(op)
        self.update_nonlin_terms(op, u, S)


def timestep_with_util(op: Pipe, util) -> int:
    """main.f90:20-41 with var_null(2) after every nonlinear evaluation
    (fixed dt).  util(op) adds its terms.  Returns the corrector passes."""
    op.vel_imposesym()
    op.vel_transform()
    op.vel_nonlinear()
    util(op)
    op.vel_predictor()
    op.tim_it = 1
    n = 0
    while op.tim_it != 0:
        op.vel_transform()
        op.vel_nonlinear()
        util(op)
        op.vel_corrector()
        op.tim_check_cgce()
        n += 1
    op.tim_t = op.tim_t + op.tim_dt
    op.tim_step = op.tim_step + 1
    return n
