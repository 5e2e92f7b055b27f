"""CPU oracle of the util plug-ins (Coriolis.f90, nonnewtonian.f90) and of
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
