"""util plug-ins through main.f90's var_null hook (Coriolis.f90,
nonnewtonian.f90, LES.f90) and the host callback.

CPU: invariants of the oracle's restatements.  GPU: pf_timestep with each
built-in plug-in against the oracle's main loop with the same plug-in, the
Carreau-Yasuda viscosity statistics, and the order of the hook calls."""
import numpy as np
import pytest

import pipeflow_oracle as O
import util_oracle as UO
from _util import SMALL, device_pipe, oracle_pipe, state_from_dev, state_to_dev

CFG = dict(N=20, K=5, M=4, Mp=1, Re=2000.0, alpha=1.25, dt=0.01)
CY = (1000.0, 0.01, 0.05, 0.0035, 3.3, 0.36, 2.0)  # rho, radius, mu_0, mu_inf, lam, n, a


def _oracle(cfgd, seed=6):
    o = oracle_pipe(cfgd)
    o.vel_matrices()
    st = O.seeded_state(o, seed, 1e-3)
    o.set_state(*st)
    return o, st


def test_coriolis_about_the_pipe_axis_leaves_axial_terms():
    """Omega along the pipe axis (phi = 0): Omega x u has no z component."""
    o, _ = _oracle(CFG)
    o.vel_imposesym()
    o.vel_transform()
    o.vel_nonlinear()
    Nz = o.vel_Nz.copy()
    Nr = o.vel_Nr.copy()
    UO.coriolis(o, 0.5, 0.0)
    assert np.array_equal(o.vel_Nz.re, Nz.re) or np.max(np.abs(o.vel_Nz.re - Nz.re)) < 1e-15
    assert np.max(np.abs(o.vel_Nr.re - Nr.re)) > 1e-9


def test_carreau_yasuda_newtonian_limit_adds_nothing():
    """mu_inf = mu_0 makes nu = 1 everywhere: no extra stress."""
    o, _ = _oracle(CFG)
    o.vel_imposesym()
    o.vel_transform()
    o.vel_nonlinear()
    N0 = [o.vel_Nr.copy(), o.vel_Nt.copy(), o.vel_Nz.copy()]
    stats = UO.carreau_yasuda(o, 1000.0, 0.01, 0.05, 0.05, 3.3, 0.36, 2.0)
    assert stats[1] == pytest.approx(1.0, abs=1e-15) and stats[2] == pytest.approx(1.0, abs=1e-15)
    assert O.rel_l2([o.vel_Nr, o.vel_Nt, o.vel_Nz], N0) < 1e-10


SMAG = (1.0, 0.025, 1.0, 25.0)   # model, C_s, filter, A_plus (LES.f90:4-6)
VREMAN = (2.0, 0.03, 2.0, 0.0)   # (LES.f90:8-10)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["coriolis", "carreau_yasuda", "les_smagorinsky", "les_vreman",
                                  "les_smagorinsky_filter3", "les_vreman_filter3"])
def test_plugin_steps_match_oracle(kind):
    import pipeflow as P
    o, st = _oracle(CFG)
    g = device_pipe(CFG)
    g.vel_matrices()
    state_to_dev(g, st)
    if kind == "coriolis":
        g.util_set(P._lib.PF_UTIL_CORIOLIS, (0.5, 0.3))
        util = lambda op: UO.coriolis(op, 0.5, 0.3)  # noqa: E731
    elif kind == "carreau_yasuda":
        g.util_set(P._lib.PF_UTIL_CARREAU_YASUDA, CY)
        o.tim_pcn = 1  # nonnewtonian.f90:66-67
        o.tim_it = 0
        stats = []
        util = lambda op: stats.append(UO.carreau_yasuda(op, *CY))  # noqa: E731
    else:
        par = list(SMAG if "smagorinsky" in kind else VREMAN)
        if kind.endswith("filter3"):
            par[2] = 3.0
            par[3] = 25.0
        g.util_set(P._lib.PF_UTIL_LES, par)
        util = UO.LES(o, *par)
    for _ in range(3):
        no = UO.timestep_with_util(o, util)
        ng = g.timestep()
        assert no == ng
    assert O.rel_l2(state_from_dev(g), o.state()) <= 1e-11
    if kind.startswith("les"):
        # update_nu_r moved the reference viscosity (and the matrices) alike
        assert g.vel_nu == pytest.approx(o.vel_nu, rel=1e-12)
        if "smagorinsky" in kind:
            assert o.vel_nu > 1.0
        wall, lo, hi = g.util_nu_stats()
        assert hi == pytest.approx(util.nu_max, rel=1e-11)
        assert hi > 0.0 and lo >= 0.0
    if kind == "carreau_yasuda":
        wall, lo, hi = g.util_nu_stats()
        assert wall == pytest.approx(stats[-1][0], rel=1e-11)
        assert lo == pytest.approx(stats[-1][1], rel=1e-11) and hi == pytest.approx(stats[-1][2], rel=1e-11)
        assert lo < hi <= 1.0


@pytest.mark.gpu
def test_callback_order_and_effect():
    """The callback runs at var_null(2), var_null(1), var_null(2) for a step
    with one corrector pass, and what it adds to vel_N changes the step as
    the same addition does in the oracle's loop."""
    import pipeflow as P
    o, st = _oracle(CFG)
    g = device_pipe(CFG)
    g.vel_matrices()
    state_to_dev(g, st)
    flags = []
    extra = P.Coll(g)
    rng = np.random.default_rng(2)
    add = O.Coll(1e-4 * rng.standard_normal((g.N, g.H)), np.zeros((g.N, g.H)))
    add.re[:, 0] = 0.0
    extra.upload(add.re, add.im)

    def hook(flag):
        flags.append(flag)
        if flag == 2:
            g.var_coll_add(extra, g.vel_Nz)

    def util(op):
        op.vel_Nz = O.Coll(op.vel_Nz.re + add.re, op.vel_Nz.im + add.im)

    g.util_set_callback(hook)
    no = UO.timestep_with_util(o, util)
    ng = g.timestep()
    assert flags[:3] == [2, 1, 2] and len(flags) == 2 + ng
    assert no == ng
    assert O.rel_l2(state_from_dev(g), o.state()) <= 1e-11
    g.util_set_callback(None)


def test_carreau_yasuda_on_laminar_flow_matches_the_stress_divergence():
    """For Hagen-Poiseuille flow alone (u' = 0) the strain rate is |U'| = 2r
    and the extra term is the divergence of the extra viscous stress,
    N'_z(r) = [-4 (nu - 1) - 2 r nu'(r)] / Re in the mean mode, with nothing
    in the other components or modes.  The radial derivatives are the 9-point
    finite differences, so the first points off the axis carry a truncation
    error that falls fast with N (1e-4 of the maximum at N = 40, 6e-7 at 80)."""
    o = oracle_pipe(dict(N=80, K=3, M=3, Mp=1, Re=2000.0, alpha=1.25, dt=0.01))
    o.vel_matrices()
    z = O.Coll.zeros(o.N, o.H)
    o.vel_Nr, o.vel_Nt, o.vel_Nz = z.copy(), z.copy(), z.copy()
    o.vel_ur, o.vel_ut, o.vel_uz = z.copy(), z.copy(), z.copy()
    # a relaxation time that keeps nu(r) smooth on the mesh (lam * 2r <= 10)
    rho, radius, mu0, muinf, lamCY, nCY, aCY = 1000.0, 0.01, 0.05, 0.0035, 0.005, 0.36, 2.0
    UO.carreau_yasuda(o, rho, radius, mu0, muinf, lamCY, nCY, aCY)
    r = o.mes_D.r
    lam = o.cfg.Re * lamCY * mu0 / (rho * radius ** 2)
    e1, e2 = muinf / mu0, -nCY / aCY
    x = lam * 2.0 * r
    nu = e1 + (1 - e1) * (1 + x ** aCY) ** e2
    dnu = (1 - e1) * e2 * (1 + x ** aCY) ** (e2 - 1) * aCY * x ** (aCY - 1) * lam * 2.0
    want = (-4.0 * (nu - 1.0) - 2.0 * r * dnu) / o.cfg.Re
    got = o.vel_Nz.re[:, 0]
    assert np.max(np.abs(got - want)) < 2e-6 * np.max(np.abs(want))
    assert np.max(np.abs(got - want)[r > 0.2]) < 1e-8 * np.max(np.abs(want))
    assert np.max(np.abs(o.vel_Nr.re)) + np.max(np.abs(o.vel_Nt.re)) < 1e-9 * np.max(np.abs(want))
    assert np.max(np.abs(o.vel_Nz.re[:, 1:])) + np.max(np.abs(o.vel_Nz.im)) < 1e-9 * np.max(np.abs(want))


def test_coriolis_on_laminar_flow_is_the_analytic_force():
    """For Hagen-Poiseuille flow alone the Coriolis force -1/(4 Ro) Omega x U z
    has only the m = 1, k = 0 mode: N_r = (1/2) d sin(phi) U i, N_t =
    -(1/2) d sin(phi) U, with d = -1/(4 Ro), Ro = Re Ek0 (e^{+i theta}
    coefficients of -d sin(phi) U sin(theta) and -d sin(phi) U cos(theta))."""
    import math
    o = oracle_pipe(dict(N=20, K=3, M=3, Mp=1, Re=2000.0, alpha=1.25, dt=0.01))
    o.vel_matrices()
    z = O.Coll.zeros(o.N, o.H)
    o.vel_ur, o.vel_ut, o.vel_uz = z.copy(), z.copy(), z.copy()
    o.vel_transform()
    o.vel_nonlinear()
    N0 = [o.vel_Nr.copy(), o.vel_Nt.copy(), o.vel_Nz.copy()]
    Ek0, phi = 0.5, 0.3
    UO.coriolis(o, Ek0, phi)
    d = -1.0 / (4.0 * o.cfg.Re * Ek0)
    a = 0.5 * d * math.sin(phi) * o.vel_U
    nh = O.mode_index(o.K, 0, 1)
    want_r = O.Coll.zeros(o.N, o.H)
    want_r.im[:, nh] = a
    want_t = O.Coll.zeros(o.N, o.H)
    want_t.re[:, nh] = -a
    tol = 1e-12 * float(np.max(np.abs(a)))
    for got, base, want in ((o.vel_Nr, N0[0], want_r), (o.vel_Nt, N0[1], want_t), (o.vel_Nz, N0[2], z)):
        assert np.max(np.abs(got.re - base.re - want.re)) < tol
        assert np.max(np.abs(got.im - base.im - want.im)) < tol


def test_les_vreman_vanishes_on_laminar_flow():
    """Vreman's invariant P of B = Delta^2 A^T A is zero for a gradient of rank
    one, so for Hagen-Poiseuille flow alone (only dU/dr) nu_t = 0 and, with the
    reference viscosity at 1, the plug-in adds nothing."""
    o = oracle_pipe(dict(N=40, K=3, M=3, Mp=1, Re=2000.0, alpha=1.25, dt=0.01))
    o.vel_matrices()
    z = O.Coll.zeros(o.N, o.H)
    o.vel_Nr, o.vel_Nt, o.vel_Nz = z.copy(), z.copy(), z.copy()
    o.vel_ur, o.vel_ut, o.vel_uz = z.copy(), z.copy(), z.copy()
    les = UO.LES(o, *VREMAN)
    u, S = les.get_nu(o)
    assert np.max(np.abs(les.nu)) == 0.0
    les.update_nonlin_terms(o, u, S)
    assert max(np.max(np.abs(c.re)) + np.max(np.abs(c.im)) for c in (o.vel_Nr, o.vel_Nt, o.vel_Nz)) < 1e-12


def test_les_smagorinsky_on_laminar_flow_matches_the_model():
    """For Hagen-Poiseuille flow alone: the strain rate is |U'| = 2r, u_tau =
    sqrt(2/Re) (the wall derivative of U), so nu_t(r) = vanDr (C_s Delta)^2 2r
    with the van Driest factor 1 - exp(-(Re u_tau (1-r) / A+)^2); the added
    term is axisymmetric and axial only: in the mean mode
    N'_z = (1/Re)(Re nu_t + 1 - nu_r)(-4) - 4 nu_t - 2 r d(nu_t)/dr,
    (curl curl U = 4 z, 2 grad(nu_t).S has S_rz = U'/2 = -r), with the radial
    derivative that of the 9-point finite differences."""
    o = oracle_pipe(dict(N=40, K=3, M=3, Mp=1, Re=2000.0, alpha=1.25, dt=0.01))
    o.vel_matrices()
    z = O.Coll.zeros(o.N, o.H)
    o.vel_Nr, o.vel_Nt, o.vel_Nz = z.copy(), z.copy(), z.copy()
    o.vel_ur, o.vel_ut, o.vel_uz = z.copy(), z.copy(), z.copy()
    les = UO.LES(o, *SMAG)
    u, S = les.get_nu(o)
    r = o.mes_D.r
    Re = o.cfg.Re
    assert les.u_tau == pytest.approx(np.sqrt(2.0 / Re), rel=1e-12)
    Delta = (les.Delta_r * les.Rdth * les.dz) ** (1.0 / 3.0)
    vanDr = 1.0 - np.exp(-(Re * np.sqrt(2.0 / Re) * (1.0 - r) / SMAG[3]) ** 2)
    nut = vanDr * (SMAG[1] * Delta) ** 2 * 2.0 * r
    assert np.max(np.abs(les.nu - nut[:, None, None])) < 1e-12 * np.max(nut)
    les.update_nonlin_terms(o, u, S)
    dnut = o.var_coll_meshmult(o.mes_D.dr[0], O.Coll(nut[:, None] * np.ones((1, o.H)), np.zeros((o.N, o.H)))).re[:, 0]
    want = (1.0 / Re) * (Re * nut + 1.0 - o.vel_nu) * (-4.0) - 4.0 * nut - 2.0 * r * dnut
    got = o.vel_Nz.re[:, 0]
    scale = np.max(np.abs(want))
    assert np.max(np.abs(got - want)) < 1e-10 * scale
    assert np.max(np.abs(o.vel_Nr.re)) + np.max(np.abs(o.vel_Nt.re)) < 1e-10 * scale
    assert np.max(np.abs(o.vel_Nz.re[:, 1:])) + np.max(np.abs(o.vel_Nz.im)) < 1e-10 * scale
