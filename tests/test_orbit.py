"""Newton-Krylov orbit search (newton.f90, NewtonHook.f90, GMRESm.f90).

CPU: the oracle's vector maps pinned by invariants of the reference's
formulas, and the product's host-side GMRES / Newton-hookstep driver (torch
CPU tensors) against the oracle's independent restatement on small dense
problems.  GPU: the device vector maps, dot product, shift directions,
time-T map, getrhs, multJ and a short Newton search against the oracle on
the same seeded state."""
import math

import numpy as np
import pytest
import torch

import orbit_oracle as OO
import pipeflow_oracle as O
from _util import SMALL, device_pipe, oracle_pipe, rel, state_from_dev, state_to_dev

CFG = SMALL[0]  # N=16, K=4, M=4


def _oracle_with_state(cfgd, seed=8, frac=1e-3):
    o = oracle_pipe(cfgd)
    o.vel_matrices()
    st = O.seeded_state(o, seed, frac)
    o.set_state(*st)
    o.vel_imposesym()
    return o, st


# ------------------------------------------------------------------- CPU
def test_vec_roundtrip_and_layout():
    o, _ = _oracle_with_state(CFG)
    scaleU = np.array([0.7, 1.3, 2.1])
    v = np.full(OO.vec_len(o), 5.0)
    OO.rtz2vec(o, o.vel_ur, o.vel_ut, o.vel_uz, scaleU, v)
    assert np.all(v[:8] == 5.0)  # header untouched (newton.f90:593-600 writes from v(9))
    r, t, z = OO.vec2rtz(o, v, scaleU)
    assert O.rel_l2([r, t, z], [o.vel_ur, o.vel_ut, o.vel_uz]) < 1e-15
    # entry (nh, n, c) at 8 + (nh*N + n)*6 + c with the stated multipliers
    N = o.N
    nh, n = 5, 3
    k, m = int(o.kk[nh]), int(o.mm[nh])
    d = math.sqrt(abs(o.mes_D.intrdr[n]))
    w = 4.0 / (4.0 + o.cfg.alpha * abs(k) + o.Mp * abs(m))
    at = 8 + (nh * N + n) * 6
    assert v[at + 2] == pytest.approx(o.vel_ut.re[n, nh] * d * w * scaleU[1], rel=1e-15)
    # the mean mode's u_z is scaled by d(n) alone
    assert v[8 + n * 6 + 4] == pytest.approx(o.vel_uz.re[n, 0] * math.sqrt(abs(o.mes_D.intrdr[n])), rel=1e-15)


def test_shiftdir_is_derivative_of_shift():
    o, _ = _oracle_with_state(CFG)
    scaleU = np.ones(3)
    x = np.zeros(OO.vec_len(o))
    OO.rtz2vec(o, o.vel_ur, o.vel_ut, o.vel_uz, scaleU, x)
    h = 1e-6
    for i in (1, 2):
        s = OO.getshiftdir(o, i, x, scaleU)
        ds = (h, 0.0) if i == 1 else (0.0, h)
        vp, vm = np.zeros_like(x), np.zeros_like(x)
        fp = [o.var_coll_shift(ds[0], ds[1], f) for f in (o.vel_ur, o.vel_ut, o.vel_uz)]
        fm = [o.var_coll_shift(-ds[0], -ds[1], f) for f in (o.vel_ur, o.vel_ut, o.vel_uz)]
        OO.rtz2vec(o, *fp, scaleU, vp)
        OO.rtz2vec(o, *fm, scaleU, vm)
        fd = -(vp - vm) / (2 * h)  # var_coll_shift(d) moves the pattern by -d
        assert rel(s[8:], fd[8:]) < 1e-8


def _toy_problem(n=24, seed=3):
    rng = np.random.default_rng(seed)
    A = np.eye(n) * 3.0 + 0.3 * rng.standard_normal((n, n))
    xs = rng.standard_normal(n)
    b = A @ xs + 0.1 * xs ** 3
    return A, b, xs


def test_gmres_matches_oracle_and_solves():
    from pipeflow.newton import GMRES
    A, b, _ = _toy_problem()
    n = b.size
    x_ref = np.linalg.solve(A, b)
    go = OO.GMRES(n, n)
    xo, res_o, _, its_o, info_o = go.solve(np.zeros(n), b, lambda v: A @ v, lambda a, c: float(a @ c),
                                           1e-12 * np.linalg.norm(b), -1.0, n, 0)
    gp = GMRES(n, n, torch.zeros(n, dtype=torch.float64))
    At = torch.tensor(A)
    xp, res_p, _, its_p, info_p = gp.solve(torch.zeros(n, dtype=torch.float64), torch.tensor(b),
                                           lambda v: At @ v, lambda a, c: float(a @ c),
                                           1e-12 * np.linalg.norm(b), -1.0, n, 0)
    assert its_o == its_p and info_o == info_p == 0
    assert rel(xo, x_ref) < 1e-10
    assert rel(xp.numpy(), xo) < 1e-12
    # hookstep with a trust region smaller than the Newton step
    y_o, pred_o = OO.hookstep(5, go.h, go.beta, 0.1)
    from pipeflow.newton import hookstep
    y_p, pred_p = hookstep(5, gp.h, gp.beta, 0.1)
    assert np.linalg.norm(y_o) <= 0.1 + 1e-12
    assert rel(y_p, y_o) < 1e-12 and abs(pred_p - pred_o) < 1e-12


@pytest.mark.parametrize("delta", [-1.0, 0.05])
def test_newtonhook_matches_oracle_on_toy_problem(delta):
    from pipeflow.newton import newtonhook
    A, b, xs = _toy_problem()
    n = b.size

    def f(x):
        return A @ x + 0.1 * x ** 3 - b

    def df_factory(state, M):
        def df(s):
            x = state.new_x
            return M @ s + 0.3 * (x ** 2) * s
        return df

    class S:
        pass

    so, sp = S(), S()
    ro = OO.newtonhook(f, df_factory(so, A), lambda a, c: float(a @ c), np.zeros(n), 10, 1e-3, 1e-11,
                       delta, 1e-12, 1e3, 40, state=so)
    At, bt = torch.tensor(A), torch.tensor(b)
    rp = newtonhook(lambda x: At @ x + 0.1 * x ** 3 - bt, df_factory(sp, At), lambda a, c: float(a @ c),
                    torch.zeros(n, dtype=torch.float64), 10, 1e-3, 1e-11, delta, 1e-12, 1e3, 40, state=sp)
    assert ro.info == rp.info == 0
    assert ro.nits == rp.nits
    assert rel(ro.x, xs) < 1e-10
    assert rel(rp.x.numpy(), ro.x) < 1e-10
    for a, c in zip(ro.history, rp.history):
        assert a[0] == c[0] and a[1] == c[1]
        assert abs(a[2] - c[2]) <= 1e-9 * max(1.0, abs(a[2]))


# ------------------------------------------------------------------- GPU
def _pair(cfgd, ndts, shifts, seed=8):
    from pipeflow.newton import Orbit
    o, st = _oracle_with_state(cfgd, seed)
    g = device_pipe(cfgd)
    g.vel_matrices()
    state_to_dev(g, st)
    g.vel_imposesym()
    orb = Orbit(g, ndts, shifts)
    oo = OO.Orbit(o, list(ndts))
    oo.new_x = np.zeros(len(ndts) * oo.n)
    for p, s in enumerate(shifts):
        oo.new_x[p * oo.n:p * oo.n + 3] = s
    return o, oo, g, orb


def _np(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


@pytest.mark.gpu
def test_device_vectors_scales_dot_shiftdir():
    o, oo, g, orb = _pair(CFG, [10], [(0.0, 0.4, 0.1)])
    oo.get_scales()
    orb.get_scales()
    assert rel(orb.scaleU, oo.scaleU) < 1e-13
    assert abs(orb.scaleT - oo.scaleT) <= 1e-13 * abs(oo.scaleT)
    x = _np(orb.new_x)
    assert rel(x, oo.new_x) < 1e-13
    assert x[:3] == pytest.approx(oo.new_x[:3], rel=1e-13)
    # dot products, with and without the header
    for n_ in (-1, 1):
        d = orb.dotprod(n_, orb.new_x, orb.new_x)
        assert d == pytest.approx(OO.dotprod(n_, oo.new_x, oo.new_x), rel=1e-14)
    assert orb.dotprod(-1, orb.new_x, orb.new_x) == orb.dotprod(-1, orb.new_x, orb.new_x)
    # vec2rtz then rtz2vec
    orb.vec2rtz(orb.new_x)
    with torch.cuda.stream(orb.stream):
        v = torch.full_like(orb.new_x, 7.0)
    orb.rtz2vec(v)
    vh = _np(v)
    assert np.all(vh[:8] == 7.0)
    assert rel(vh[8:], x[8:]) < 1e-15
    for i in (1, 2):
        s = _np(orb.getshiftdir(i, orb.new_x))
        assert rel(s[8:], OO.getshiftdir(o, i, oo.new_x, oo.scaleU)[8:]) < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("ndts,shifts", [([10], [(0.0, 0.4, 0.1)]), ([6, 4], [(0.0, 0.2, 0.06), (0.0, 0.1, 0.04)])],
                         ids=["ms1", "ms2"])
def test_device_steporbit_and_getrhs(ndts, shifts):
    o, oo, g, orb = _pair(CFG, ndts, shifts)
    oo.get_scales()
    orb.get_scales()
    oo.new_x[:oo.n][8:] = _np(orb.new_x)[8:orb.n]  # identical start vectors
    with torch.cuda.stream(orb.stream):
        orb.new_x.copy_(torch.tensor(oo.new_x, device=orb.dev))
    if len(ndts) > 1:
        oo.new_x[oo.n + 8:] = 0.0
        y = np.zeros(oo.n)
        oo.steporbit(ndts[0], oo.new_x[:oo.n].copy(), y)
        oo.new_x[oo.n + 8:] = y[8:]
        orb.load_ms_states()
        assert rel(_np(orb.new_x)[orb.n + 8:], oo.new_x[oo.n + 8:]) < 1e-11
        with torch.cuda.stream(orb.stream):
            orb.new_x.copy_(torch.tensor(oo.new_x, device=orb.dev))
    t0 = g.tim.t
    fo = oo.getrhs(oo.new_x)
    fg = _np(orb.getrhs(orb.new_x))
    assert np.all(fg.reshape(len(ndts), -1)[:, :8] == 0.0)
    assert rel(fg, fo) < 1e-10
    # time advanced by the whole period; dt = period / ndts of the last point
    assert g.tim.t == pytest.approx(t0 + sum(s[2] for s in shifts), rel=1e-12)
    assert g.tim.dt == pytest.approx(shifts[-1][2] / ndts[-1], rel=1e-14)
    # a single step leaves time and step count alone
    st0 = (g.tim.t, g.tim.step)
    with torch.cuda.stream(orb.stream):
        y = torch.zeros(orb.n, dtype=torch.float64, device=orb.dev)
    orb.steporbit(1, orb.new_x[:orb.n], y)
    assert (g.tim.t, g.tim.step) == st0


@pytest.mark.gpu
def test_device_multJ_and_short_newton_search():
    ndts, shifts = [8], [(0.0, 0.4, 0.08)]
    o, oo, g, orb = _pair(CFG, ndts, shifts)
    oo.get_scales()
    orb.get_scales()
    with torch.cuda.stream(orb.stream):
        orb.new_x.copy_(torch.tensor(oo.new_x, device=orb.dev))
    oo.new_fx = oo.getrhs(oo.new_x)
    orb.new_fx = orb.getrhs(orb.new_x)
    rng = np.random.default_rng(11)
    dx = rng.standard_normal(oo.n) * 1e-2
    jo = oo.multJ(dx)
    jg = _np(orb.multJ(torch.tensor(dx, device=orb.dev)))
    # finite-difference Jacobian: rounding differences of F are divided by
    # eps ~ epsJ |x| / |dx|, so agreement is ~1e-7 of |J dx|
    assert rel(jg, jo) < 1e-5
    assert jg[:3] == pytest.approx(jo[:3], rel=1e-5, abs=1e-12)
    # two Newton iterations with a 4-vector Krylov space
    rg = orb.solve(m=4, nits=2, rel_err=1e-12)
    sd = math.sqrt(oo.dotprod_ms(-1, oo.new_x, oo.new_x))
    ro = OO.newtonhook(oo.getrhs, oo.multJ, lambda a, c: oo.dotprod_ms(1, a, c), oo.new_x, 4, 1e-3,
                       1e-12 * sd, -sd, 1e-7 * sd, 1e7 * sd, 2, state=oo)
    assert rg.info == ro.info and rg.nits == ro.nits == 2
    assert rg.tol == pytest.approx(ro.tol, rel=1e-4)
    assert rg.tol < ro.history[0][2]  # the residual went down
    assert len(orb.history) == 3
    orb.close()


def test_arnoldi_host_logic_finds_leading_eigenpairs():
    """arnold (arnoldi.f) on a dense operator with known spectrum: the
    converged values are the largest-magnitude eigenvalues, in that order,
    and the returned vectors are eigenvectors (Re, Im columns for a pair)."""
    from pipeflow.newton import Arnoldi, logeig
    rng = np.random.default_rng(5)
    n = 40
    lam = np.concatenate([[0.95], [0.9 + 0.2j, 0.9 - 0.2j], rng.uniform(-0.5, 0.5, n - 3)])
    # a real operator with these eigenvalues: 2x2 rotation-scaling block for the pair
    D = np.zeros((n, n))
    D[0, 0] = 0.95
    D[1:3, 1:3] = [[0.9, 0.2], [-0.2, 0.9]]
    for i in range(3, n):
        D[i, i] = lam[i].real
    X = rng.standard_normal((n, n))
    A = X @ D @ np.linalg.inv(X)
    At = torch.tensor(A)
    ar = Arnoldi(n, 40, 2, lambda a, b: float(a @ b), 1e-10, torch.zeros(n, dtype=torch.float64))
    sv = torch.tensor(rng.standard_normal(n))
    while True:
        ifail, sv = ar.step(sv)
        if ifail != 0:
            break
        sv = At @ sv
    assert ifail == -1
    got = ar.wr2 + 1j * ar.wi2
    assert abs(got[0] - 0.95) < 1e-9
    assert abs(got[1] - (0.9 + 0.2j)) < 1e-9
    b = ar.b.numpy()
    assert b.shape == (3, n)
    assert np.linalg.norm(A @ b[0] - 0.95 * b[0]) < 1e-8 * np.linalg.norm(b[0])
    v = b[1] + 1j * b[2]
    assert np.linalg.norm(A @ v - (0.9 + 0.2j) * v) < 1e-8 * np.linalg.norm(v)
    sr, si = logeig(ar.wr2, ar.wi2, 2.0)
    assert sr[1] == pytest.approx(math.log(abs(0.9 + 0.2j)) / 2.0, rel=1e-9)
    assert si[1] == pytest.approx(math.atan2(0.2, 0.9) / 2.0, rel=1e-9)


@pytest.mark.gpu
def test_device_floquet_spectrum_matches_dense_linear_map():
    """get_eigen (Arnoldi on multA, newton.f90:868-979) about a 1e-12-energy
    state, i.e. about laminar flow to first order: the converged Floquet
    multipliers of the 50-step map are eigenvalues of the 50th power of the
    oracle's dense linearised one-step map (all modes, 6NH x 6NH), the
    leading one the largest.  Re = 100 and T = 0.5 keep the leading
    multipliers apart, so the reference's stopping rule (successive Ritz
    values within min(rel_err, gtol)) stops on converged values."""
    import pipeflow as P
    from pipeflow.newton import Orbit
    cfgd = dict(N=16, K=2, M=2, Re=100.0, alpha=1.0, dt=0.01)
    o = oracle_pipe(cfgd)
    o.vel_matrices()
    N, H = o.N, o.H
    ns = 6 * N * H
    eps = 1e-8

    def unpack(vec):
        a = vec.reshape(3, 2, N, H)
        return [O.Coll(a[c, 0].copy(), a[c, 1].copy()) for c in range(3)]

    def pack(st):
        return np.concatenate([np.concatenate([f.re.ravel(), f.im.ravel()]) for f in st])

    J = np.empty((ns, ns))
    for i in range(ns):
        e = np.zeros(ns)
        e[i] = eps
        o.set_state(*unpack(e))
        o.timestep(orbit=True)
        J[:, i] = pack(o.state()) / eps
    mu = np.linalg.eigvals(J) ** 50
    g = device_pipe(cfgd)
    g.vel_matrices()
    P.seeded_state(g, 3, 1e-12)
    orb = Orbit(g, [50], [(0.0, 0.0, 0.5)])
    orb.set_scales([1.0, 1.0, 1.0], 1.0)
    orb.rtz2vec(orb.new_x)
    res = orb.get_eigen(m=80, ncgd=2)
    assert res["status"] == "converged"
    wr, wi = res["multipliers"]
    lams = wr + 1j * wi
    assert abs(lams[0] - mu[np.argmax(np.abs(mu))]) < 1e-6 * abs(lams[0])
    for lam in lams[1:]:
        assert np.min(np.abs(mu - lam)) < 1e-4 * abs(lam)
    sr, _ = res["exponents"]
    assert sr[0] == pytest.approx(math.log(abs(lams[0])) / 0.5, rel=1e-12)
    assert res["eigvecs"] is not None
    orb.close()


@pytest.mark.gpu
def test_device_continuation_in_re():
    """Parameter continuation (newton.f90:89-170, 730-735): the start sets
    new_x = x1 + ctdp0 (x2 - x1) with the parameter entries over ctpsc,
    steporbit runs at Re = x[3]*ctpsc (against an oracle pipe built at that
    Re), and multJ's fourth row is dotprod(ctstp, x)."""
    from pipeflow.newton import Orbit
    ndts, shifts = [6], [(0.0, 0.3, 0.06)]
    o, st = _oracle_with_state(CFG)
    g = device_pipe(CFG)
    g.vel_matrices()
    state_to_dev(g, st)
    g.vel_imposesym()
    orb = Orbit(g, ndts, shifts, continuation=dict(param="Re", ctdp0=0.5, ctntmn=3, ctntmx=8))
    orb.set_scales([1.0, 1.0, 1.0], 1.0)
    orb.rtz2vec(orb.new_x)
    x1 = _np(orb.new_x).copy()
    assert x1[3] == CFG["Re"]
    d = float(np.dot(x1[8:], x1[8:]))
    x2 = x1.copy()
    x2[3] = CFG["Re"] + 100.0
    x2[8:] *= 1.01
    orb.start_continuation(torch.tensor(x2, device=orb.dev))
    ctpsc = CFG["Re"] / math.sqrt(d)
    assert orb.ctpsc == pytest.approx(ctpsc, rel=1e-12)
    want = x2 + 0.5 * (x2 - x1)
    want[3] /= ctpsc
    assert rel(_np(orb.new_x), want) < 1e-14
    # the time-T map at the parameter the vector carries
    Re2 = float(_np(orb.new_x)[3]) * ctpsc
    y = torch.zeros_like(orb.new_x)
    orb.steporbit(ndts[0], orb.new_x, y)
    assert g.cfg.Re == pytest.approx(Re2, rel=1e-14)
    o2 = oracle_pipe(dict(CFG, Re=Re2))
    oo = OO.Orbit(o2, list(ndts))
    oo.scaleU, oo.scaleT = np.ones(3), 1.0
    yo = np.zeros(oo.n)
    oo.steporbit(ndts[0], _np(orb.new_x), yo)
    assert rel(_np(y)[8:], yo[8:]) < 1e-10
    # the parameter row of the Jacobian
    orb.new_fx = orb.getrhs(orb.new_x)
    dx = torch.tensor(np.random.default_rng(4).standard_normal(orb.n) * 1e-3, device=orb.dev)
    jx = _np(orb.multJ(dx))
    assert jx[3] == pytest.approx(float(_np(orb.ctstp) @ _np(dx)), rel=1e-12)
    orb.close()


def test_continuation_arithmetic():
    """newton.f90:102-117 and 155-170 on host tensors: the start from two
    solutions, the scaled parameter entries, the step-size rule and the
    fixed-period rescaling."""
    from pipeflow.newton import continuation_next, continuation_start
    n, ms = 12, 2
    rng = np.random.default_rng(7)
    x1 = rng.standard_normal(n * ms)
    x2 = x1 + 0.1 * rng.standard_normal(n * ms)
    x1[3::n] = 2000.0
    x2[3::n] = 2100.0
    d = 4.0
    nx, st, cx, ctpsc = continuation_start(torch.tensor(x1), torch.tensor(x2), n, ms, 0.25, 2000.0, d)
    assert ctpsc == 2000.0 / 2.0
    want_st = x2 - x1
    want_nx = x2 + 0.25 * want_st
    want_cx = x2.copy()
    for w in (want_st, want_nx, want_cx):
        w[3::n] /= ctpsc
    assert np.allclose(st.numpy(), want_st, rtol=0, atol=1e-14)
    assert np.allclose(nx.numpy(), want_nx, rtol=0, atol=1e-12)
    assert np.array_equal(cx.numpy(), want_cx)
    # equal solutions: a unit step in the parameter
    _, st0, _, _ = continuation_start(torch.tensor(x1), torch.tensor(x1), n, ms, 0.25, 2000.0, d)
    assert np.array_equal(st0.numpy()[3::n], np.full(ms, 1.0 / ctpsc))
    # step rule: 1.1, 0.5 above ctntmx Newton iterations, 2 below ctntmn
    for nits, f in ((5, 1.1), (9, 0.5), (2, 2.0)):
        a, s, c, nd = continuation_next(torch.tensor(x2), torch.tensor(x1), nits, 50, 3, 8, n, ms, [100, 50],
                                        False, 150)
        assert np.allclose(a.numpy(), x2 + f * (x2 - x1), rtol=0, atol=1e-12)
        assert np.array_equal(c.numpy(), x2) and nd == [100, 50]
    # fixed period: GMRES iterations above 2m/3 double the steps per period and the times
    a, s, c, nd = continuation_next(torch.tensor(x2), torch.tensor(x1), 5, 120, 3, 8, n, ms, [100, 51], True, 150)
    assert nd == [200, 102]
    want = x2 + 1.1 * (x2 - x1)
    for p in range(ms):
        want[p * n:p * n + 3] *= 2.0
    assert np.allclose(a.numpy(), want, rtol=0, atol=1e-12)
    assert np.allclose(c.numpy()[0:3], 2.0 * x2[0:3], rtol=0, atol=1e-15)
