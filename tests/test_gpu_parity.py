"""Per-routine parity of the CUDA path (through the C ABI) against the FP64
oracle on identical seeded inputs.  Tolerances are relative L2 unless noted;
FP64 routines are held to ~1e-13, i.e. rounding-order differences only."""
import numpy as np
import pytest

import pipeflow_oracle as O
from _util import (CFG1, SMALL, device_pipe, from_dev, oracle_pipe, rand_coll, rel, rel_coll,
                   state_from_dev, state_to_dev, to_dev)

pytestmark = pytest.mark.gpu
CASES = SMALL + [CFG1]
TOL = 1e-13


@pytest.fixture(params=range(len(CASES)), ids=lambda i: "N{N}K{K}M{M}Mp{Mp}".format(**CASES[i]))
def pair(request):
    cfgd = CASES[request.param]
    return oracle_pipe(cfgd), device_pipe(cfgd)


def test_mesh(pair):
    o, g = pair
    m = g.mes_D()
    D = o.mes_D
    assert rel(m["r"], D.r) < 1e-15
    for i in range(O.KL):
        assert rel(m["dr"][i].T, D.dr[i]) < 1e-11
    assert rel(m["radLap"].T, D.radLap) < 1e-11
    assert rel(m["intrdr"], D.intrdr) < 1e-13


def test_coll_roundtrip_and_algebra(pair):
    o, g = pair
    rng = np.random.default_rng(1)
    a, b = rand_coll(o.N, o.H, rng), rand_coll(o.N, o.H, rng)
    da, db = to_dev(g, a), to_dev(g, b)
    assert rel_coll(from_dev(da), a) == 0.0
    g.var_coll_add(da, db)
    assert rel_coll(from_dev(db), O.Coll(a.re + b.re, a.im + b.im)) == 0.0
    g.var_coll_dmult(0.5, db)
    assert rel_coll(from_dev(db), O.Coll(0.5 * (a.re + b.re), 0.5 * (a.im + b.im))) == 0.0


def test_meshmult_curl_grad_div(pair):
    o, g = pair
    rng = np.random.default_rng(2)
    r, t, z = (rand_coll(o.N, o.H, rng) for _ in range(3))
    dr, dt, dz = to_dev(g, r), to_dev(g, t), to_dev(g, z)
    out = [g.coll() for _ in range(3)]
    for p in range(1, O.KL + 1):
        g.var_coll_meshmult(p, dr, out[0])
        assert rel_coll(from_dev(out[0]), o.var_coll_meshmult(o.mes_D.dr[p - 1], r)) < TOL
    g.var_coll_curl(dr, dt, dz, *out)
    for got, ref in zip(out, o.var_coll_curl(r, t, z)):
        assert rel_coll(from_dev(got), ref) < TOL
    g.var_coll_grad(dr, *out)
    for got, ref in zip(out, o.var_coll_grad(r)):
        assert rel_coll(from_dev(got), ref) < TOL
    g.var_coll_div(dr, dt, dz, out[0])
    assert rel_coll(from_dev(out[0]), o.var_coll_div(r, t, z)) < TOL
    # in-place use: curl(u) written over u (copy-in semantics)
    g.var_coll_curl(dr, dt, dz, dr, dt, dz)
    for got, ref in zip((dr, dt, dz), o.var_coll_curl(r, t, z)):
        assert rel_coll(from_dev(got), ref) < TOL


def test_transforms(pair):
    o, g = pair
    rng = np.random.default_rng(3)
    c = rand_coll(o.N, o.H, rng)
    dc = to_dev(g, c)
    p = g.phys()
    g.tra_coll2phys(dc, p)
    ref = o.tra_spec2phys(c)
    assert rel(p.download(), ref) < TOL
    phys = rng.standard_normal((o.N, o.cfg.Th, o.cfg.Z))
    dp = g.phys(phys)
    out = g.coll()
    g.tra_phys2coll(dp, out)
    assert rel_coll(from_dev(out), o.tra_phys2spec(phys)) < TOL


def test_lumesh_factor_and_solve(pair):
    o, g = pair
    rng = np.random.default_rng(4)
    for PM, BC, c1, c2 in ((0, 1, 0.0, 1.0), (1, 0, 100.0, -0.51 / 2000), (-1, 0, 50.0, -2e-4),
                           (0, 0, 100.0, -0.51 / 2000)):
        ref_AB, ref_piv = o.tim_lumesh_init(PM, BC, c1, c2)
        A = g.tim_lumesh_init(PM, BC, c1, c2)
        M, piv = A.download()
        for nh in range(o.H):
            if BC == 1 and nh == 0:
                continue
            assert np.array_equal(piv[nh] - 1, ref_piv[nh]), (PM, BC, nh)
            assert rel(M[nh].T, ref_AB[nh]) < 1e-13
        b = rand_coll(o.N, o.H, rng)
        db = to_dev(g, b)
        g.tim_lumesh_invert(BC, A, db)
        x = b.copy()
        o.tim_lumesh_invert(BC, (ref_AB, ref_piv), x)
        assert rel_coll(from_dev(db), x) < 1e-12


def test_tim_meshmult(pair):
    o, g = pair
    rng = np.random.default_rng(5)
    b, c = rand_coll(o.N, o.H, rng), rand_coll(o.N, o.H, rng)
    for PM in (-1, 0, 1):
        A = g.tim_mesh_init(PM, 100.0, 2.5e-4)
        ref = o.tim_meshmult(o.tim_mesh_init(PM, 100.0, 2.5e-4), b, c)
        d = g.coll()
        g.tim_meshmult(1, A, to_dev(g, b), to_dev(g, c), d)
        assert rel_coll(from_dev(d), ref) < TOL
        off, diag = o.tim_mesh_init(PM, 100.0, 2.5e-4)
        M = A.download()
        assert rel(M[:, :, O.KL], diag.T) < 1e-15


def test_norm_symmetry_shift(pair):
    o, g = pair
    rng = np.random.default_rng(6)
    r, t, z = (rand_coll(o.N, o.H, rng) for _ in range(3))
    E, Ek, Em = g.var_coll_norm(to_dev(g, r))
    Er, Ekr, Emr = o.var_coll_norm(r)
    assert abs(E - Er) < 1e-13 * Er and rel(Ek, Ekr) < 1e-13 and rel(Em, Emr) < 1e-13
    for i in (0, 1, 2, 3):
        dr, dt, dz = to_dev(g, r), to_dev(g, t), to_dev(g, z)
        g.var_imposesym(i, dr, dt, dz)
        rr, tt, zz = r.copy(), t.copy(), z.copy()
        o.var_imposesym(i, rr, tt, zz)
        for got, ref in zip((dr, dt, dz), (rr, tt, zz)):
            assert rel_coll(from_dev(got), ref) < 1e-15
    out = g.coll()
    g.var_coll_shift(0.3, 1.1, to_dev(g, r), out)
    assert rel_coll(from_dev(out), o.var_coll_shift(0.3, 1.1, r)) < 1e-14


def test_influence_matrices(pair):
    o, g = pair
    o.vel_matrices()
    g.vel_matrices()
    U, A = g.influence()
    for c in range(3):
        assert rel(U[c].T, o._U[c]) < 1e-12
    # columns 4-6 are gradients of the Neumann pressure solution (LNp), whose
    # near-singular low-k systems amplify rounding by their condition number
    for c in range(3, 6):
        assert rel(U[c].T, o._U[c]) < 1e-10
    assert rel(A[1:], o._A[1:]) < 1e-10


def test_transform_nonlinear_predictor_corrector(pair):
    o, g = pair
    o.vel_matrices()
    g.vel_matrices()
    st = O.seeded_state(o, 11, 1e-3)
    o.set_state(*st)
    state_to_dev(g, st)
    o.vel_transform()
    g.vel_transform()
    for i, name in enumerate(("r", "t", "z", "curlr", "curlt", "curlz")):
        assert rel(g.vel_physfield(i).download(), o.phys[name]) < TOL
    o.vel_nonlinear()
    g.vel_nonlinear()
    for i, ref in enumerate((o.vel_Nr, o.vel_Nt, o.vel_Nz)):
        assert rel_coll(from_dev(g.vel_field(3 + i)), ref) < 1e-12
    assert abs(g.vel_Pr0 - o.vel_Pr0) <= 1e-12 * max(1.0, abs(o.vel_Pr0))
    o.vel_predictor()
    g.vel_predictor()
    for got, ref in zip(state_from_dev(g), o.state()):
        assert rel_coll(got, ref) < 1e-12
    o.vel_transform(); o.vel_nonlinear(); o.vel_corrector()
    g.vel_transform(); g.vel_nonlinear(); g.vel_corrector()
    for got, ref in zip(state_from_dev(g), o.state()):
        assert rel_coll(got, ref) < 1e-12
    assert abs(g.tim.dterr - o.tim_dterr) <= 1e-9 * o.tim_dterr


def test_hagen_poiseuille_preserved_exactly():
    g = device_pipe(CFG1)
    g.vel_matrices()
    for _ in range(3):
        g.timestep()
    for re, im in g.get_state():
        assert np.all(re == 0.0) and np.all(im == 0.0)


def test_one_step_parity_cfg1():
    o, g = oracle_pipe(CFG1), device_pipe(CFG1)
    o.vel_matrices()
    g.vel_matrices()
    st = O.seeded_state(o, 1, 1e-3)
    o.set_state(*st)
    state_to_dev(g, st)
    nco = o.timestep()
    ncg = g.timestep()
    assert nco == ncg
    err = O.rel_l2(state_from_dev(g), o.state())
    assert err <= 1e-12, err


@pytest.mark.slow
def test_hundred_step_parity_cfg1():
    o, g = oracle_pipe(CFG1), device_pipe(CFG1)
    o.vel_matrices()
    g.vel_matrices()
    st = O.seeded_state(o, 1, 1e-3)
    o.set_state(*st)
    state_to_dev(g, st)
    for _ in range(100):
        o.timestep()
        g.timestep()
    err = O.rel_l2(state_from_dev(g), o.state())
    assert err <= 1e-9, err
    assert abs(g.energy() - o.energy()) <= 1e-9 * o.energy()
    fr_g, fr_o = g.friction(), o.friction()
    assert abs(fr_g[2] - fr_o[2]) <= 1e-9 * fr_o[2]


def test_noslip_flux_after_steps():
    g = device_pipe(CFG1)
    g.vel_matrices()
    import pipeflow as P
    P.seeded_state(g, 5, 1e-3)
    for _ in range(3):
        g.timestep()
    st = g.get_state()
    scale = max(np.abs(re).max() + np.abs(im).max() for re, im in st)
    for re, im in st:
        assert np.max(np.abs(re[-1])) < 1e-13 * scale and np.max(np.abs(im[-1])) < 1e-13 * scale
    intrdr = g.mes_D()["intrdr"]
    assert abs(2.0 * st[2][0][:, 0] @ intrdr) < 1e-14 * scale


def test_device_seeded_state_matches_oracle():
    import pipeflow as P
    o, g = oracle_pipe(CFG1), device_pipe(CFG1)
    P.seeded_state(g, 9, 1e-3)
    err = O.rel_l2(state_from_dev(g), O.seeded_state(o, 9, 1e-3))
    assert err < 1e-13
    assert abs(g.energy() - 1e-3 * np.pi ** 2 / (3 * 1.25)) < 1e-15


FALLBACK = dict(N=18, K=7, M=3, Mp=1, Re=2500.0, alpha=1.1, dt=0.01)  # Z=21, Th=9: generic transform path


@pytest.mark.parametrize("cfgd", SMALL + [FALLBACK], ids=lambda c: "N{N}K{K}M{M}".format(**c))
def test_timestep_driver_parity(cfgd):
    o, g = oracle_pipe(cfgd), device_pipe(cfgd)
    o.vel_matrices()
    g.vel_matrices()
    st = O.seeded_state(o, 4, 1e-3)
    o.set_state(*st)
    state_to_dev(g, st)
    for _ in range(3):
        assert o.timestep() == g.timestep()
    assert O.rel_l2(state_from_dev(g), o.state()) <= 1e-12
    assert abs(g.vel_Pr0 - o.vel_Pr0) <= 1e-12 * max(1.0, abs(o.vel_Pr0))


@pytest.mark.parametrize("cfgd", [SMALL[0], CFG1], ids=["small", "cfg1"])
def test_steporbit_parity(cfgd):
    o, g = oracle_pipe(cfgd), device_pipe(cfgd)
    o.vel_matrices()
    g.vel_matrices()
    st = O.seeded_state(o, 8, 1e-3)
    o.set_state(*st)
    state_to_dev(g, st)
    for _ in range(4):
        o.timestep(orbit=True)
    g.steporbit(4)
    assert O.rel_l2(state_from_dev(g), o.state()) <= 1e-12


def test_multi_corrector_graph_path_parity():
    """A tight corrector tolerance forces several corrector passes per step,
    exercising the replayed corrector graphs at both pointer parities."""
    cfgd = dict(SMALL[0], dterr=1e-9)
    o, g = oracle_pipe(cfgd), device_pipe(cfgd)
    o.vel_matrices()
    g.vel_matrices()
    st = O.seeded_state(o, 6, 1e-2)
    o.set_state(*st)
    state_to_dev(g, st)
    counts = []
    for _ in range(4):
        nco = o.timestep()
        ncg = g.timestep()
        assert nco == ncg
        counts.append(ncg)
    assert max(counts) >= 2
    assert O.rel_l2(state_from_dev(g), o.state()) <= 1e-12
    assert g.launches() > 0


PIVOTING = dict(N=64, K=4, M=4, Mp=1, Re=1900.0, alpha=1.2, dt=0.01)  # Helmholtz factors pivot


def test_pivoting_helmholtz_fused_path_parity():
    """At N=64 and Re~1900 dgbtrf pivots in the u+-/uz systems too; the fused
    step then uses the pivoting sweep for them."""
    o, g = oracle_pipe(PIVOTING), device_pipe(PIVOTING)
    o.vel_matrices()
    g.vel_matrices()
    for lu in (o.LDp, o.LDm, o.LDz):
        assert (lu[1] != np.arange(o.N)[None, :]).any()
    st = O.seeded_state(o, 12, 1e-3)
    o.set_state(*st)
    state_to_dev(g, st)
    for _ in range(5):
        assert o.timestep() == g.timestep()
    assert O.rel_l2(state_from_dev(g), o.state()) <= 1e-12
    o.vel_predictor()
    g.vel_predictor()
    assert O.rel_l2(state_from_dev(g), o.state()) <= 1e-12


def test_adaptive_dt_parity():
    """Variable dt (main.f90:24-29): vel_maxtstep, tim_new_tstep and the
    re-factorisation on a dt change follow the oracle step for step."""
    cfgd = dict(SMALL[0], dt=-1.0, maxdt=0.01, courant=0.5)
    o, g = oracle_pipe(cfgd), device_pipe(cfgd)
    o.tim_dt = 0.004
    t = g.tim
    t.dt = 0.004
    g.set_tim(t)
    o.vel_matrices()
    g.vel_matrices()
    st = O.seeded_state(o, 11, 1e-3)
    o.set_state(*st)
    state_to_dev(g, st)
    dts = [g.tim.dt]
    for _ in range(6):
        assert o.timestep() == g.timestep()
        assert abs(g.tim.dt - o.tim_dt) <= 1e-15 * o.tim_dt
        dts.append(g.tim.dt)
    assert len(set(dts)) > 1  # dt did change
    assert O.rel_l2(state_from_dev(g), o.state()) <= 1e-12


def test_device_path_matches_golden_fixtures():
    """The device timestep against the committed oracle fixtures
    (tests/golden/oracle_small.json, made by tests/golden/make_golden.py)."""
    import json
    from pathlib import Path
    gold = json.loads((Path(__file__).parent / "golden" / "oracle_small.json").read_text())
    for case in gold["cases"]:
        o = oracle_pipe(case["cfg"])
        st = O.seeded_state(o, case["seed"], case["energy"])
        g = device_pipe(case["cfg"])
        g.vel_matrices()
        state_to_dev(g, st)
        ncorr = [g.timestep() for _ in range(case["steps"])]
        assert ncorr == case["ncorr"]
        assert abs(g.energy() - case["energy_after"]) <= 1e-12 * case["energy_after"]
        (urr, uri), (utr, uti), (uzr, uzi) = g.get_state()
        for name, (re, im) in (("ur", (urr, uri)), ("ut", (utr, uti)), ("uz", (uzr, uzi))):
            cs = case["checksums"][name]
            assert abs(float(np.sum(re)) - cs[0]) <= 1e-10 * max(1.0, abs(cs[0]))
            assert abs(float(np.sum(im)) - cs[1]) <= 1e-10 * max(1.0, abs(cs[1]))
        prof = np.array(case["uz_mean_profile"])
        assert np.max(np.abs(uzr[:, 0] - prof)) <= 1e-12 * np.max(np.abs(prof))
        K = case["cfg"]["K"]
        nh11 = (2 * K - 1) + (K - 1) + 1
        m11 = np.array(case["ur_mode11"])
        assert np.max(np.abs(urr[:, nh11] - m11[:, 0])) <= 1e-10 * np.max(np.abs(m11))
        assert np.max(np.abs(uri[:, nh11] - m11[:, 1])) <= 1e-10 * np.max(np.abs(m11))


def test_linear_decay_rate_matches_oracle_eigenvalue():
    """A 1e-8 perturbation of one (k, m) mode, stepped on the device, decays
    at the rate of the leading eigenvalue of the oracle's linearised one-step
    map (dense, 6N x 6N, built column by column from oracle steps)."""
    import math
    cfgd = dict(N=16, K=2, M=2, Re=500.0, alpha=1.0, dt=0.01)
    o = oracle_pipe(cfgd)
    o.vel_matrices()
    nh, N = 4, o.N  # (k=1, m=1) in the H=5 ordering (0,0),(1,0),(-1,1),(0,1),(1,1)
    eps = 1e-8

    def pack(st):
        out = np.empty(6 * N)
        for c, f in enumerate(st):
            out[c * 2 * N: c * 2 * N + N] = f.re[:, nh]
            out[c * 2 * N + N: (c + 1) * 2 * N] = f.im[:, nh]
        return out

    def unpack(vec):
        st = [O.Coll.zeros(N, o.H) for _ in range(3)]
        for c in range(3):
            st[c].re[:, nh] = vec[c * 2 * N: c * 2 * N + N]
            st[c].im[:, nh] = vec[c * 2 * N + N: (c + 1) * 2 * N]
        return st

    def oracle_step(vec):
        o.set_state(*unpack(vec))
        o.timestep(orbit=True)
        return pack(o.state())

    n = 6 * N
    J = np.empty((n, n))
    for i in range(n):
        e = np.zeros(n)
        e[i] = eps
        J[:, i] = oracle_step(e) / eps
    w, V = np.linalg.eig(J)
    lead = np.argmax(np.abs(w))
    rate = math.log(abs(w[lead])) / cfgd["dt"]
    vec = V[:, lead] / np.linalg.norm(V[:, lead])
    g = device_pipe(cfgd)
    g.vel_matrices()
    norms = []
    for part in (np.real(vec), np.imag(vec)):
        state_to_dev(g, unpack(eps * part))
        n0 = np.linalg.norm(eps * part)
        g.steporbit(20)
        st = state_from_dev(g)
        norms.append((n0, np.linalg.norm(pack(st))))
    n0 = math.sqrt(sum(a * a for a, _ in norms))
    n1 = math.sqrt(sum(b * b for _, b in norms))
    measured = math.log(n1 / n0) / (20 * cfgd["dt"])
    assert rate < 0
    assert abs(measured - rate) < 1e-3 * abs(rate) + 1e-6
