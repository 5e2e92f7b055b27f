"""Known-answer checks that pin the CPU oracle (no GPU needed).

The reference ships no tests or golden data, so the oracle is pinned by
invariants that follow from the reference's own code: FD weights exact on
polynomials (meshs.f90:149-159), FFT round trip (transform.fftw3.f90),
Hagen-Poiseuille preservation (velocity.f90:338-361), no-slip to machine
precision (velocity.f90:238-256), zero perturbation mean flux
(velocity.f90:152-177), a convergent divergence, banded LU == dense solve,
and the committed golden fixtures (tests/golden/).
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest

import pipeflow_oracle as O
from _util import SMALL, oracle_pipe, rand_coll

GOLDEN = Path(__file__).resolve().parent / "golden"


def _band_apply(band, f):
    N = len(f)
    out = np.zeros(N)
    for j in range(N):
        for n in range(max(0, j - O.KL), min(j + O.KL, N - 1) + 1):
            out[n] += band[O.KL + n - j, j] * f[j]
    return out


@pytest.mark.parametrize("N", [12, 24, 40])
def test_fd_weights_exact_on_local_polynomials(N):
    D = O.mes_rdom_init(O.default_mesh(N))
    x = D.r
    for i in range(1, O.KL + 1):
        for deg in range(0, 2 * O.KL + 1):
            f = x ** deg
            d = _band_apply(D.dr[i - 1], f)
            exact = (math.factorial(deg) / math.factorial(deg - i)) * x ** (deg - i) if deg >= i else 0 * x
            for n in range(N):
                nn = min(n + O.KL, N - 1) - max(0, n - O.KL) + 1
                if deg < nn:  # the stencil at row n is exact up to degree nn-1
                    assert abs(d[n] - exact[n]) <= 1e-7 * max(1.0, abs(exact[n])) * 10 ** i


def test_axis_and_wall_extrapolation_weights():
    D = O.mes_rdom_init(O.default_mesh(32))
    x0 = D.r[:O.KL + 1]
    x1 = D.r[-O.KL - 1:]
    for deg in range(O.KL + 1):
        assert abs(D.dr0[:, 0] @ x0 ** deg - (1.0 if deg == 0 else 0.0)) < 1e-12
        assert abs(D.dr1[:, 0] @ x1 ** deg - 1.0) < 1e-12
        assert abs(D.dr1[:, 1] @ x1 ** deg - deg) < 1e-9


def test_intrdr_integrates_r_dr():
    D = O.mes_rdom_init(O.default_mesh(64))
    assert abs(D.intrdr.sum() - 0.5) < 1e-12          # int_0^1 r dr
    assert abs(D.intrdr @ D.r ** 2 - 0.25) < 2e-3      # int_0^1 r^3 dr


def test_default_mesh_endpoints():
    for N in (16, 40, 64):
        r = O.default_mesh(N)
        assert abs(r[-1] - 1.0) < 1e-14
        assert r[0] > 0 and np.all(np.diff(r) > 0)


@pytest.mark.parametrize("cfgd", SMALL)
def test_fft_round_trip(cfgd):
    p = oracle_pipe(cfgd)
    rng = np.random.default_rng(0)
    c = rand_coll(p.N, p.H, rng)
    p.var_imposesym(0, c, O.Coll.zeros(p.N, p.H), O.Coll.zeros(p.N, p.H))
    c.im[:, 0] = 0.0
    back = p.tra_phys2spec(p.tra_spec2phys(c))
    assert np.max(np.abs(back.re - c.re)) < 1e-13
    assert np.max(np.abs(back.im - c.im)) < 1e-13


@pytest.mark.parametrize("cfgd", SMALL)
def test_banded_lu_matches_dense_solve(cfgd):
    p = oracle_pipe(cfgd)
    c1, c2 = 1.0 / p.cfg.dt, -0.51 / p.cfg.Re
    AB, ipiv = p.tim_lumesh_init(1, 0, c1, c2)
    rng = np.random.default_rng(1)
    b = rand_coll(p.N, p.H, rng)
    x = b.copy()
    p.tim_lumesh_invert(0, (AB, ipiv), x)
    # rebuild the dense matrix of mode nh and check A x = b
    D = p.mes_D
    for nh in (0, p.H // 2, p.H - 1):
        k, m = int(p.kk[nh]), int(p.mm[nh])
        A = np.zeros((p.N, p.N))
        d = p._dvec(1)[:, nh]
        for j in range(p.N):
            for n in range(max(0, j - O.KL), min(j + O.KL, p.N - 1) + 1):
                A[n, j] = c2 * D.radLap[O.KL + n - j, j]
            A[j, j] += c2 * d[j] + c1
        S = (m * p.Mp + 1) % 2
        A[0, :] = 0.0
        A[0, :O.KL + 1] = D.dr0[:, 1 - S]
        A[-1, :] = 0.0
        A[-1, -O.KL - 1:] = D.dr1[:, 0]
        assert np.max(np.abs(A @ x.re[:, nh] - b.re[:, nh])) < 1e-9 * np.max(np.abs(A))
        assert np.max(np.abs(A @ x.im[:, nh] - b.im[:, nh])) < 1e-9 * np.max(np.abs(A))


@pytest.mark.parametrize("cfgd", SMALL)
def test_hagen_poiseuille_preserved_exactly(cfgd):
    p = oracle_pipe(cfgd)
    p.vel_matrices()
    for _ in range(3):
        p.timestep()
    for f in p.state():
        assert np.all(f.re == 0.0) and np.all(f.im == 0.0)


@pytest.mark.parametrize("cfgd", SMALL)
def test_step_noslip_flux_and_symmetry(cfgd):
    p = oracle_pipe(cfgd)
    p.vel_matrices()
    p.set_state(*O.seeded_state(p, 3, 1e-3))
    for _ in range(2):
        p.timestep()
    ur, ut, uz = p.state()
    scale = max(np.abs(f.re).max() + np.abs(f.im).max() for f in (ur, ut, uz))
    for f in (ur, ut, uz):
        assert np.max(np.abs(f.re[-1])) < 1e-13 * scale
        assert np.max(np.abs(f.im[-1])) < 1e-13 * scale
    if p.cfg.const_flux:
        assert abs(2.0 * uz.re[:, 0] @ p.mes_D.intrdr) < 1e-14 * scale
    assert np.all(ur.re[:, 0] == 0) and np.all(ur.im[:, 0] == 0)
    assert np.all(ut.im[:, 0] == 0) and np.all(uz.im[:, 0] == 0)


def test_divergence_converges_with_N():
    errs = []
    for N in (16, 32, 64):
        p = oracle_pipe(dict(N=N, K=4, M=4, Re=2000.0, alpha=1.25, dt=0.01))
        p.vel_matrices()
        p.set_state(*O.seeded_state(p, 1, 1e-3))
        p.timestep()
        ur, ut, uz = p.state()
        dv = p.var_coll_div(ur, ut, uz)
        w = p.mes_D.intrdr[:, None]
        g = p.var_coll_meshmult(p.mes_D.dr[0], ur)
        errs.append(math.sqrt(np.sum(w * (dv.re ** 2 + dv.im ** 2)) / np.sum(w * (g.re ** 2 + g.im ** 2))))
    assert errs[1] < errs[0] and errs[2] < errs[1] and errs[2] < 1e-4


def test_decay_rate_matches_linear_operator():
    """A 1e-8 perturbation of one (k,m) mode decays at the leading eigenvalue
    of the linearised one-step map (dense, built from the oracle itself)."""
    cfgd = dict(N=16, K=2, M=2, Re=500.0, alpha=1.0, dt=0.01)
    p = oracle_pipe(cfgd)
    p.vel_matrices()
    nh = 2  # (k=1, m=1)... the H=5 ordering: (0,0),(1,0),(-1,1),(0,1),(1,1)
    base = [O.Coll.zeros(p.N, p.H) for _ in range(3)]
    eps = 1e-8

    def step_of(vec):
        st = [O.Coll.zeros(p.N, p.H) for _ in range(3)]
        for c in range(3):
            st[c].re[:, nh] = vec[c * 2 * p.N: c * 2 * p.N + p.N]
            st[c].im[:, nh] = vec[c * 2 * p.N + p.N: (c + 1) * 2 * p.N]
        p.set_state(*st)
        p.tim_t = 0.0
        p.timestep(orbit=True)
        out = np.empty(6 * p.N)
        for c, f in enumerate(p.state()):
            out[c * 2 * p.N: c * 2 * p.N + p.N] = f.re[:, nh]
            out[c * 2 * p.N + p.N: (c + 1) * 2 * p.N] = f.im[:, nh]
        return out

    n = 6 * p.N
    J = np.empty((n, n))
    for i in range(n):
        e = np.zeros(n)
        e[i] = eps
        J[:, i] = step_of(e) / eps
    lam = np.linalg.eigvals(J)
    lead = lam[np.argmax(np.abs(lam))]
    rate = math.log(abs(lead)) / p.cfg.dt
    # integrate the leading eigenvector (real and imaginary parts span the
    # invariant subspace) and measure its norm decay
    w, V = np.linalg.eig(J)
    vec = V[:, np.argmax(np.abs(w))]
    a = eps * np.real(vec) / np.linalg.norm(vec)
    b = eps * np.imag(vec) / np.linalg.norm(vec)
    n0 = math.sqrt(a @ a + b @ b)
    for _ in range(20):
        a = step_of(a)
        b = step_of(b)
    measured = math.log(math.sqrt(a @ a + b @ b) / n0) / (20 * p.cfg.dt)
    assert rate < 0
    assert abs(measured - rate) < 1e-3 * abs(rate) + 1e-6


def test_golden_fixtures_match_oracle():
    path = GOLDEN / "oracle_small.json"
    if not path.exists():
        pytest.skip("golden fixture not generated")
    gold = json.loads(path.read_text())
    for case in gold["cases"]:
        p = oracle_pipe(case["cfg"])
        p.vel_matrices()
        p.set_state(*O.seeded_state(p, case["seed"], case["energy"]))
        for _ in range(case["steps"]):
            p.timestep()
        E = p.energy()
        assert abs(E - case["energy_after"]) <= 1e-12 * abs(case["energy_after"])
        ur, ut, uz = p.state()
        for name, f in (("ur", ur), ("ut", ut), ("uz", uz)):
            cs = case["checksums"][name]
            assert abs(float(np.sum(f.re)) - cs[0]) <= 1e-10 * max(1.0, abs(cs[0]))
            assert abs(float(np.sum(f.im)) - cs[1]) <= 1e-10 * max(1.0, abs(cs[1]))
        prof = np.array(case["uz_mean_profile"])
        assert np.max(np.abs(uz.re[:, 0] - prof)) <= 1e-12 * np.max(np.abs(prof))
