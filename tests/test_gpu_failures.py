"""The reference's abort paths, and failures inside a served batch, injected
on the host.

The reference stops on the corrector control's three aborts (tim_check_cgce,
timestep.f90:222-240: "dt --> 0", "too many its", "increasing error") and on
a LAPACK factorisation error (timestep.f90:93; velocity.f90:166-168).  Here
each returns a status with the reference's message instead.  The corrector
aborts are driven by setting the time-stepping counters through the C ABI
(pf_tim_set) before pf_tim_check_cgce; the singular factorisation by a
matrix with zero interior rows (c1 = c2 = 0).  In a served batch a request
whose state holds a NaN fails alone, a cancelled request leaves at once, and
every other request's result equals, bit for bit, the same request run
alone.  Nothing here faults the GPU: the kernels only compute NaNs or record
a zero pivot, and the failure is decided on the host.
"""
import numpy as np
import pytest

from _util import SMALL, device_pipe

pytestmark = pytest.mark.gpu


def _fresh(**over):
    g = device_pipe(SMALL[0])
    g.vel_matrices()
    t = g.tim
    t.dt = SMALL[0]["dt"]
    t.step = 5
    t.it = 1
    t.pcn = -1
    t.dterr = 0.0
    for k, v in over.items():
        setattr(t, k, v)
    g.set_tim(t)
    return g


def _raises(fn, status, text):
    import pipeflow as P
    with pytest.raises(P.PipeflowError) as e:
        fn()
    assert e.value.status == status, e.value
    assert text in str(e.value), e.value


def test_check_cgce_dt_to_zero():
    from pipeflow import _lib as L
    g = _fresh(dt=1e-10, step=31)
    _raises(g.tim_check_cgce, L.PF_ERR_CONVERGE, "dt --> 0")
    assert g.tim.it == 0


def test_check_cgce_too_many_iterations():
    from pipeflow import _lib as L
    g = _fresh()
    dterr = g.cfg.dterr
    for it in range(1, 11):  # a slowly decreasing error keeps the corrector going
        t = g.tim
        t.it = it
        t.dterr = dterr * (100.0 - it)
        g.set_tim(t)
        g.tim_check_cgce()
        assert g.tim.it == it + 1
    t = g.tim
    t.dterr = dterr * 50.0
    g.set_tim(t)
    _raises(g.tim_check_cgce, L.PF_ERR_CONVERGE, "too many its")
    assert g.tim.it == 0


def test_check_cgce_increasing_error():
    from pipeflow import _lib as L
    g = _fresh(dterr=0.0)
    d = g.cfg.dterr
    t = g.tim
    t.it, t.dterr = 1, 10.0 * d
    g.set_tim(t)
    g.tim_check_cgce()
    assert g.tim.it == 2
    t = g.tim
    t.dterr = 20.0 * d  # larger than the last one and than 2 d_dterr
    g.set_tim(t)
    _raises(g.tim_check_cgce, L.PF_ERR_CONVERGE, "increasing error")
    # slightly increasing but under 2 d_dterr: no abort, a smaller corrector dt
    g2 = _fresh()
    t = g2.tim
    t.it, t.dterr = 1, 1.5 * d
    g2.set_tim(t)
    g2.tim_check_cgce()
    t = g2.tim
    t.dterr = 1.8 * d
    g2.set_tim(t)
    g2.tim_check_cgce()
    assert g2.tim.it == 0
    assert abs(g2.tim.corr_dt - g2.tim.dt / (10.0 * g2.cfg.courant)) < 1e-15


def test_singular_factorisation_is_reported():
    from pipeflow import _lib as L
    g = device_pipe(SMALL[0])
    # c1 = c2 = 0: every interior row of the band is zero, so dgbtrf meets a
    # zero pivot (LAPACK info > 0; timestep.f90:93 stops there)
    _raises(lambda: g.tim_lumesh_init(0, 0, 0.0, 0.0), L.PF_ERR_SINGULAR, "zero pivot")
    # the context stays usable
    g.vel_matrices()
    g.timestep()


def test_nan_state_steps_without_fault_and_reports_non_finite_error():
    g = device_pipe(SMALL[0])
    g.vel_matrices()
    import pipeflow as P
    P.seeded_state(g, 3, 1e-3)
    st = g.get_state()
    st[1][0][3, 2] = np.nan
    g.set_state(*st)
    g.timestep()  # the reference carries a NaN on; so does the lone pipe
    assert not np.all(np.isfinite(g.get_state()[1][0]))


# ------------------------------------------------------------------ serving
SHAPES = [
    dict(N=32, K=16, M=12, Mp=1, Re=1800.0, alpha=0.8, dt=0.01, precision=1),
    dict(N=24, K=8, M=6, Mp=2, Re=3000.0, alpha=1.6, dt=0.01, precision=0),
]


def _state(cfgd, seed):
    import pipeflow as P
    p = P.Pipe(P.PipeConfig(**cfgd))
    P.seeded_state(p, seed, 1e-3)
    st = p.get_state()
    p.close()
    return st


def _alone(cfgd, state, nsteps):
    import pipeflow as P
    p = P.Pipe(P.PipeConfig(**cfgd))
    p.vel_matrices()
    p.set_state(*state)
    p.steporbit(nsteps)
    out = p.get_state()
    p.close()
    return out


def _same(a, b):
    return all(np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1]) for x, y in zip(a, b))


def test_served_nan_request_fails_alone_and_cancel():
    import pipeflow as P
    from pipeflow import _lib as L
    srv = P.Server(hbm_budget=20 * 10**9)
    good = {}
    for i, (cfgd, n) in enumerate([(SHAPES[0], 5), (SHAPES[1], 6), (SHAPES[0], 4)]):
        st = _state(cfgd, 70 + i)
        good[srv.submit(P.PipeConfig(**cfgd), n, st)] = (cfgd, st, n)
    bad_state = _state(SHAPES[0], 80)
    bad_state[2][1][5, 7] = np.nan
    bad = srv.submit(P.PipeConfig(**SHAPES[0]), 5, bad_state)
    cancel_running = srv.submit(P.PipeConfig(**SHAPES[1]), 8, _state(SHAPES[1], 81))
    srv.step()
    srv.step()
    cancel_queued = srv.submit(P.PipeConfig(**SHAPES[1]), 3, _state(SHAPES[1], 82))
    srv.cancel(cancel_queued)
    srv.cancel(cancel_running)
    with pytest.raises(P.PipeflowError):
        srv.cancel(10**9)
    done = set()
    for _ in range(20):
        srv.step()
        done |= set(srv.finished())
        if srv.stats()["active"] == 0 and srv.stats()["queued"] == 0:
            break
    done |= set(srv.finished())
    assert {bad, cancel_running, cancel_queued} | set(good) <= done
    _raises(lambda: srv.result(bad), L.PF_ERR_CONVERGE, "non-finite")
    _raises(lambda: srv.result(cancel_running), L.PF_ERR_CANCELLED, "cancelled")
    _raises(lambda: srv.result(cancel_queued), L.PF_ERR_CANCELLED, "cancelled")
    for rid, (cfgd, st, n) in good.items():
        assert _same(srv.result(rid), _alone(cfgd, st, n)), rid
    srv.close()
