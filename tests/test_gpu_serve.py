"""Request serving with continuous batching (pf_serve_*).

Each request advances a seeded state by nsteps steporbit timesteps.  Requests
arrive while others are running, join the running batch, leave it when done,
and hand their contexts to later requests of the same shape.  Every result
must equal, bit for bit, the same request run alone on a lone pipe.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [
    dict(N=32, K=16, M=12, Mp=1, Re=1800.0, alpha=0.8, dt=0.01, precision=1),
    dict(N=48, K=32, M=24, Mp=1, Re=2400.0, alpha=1.1, dt=0.01, precision=0),
    dict(N=24, K=8, M=6, Mp=2, Re=3000.0, alpha=1.6, dt=0.01, precision=1),
]


def _state(cfgd, seed, eps=1e-3):
    import pipeflow as P
    p = P.Pipe(P.PipeConfig(**cfgd))
    P.seeded_state(p, seed, eps)
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


def test_results_equal_alone_and_in_the_mix():
    import pipeflow as P
    srv = P.Server(hbm_budget=40 * 10**9)
    reqs = {}  # id -> (cfg, state, nsteps)

    def submit(cfgd, seed, nsteps):
        st = _state(cfgd, seed)
        rid = srv.submit(P.PipeConfig(**cfgd), nsteps, st)
        reqs[rid] = (cfgd, st, nsteps)
        return rid

    submit(SHAPES[0], 1, 4)
    submit(SHAPES[1], 2, 9)
    results = {}
    for _ in range(3):
        srv.step()
    assert srv.stats()["active"] == 2
    # arrive while the first two are on the GPU
    submit(SHAPES[2], 3, 6)
    # same shape as the first request, other physics: reuses its context once
    # the first request has finished
    submit(dict(SHAPES[0], Re=2600.0, alpha=1.3), 4, 5)
    saw_pool = False
    while len(results) < len(reqs):
        srv.step()
        saw_pool |= srv.stats()["pooled"] > 0
        for rid in srv.finished():
            results[rid] = srv.result(rid)
    assert saw_pool
    for rid, (cfgd, st, n) in reqs.items():
        assert _same(results[rid], _alone(cfgd, st, n)), rid
    assert srv.launches() > 0
    srv.close()


def test_admission_waits_for_the_hbm_budget():
    import pipeflow as P
    cfgd = SHAPES[1]
    one = P.Pipe(P.PipeConfig(**cfgd))
    budget = one.device_bytes() * 3 // 2  # room for one context of this shape, not two
    one.close()
    srv = P.Server(hbm_budget=budget)
    a = srv.submit(P.PipeConfig(**cfgd), 3, _state(cfgd, 7))
    b = srv.submit(P.PipeConfig(**dict(cfgd, Re=2000.0)), 2, _state(cfgd, 8))
    srv.step()
    s = srv.stats()
    assert s["active"] == 1 and s["queued"] == 1
    done = []
    while len(done) < 2:
        srv.step()
        done += srv.finished()
        assert srv.stats()["bytes"] <= budget
    assert done == [a, b]
    srv.close()


def test_bad_requests_are_rejected():
    import pipeflow as P
    srv = P.Server()
    st = _state(SHAPES[0], 1)
    with pytest.raises(P.PipeflowError):
        srv.submit(P.PipeConfig(**dict(SHAPES[0], dt=-0.01)), 5, st)
    with pytest.raises(P.PipeflowError):
        srv.submit(P.PipeConfig(**SHAPES[0]), 0, st)
    srv.close()
