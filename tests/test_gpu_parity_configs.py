"""Parity of the CUDA path against the oracle at the two remaining named
configurations.

Config-2, the large FP64 drop-in (N=64, K=128, M=48, Mp=2, Re=5300,
alpha=0.5, dt=0.005, seeded perturbation at 0.1 of the laminar energy): one
main-loop step against the numpy oracle at the FP64 bar of 1e-12, and three
steporbit steps (newton.f90:740-762, exactly one corrector each).  It runs
the FP64 length-384 z transform and the length-144 theta transform.

Mixed precision at config-1 sizes (N=40, K=24, M=16): FP32 transforms and
u x curl(u), FP64 solves, against the FP64 oracle itself after 1, 100 and
1000 steps.  The 1000-step leg uses the C++ restatement of the reference
step (oracle/pipeflow_cpu.cpp), which the numpy oracle holds to 1e-13.  The
bar is the mixed-precision budget: state relative L2 <= 1e-6, and the same
relative bound on the kinetic energy (var_coll_norm, variables.f90:718-751)
and the friction velocity (io.f90:627-639).
"""
import numpy as np
import pytest

import pipeflow_oracle as O
from _util import CFG1, device_pipe, oracle_pipe, state_from_dev, state_to_dev

pytestmark = pytest.mark.gpu

CFG2 = dict(N=64, K=128, M=48, Mp=2, Re=5300.0, alpha=0.5, dt=0.005)


@pytest.fixture(scope="module")
def cfg2_start():
    o = oracle_pipe(CFG2)
    o.vel_matrices()
    st = O.seeded_state(o, 2, 0.1)
    return o, st


def test_one_step_parity_cfg2(cfg2_start):
    o0, st = cfg2_start
    o = oracle_pipe(CFG2)
    o.vel_matrices()
    o.set_state(*st)
    g = device_pipe(CFG2)
    g.vel_matrices()
    state_to_dev(g, st)
    assert o.timestep() == g.timestep()
    err = O.rel_l2(state_from_dev(g), o.state())
    print(f"config-2 FP64, 1 step: state rel-L2 vs oracle = {err:.3e}")
    assert err <= 1e-12, err
    assert abs(g.vel_Pr0 - o.vel_Pr0) <= 1e-12 * max(1.0, abs(o.vel_Pr0))
    assert abs(g.energy() - o.energy()) <= 1e-12 * o.energy()
    g.close()


def test_steporbit_parity_cfg2(cfg2_start):
    o0, st = cfg2_start
    o = oracle_pipe(CFG2)
    o.vel_matrices()
    o.set_state(*st)
    g = device_pipe(CFG2)
    g.vel_matrices()
    state_to_dev(g, st)
    for _ in range(3):
        o.timestep(orbit=True)
    g.steporbit(3)
    err = O.rel_l2(state_from_dev(g), o.state())
    print(f"config-2 FP64, 3 steporbit steps: state rel-L2 vs oracle = {err:.3e}")
    assert err <= 1e-12, err
    g.close()


def _diag_of(o, state):
    """Energy and friction velocity of a state, by the oracle's formulas."""
    o.set_state(*state)
    return o.energy(), o.friction()[2]


def test_mixed_precision_cfg1_against_oracle():
    import pipeflow as P
    import pipeflow_cpu as PC

    o = oracle_pipe(CFG1)
    o.vel_matrices()
    st = O.seeded_state(o, 1, 1e-3)
    o.set_state(*st)
    cpu = PC.CpuPipe(o)
    g = device_pipe(CFG1, precision=P.PF_PREC_MIXED)
    g.vel_matrices()
    state_to_dev(g, st)
    probe = oracle_pipe(CFG1)
    probe.vel_matrices()
    done = 0
    rows = []
    for mark in (1, 100, 1000):
        for _ in range(mark - done):
            cpu.timestep()
            g.timestep()
        done = mark
        ref = [O.Coll(re, im) for re, im in cpu.state()]
        got = state_from_dev(g)
        err = O.rel_l2(got, ref)
        e_ref, f_ref = _diag_of(probe, ref)
        e_got, f_got = g.energy(), g.friction()[2]
        rows.append((mark, err, abs(e_got - e_ref) / e_ref, abs(f_got - f_ref) / f_ref))
    for mark, err, de, df in rows:
        print(f"mixed precision, config-1, {mark:5d} steps vs FP64 oracle: state rel-L2 {err:.3e}, "
              f"energy {de:.3e}, friction {df:.3e}")
    for mark, err, de, df in rows:
        assert err <= 1e-6, (mark, err)
        assert de <= 1e-6 and df <= 1e-6, (mark, de, df)
    cpu.close()
    g.close()
