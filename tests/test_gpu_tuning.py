"""Launch choices (pf_ctx_set_tuning) change the speed, never the numbers.

The banded solves of the fused step stream the LU factors that k_lu_factor
stored (PF_LD_STREAMED, the built-in choice), or do so with modes k and -k on
one thread (PF_LD_PAIRED), or rebuild the Helmholtz factors on chip in the
same order of operations (PF_LD_REBUILT, for factorisations that did not
pivot);
the transform passes take any z-pass column tile and any even theta-pass row
tile.  Each pair of pipes here starts from the same seeded state and must
stay bitwise equal step after step, and one of them is held to the oracle.
"""
import numpy as np
import pytest

import pipeflow_oracle as O
from _util import CFG1, SMALL, device_pipe, oracle_pipe, state_from_dev, state_to_dev

pytestmark = pytest.mark.gpu


def _states_equal(a, b):
    for (ar, ai), (br, bi) in zip(a.get_state(), b.get_state()):
        if not (np.array_equal(ar, br) and np.array_equal(ai, bi)):
            return False
    return True


def _pair(cfgd, **extra):
    a, b = device_pipe(cfgd, **extra), device_pipe(cfgd, **extra)
    for g in (a, b):
        g.vel_matrices()
    return a, b


PIVOTING = dict(N=64, K=4, M=4, Mp=1, Re=1900.0, alpha=1.2, dt=0.01)  # Helmholtz factors pivot


@pytest.mark.parametrize("cfgd", [SMALL[0], SMALL[1], CFG1, PIVOTING], ids=["small0", "small1", "cfg1", "pivoting"])
@pytest.mark.parametrize("mixed", [False, True], ids=["fp64", "mixed"])
@pytest.mark.parametrize("solver", ["rebuilt", "paired", "warpring"])
def test_helmholtz_solver_choices_equal_streamed(cfgd, mixed, solver):
    import pipeflow as P
    extra = {"precision": P.PF_PREC_MIXED} if mixed else {}
    a, b = _pair(cfgd, **extra)
    choice = {"rebuilt": P.PF_LD_REBUILT, "paired": P.PF_LD_PAIRED, "warpring": P.PF_LD_WARPRING}[solver]
    a.set_tuning(ld_solver=choice)
    b.set_tuning(ld_solver=P.PF_LD_STREAMED)
    assert a.get_tuning()["ld_solver"] == choice
    o = oracle_pipe(cfgd)
    o.vel_matrices()
    st = O.seeded_state(o, 3, 1e-3)
    for g in (a, b):
        state_to_dev(g, st)
    for _ in range(4):
        assert a.timestep() == b.timestep()
        assert _states_equal(a, b)
    a.steporbit(2)
    b.steporbit(2)
    assert _states_equal(a, b)
    if not mixed:
        o.set_state(*st)
        for _ in range(4):
            o.timestep()
        for _ in range(2):
            o.timestep(orbit=True)
        assert O.rel_l2(state_from_dev(a), o.state()) <= 1e-12


@pytest.mark.parametrize("mixed", [False, True], ids=["fp64", "mixed"])
def test_transform_tiles_do_not_change_results(mixed):
    import pipeflow as P
    extra = {"precision": P.PF_PREC_MIXED} if mixed else {}
    ref = device_pipe(CFG1, **extra)
    ref.vel_matrices()
    P.seeded_state(ref, 11, 1e-3)
    start = ref.get_state()
    for _ in range(2):
        ref.timestep()
    for mc, zc in [(1, 2), (3, 4), (16, 8), (5, 16), (0, 6)]:
        g = device_pipe(CFG1, **extra)
        g.vel_matrices()
        g.set_tuning(nl_mc=mc, nl_zc=zc)
        g.set_state(*start)
        for _ in range(2):
            g.timestep()
        assert _states_equal(g, ref), (mc, zc)
        g.close()
    ref.close()


def test_tuning_rejects_bad_choices():
    import pipeflow as P
    g = device_pipe(SMALL[0])
    with pytest.raises(Exception):
        g.set_tuning(nl_zc=3)
    with pytest.raises(Exception):
        g.set_tuning(ld_solver=7)
    with pytest.raises(Exception):
        g.set_tuning(nl_fused=2)
    g.set_tuning(ld_solver=P.PF_LD_REBUILT, nl_fused=1)
    g.set_tuning()
    assert g.get_tuning() == {"ld_solver": P.PF_LD_AUTO, "nl_mc": 0, "nl_zc": 0, "nl_fused": 0}


def _batch(cfgs):
    import pipeflow as P
    b = P.Batch([P.PipeConfig(**d) for d in cfgs])
    b.matrices()
    for i, p in enumerate(b.pipes):
        P.seeded_state(p, 40 + i, 1e-3)
    return b


def test_batch_with_every_solver_choice_equals_streamed():
    """A batch whose pipes take different solver choices (so every batched
    solve launch runs, pivoting and not) steps bitwise like one that streams
    the factors everywhere."""
    import pipeflow as P
    mix = [dict(SMALL[0]), dict(SMALL[1]), dict(CFG1, precision=P.PF_PREC_MIXED), dict(PIVOTING),
           dict(SMALL[1], precision=P.PF_PREC_MIXED), dict(CFG1), dict(PIVOTING, Re=2100.0), dict(SMALL[0])]
    choices = [P.PF_LD_WARPRING, P.PF_LD_PAIRED, P.PF_LD_WARPRING, P.PF_LD_WARPRING, P.PF_LD_REBUILT, P.PF_LD_AUTO,
               P.PF_LD_PAIRED, P.PF_LD_STREAMED]
    a, b = _batch(mix), _batch(mix)
    for p, c in zip(a.pipes, choices):
        p.set_tuning(ld_solver=c)
    for p in b.pipes:
        p.set_tuning(ld_solver=P.PF_LD_STREAMED)
    for _ in range(2):
        a.step(2)
        b.step(2)
        for pa, pb in zip(a.pipes, b.pipes):
            assert _states_equal(pa, pb)


def test_autotuned_batch_equals_untuned(tmp_path):
    """The tuner restores the states it advanced while timing, caches its
    choices, and a tuned batch steps bit for bit like an untuned one."""
    import pipeflow as P
    mix = [dict(SMALL[0]), dict(SMALL[1]), dict(SMALL[0], precision=P.PF_PREC_MIXED),
           dict(CFG1, precision=P.PF_PREC_MIXED)]
    a, b = _batch(mix), _batch(mix)
    tuner = P.Tuner(cache_path=tmp_path / "tuning.json", steps=2, reps=1)
    choice = tuner.tune_batch(a)
    assert len(choice) == 5 and len(tuner.log) > 8
    assert choice["batch"]["worklist"] in (0, 1) and a.worklist == bool(choice["batch"]["worklist"])
    for pa, pb in zip(a.pipes, b.pipes):
        assert _states_equal(pa, pb)
        assert pa.tim.step == pb.tim.step
    a.step(3)
    b.step(3)
    for pa, pb in zip(a.pipes, b.pipes):
        assert _states_equal(pa, pb)
    again = P.Tuner(cache_path=tmp_path / "tuning.json", steps=2, reps=1)
    assert again.tune_batch(a) == choice and again.log == []


def test_autotuned_pipe_equals_untuned(tmp_path):
    import pipeflow as P
    a, b = _pair(CFG1)
    P.seeded_state(a, 12, 1e-3)
    b.set_state(*a.get_state())
    t = P.Tuner(cache_path=tmp_path / "tuning.json", steps=2, reps=1)
    t.tune_pipe(a)
    assert _states_equal(a, b)
    for _ in range(3):
        a.timestep()
        b.timestep()
    assert _states_equal(a, b)


MIXED_IDS = ["small0", "small1", "small2", "cfg1"]


@pytest.mark.parametrize("cfgd", [SMALL[0], SMALL[1], SMALL[2], CFG1], ids=MIXED_IDS)
def test_one_block_per_radial_point_equals_three_passes(cfgd):
    """Mixed precision: the transforms of a radial point in one block (plane
    in shared memory) give bitwise the three-pass kernels' states."""
    import pipeflow as P
    a, b = _pair(cfgd, precision=P.PF_PREC_MIXED)
    a.set_tuning(nl_fused=1)
    assert a.nl_passes == 1 and b.nl_passes == 3
    st = O.seeded_state(oracle_pipe(cfgd), 5, 1e-3)
    for g in (a, b):
        state_to_dev(g, st)
    for _ in range(4):
        assert a.timestep() == b.timestep()
        assert _states_equal(a, b)
    a.steporbit(2)
    b.steporbit(2)
    assert _states_equal(a, b)


def test_one_block_per_radial_point_cfl_maxima_drive_the_same_dt():
    """Adaptive dt in mixed precision at config-1 (Z = 72: the last theta
    chunk of 16 z rows is half padding): the CFL maxima the one-block kernel
    stores outright equal the three-pass kernels' atomic maxima, so dt
    follows the same sequence."""
    import pipeflow as P
    cfgd = dict(CFG1, dt=-1.0, maxdt=0.01, courant=0.5)
    a, b = device_pipe(cfgd, precision=P.PF_PREC_MIXED), device_pipe(cfgd, precision=P.PF_PREC_MIXED)
    a.set_tuning(nl_fused=1)
    st = O.seeded_state(oracle_pipe(CFG1), 11, 1e-2)
    for g in (a, b):
        t = g.tim
        t.dt = 0.004
        g.set_tim(t)
        g.vel_matrices()
        state_to_dev(g, st)
    dts = [a.tim.dt]
    for _ in range(6):
        assert a.timestep() == b.timestep()
        assert a.tim.dt == b.tim.dt
        assert _states_equal(a, b)
        dts.append(a.tim.dt)
    assert len(set(dts)) > 1


def test_batched_one_block_per_radial_point_equals_three_passes():
    """A batch whose mixed-precision pipes take the one-block kernel (several
    (Z, Th) groups on their own streams, beside a pipe whose plane does not
    fit and an FP64 pipe, which take the three passes) steps bitwise like the
    same batch with every pipe on the three passes."""
    import pipeflow as P
    mx = P.PF_PREC_MIXED
    base = dict(Mp=1, Re=2200.0, alpha=1.1, dt=0.01)
    mix = [dict(base, N=32, K=16, M=12, precision=mx), dict(base, N=24, K=32, M=24, precision=mx),
           dict(base, N=20, K=64, M=12, precision=mx), dict(base, N=16, K=64, M=24, precision=mx),
           dict(CFG1, precision=mx), dict(SMALL[0]), dict(base, N=32, K=16, M=12, precision=mx)]
    a, b = _batch(mix), _batch(mix)
    for p in a.pipes:
        p.set_tuning(nl_fused=1)
    assert [p.nl_passes for p in a.pipes] == [1, 1, 1, 3, 1, 3, 1]
    assert all(p.nl_passes == 3 for p in b.pipes)
    for _ in range(2):
        a.step(2)
        b.step(2)
        for pa, pb in zip(a.pipes, b.pipes):
            assert _states_equal(pa, pb)
    a.step(2, orbit=True)
    b.step(2, orbit=True)
    for pa, pb in zip(a.pipes, b.pipes):
        assert _states_equal(pa, pb)
