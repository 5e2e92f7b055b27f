"""Batched pipes (pf_batch_*) and the mixed-precision transform path.

A batch runs every pipe's own kernel chain, so a pipe's state after any
number of batched steps must equal, bit for bit, the same pipe stepped alone.
Mixed precision (FP32 transforms and u x curl(u); FP64 elsewhere, including
the k=m=0 mode) is held to the 1e-6 relative-L2 budget against FP64.
"""
import numpy as np
import pytest

import pipeflow_oracle as O
from _util import CFG1, state_from_dev

pytestmark = pytest.mark.gpu

UNEVEN = [
    dict(N=32, K=16, M=12, Mp=1, Re=1800.0, alpha=0.8, dt=0.01),
    dict(N=48, K=32, M=24, Mp=1, Re=2400.0, alpha=1.1, dt=0.01),
    dict(N=64, K=16, M=32, Mp=1, Re=3000.0, alpha=1.6, dt=0.01),
    dict(N=32, K=64, M=12, Mp=2, Re=2000.0, alpha=1.3, dt=0.01),
]


PIVOTING = dict(N=64, K=4, M=4, Mp=1, Re=1900.0, alpha=1.25, dt=0.01)  # its Helmholtz factors pivot


def _cfgs(prec=0, extra=()):
    import pipeflow as P
    return [P.PipeConfig(**d, precision=prec) for d in UNEVEN] + [P.PipeConfig(**d, precision=prec) for d in extra]


def _seed(pipe, i):
    import pipeflow as P
    P.seeded_state(pipe, 100 + i, 1e-3)


# (orbit, precision, extra pipes, stage-batched graphs expected)
VARIANTS = {
    "main": (False, 0, (), True),
    "orbit": (True, 0, (), True),
    "mixed": (False, 1, (), True),
    "pivot": (False, 0, (PIVOTING,), True),
    # a mirror-symmetric pipe keeps the batch on per-pipe graph branches
    "branch": (False, 0, (dict(N=32, K=8, M=8, Mp=1, Re=2000.0, alpha=1.0, dt=0.01, mirrorsym=True),), False),
}


@pytest.mark.parametrize("variant", list(VARIANTS))
def test_batch_equals_lone_pipes(variant):
    import pipeflow as P
    orbit, prec, extra, staged = VARIANTS[variant]
    cfgs = _cfgs(prec, extra)
    batch = P.Batch(cfgs)
    batch.matrices()
    alone = [P.Pipe(c) for c in cfgs]
    for i, (bp, ap) in enumerate(zip(batch.pipes, alone)):
        ap.vel_matrices()
        _seed(bp, i)
        _seed(ap, i)
    nsteps = 5
    n0 = batch.launches()
    batch.step(nsteps, orbit=orbit)
    assert batch.staged() == staged
    assert batch.launches() > n0
    for ap in alone:
        if orbit:
            ap.steporbit(nsteps)
        else:
            for _ in range(nsteps):
                ap.timestep()
    for bp, ap in zip(batch.pipes, alone):
        for (br, bi), (ar, ai) in zip(bp.get_state(), ap.get_state()):
            assert np.array_equal(br, ar) and np.array_equal(bi, ai)
        assert bp.tim.step == ap.tim.step == nsteps
        assert bp.tim.dt == ap.tim.dt
    batch.close()


@pytest.mark.parametrize("orbit", [False, True], ids=["main", "orbit"])
def test_batch_worklist_stages_equal_lone_pipes(orbit):
    """Mixed precision with each transform stage as one persistent launch over
    a work list of every pipe's tiles (all four transform lengths of each
    pass in one launch): bitwise the lone pipes, and one launch per stage."""
    import pipeflow as P
    cfgs = _cfgs(P.PF_PREC_MIXED)
    batch = P.Batch(cfgs)
    batch.set_worklist(True)
    assert batch.worklist
    batch.matrices()
    alone = [P.Pipe(c) for c in cfgs]
    for i, (bp, ap) in enumerate(zip(batch.pipes, alone)):
        ap.vel_matrices()
        _seed(bp, i)
        _seed(ap, i)
    batch.step(1, orbit=orbit)  # eager first step
    n0 = batch.launches()
    batch.step(4, orbit=orbit)
    assert batch.staged()
    for ap in alone:
        if orbit:
            ap.steporbit(5)
        else:
            for _ in range(5):
                ap.timestep()
    for bp, ap in zip(batch.pipes, alone):
        for (br, bi), (ar, ai) in zip(bp.get_state(), ap.get_state()):
            assert np.array_equal(br, ar) and np.array_equal(bi, ai)
        assert bp.tim.step == ap.tim.step == 5
    n_wl = batch.launches() - n0
    # switching back rebuilds the per-length launches; still the lone pipes
    batch.set_worklist(False)
    batch.step(1, orbit=True)  # eager first step of the rebuilt launches
    n1 = batch.launches()
    batch.step(4, orbit=True)
    n_pl = batch.launches() - n1
    for ap in alone:
        ap.steporbit(5)
    for bp, ap in zip(batch.pipes, alone):
        for (br, bi), (ar, ai) in zip(bp.get_state(), ap.get_state()):
            assert np.array_equal(br, ar) and np.array_equal(bi, ai)
    if orbit:
        # the three work-list launches of an evaluation replace one launch per
        # stage and transform length
        assert n_wl < n_pl, (n_wl, n_pl)
    batch.close()


def test_batch_staged_launch_count():
    """A stage-batched step is a fixed number of launches, whatever the pipe count."""
    import pipeflow as P
    batch = P.Batch(_cfgs())
    batch.matrices()
    for i, bp in enumerate(batch.pipes):
        _seed(bp, i)
    batch.step(1)  # eager first step
    n0 = batch.launches()
    passes = batch.step(2, orbit=True)
    assert passes == 2 * len(batch.pipes)
    assert batch.staged()
    # per step: mean-mode symmetry, the transform stages (one launch per
    # distinct length: zinv and zfwd by Z, theta by Th), 5 step stages, the
    # transform stages again, 5 step stages, the symmetry again, scalar gather
    # (the Helmholtz solves take a second launch when some pipes' factors
    # pivot and others' do not)
    cfgs = _cfgs()
    nl = 2 * len({c.Z for c in cfgs}) + len({c.Th for c in cfgs})
    base = 1 + nl + 5 + nl + 5 + 1 + 1
    assert batch.launches() - n0 in (2 * base, 2 * (base + 2))
    batch.close()


def test_batch_state_matches_oracle():
    import pipeflow as P
    d = UNEVEN[0]
    batch = P.Batch([P.PipeConfig(**d)] * 2)
    batch.matrices()
    o = O.Pipe(O.PipeConfig(**d))
    o.vel_matrices()
    st = O.seeded_state(o, 5, 1e-3)
    o.set_state(*st)
    for bp in batch.pipes:
        bp.set_state(*[(c.re, c.im) for c in st])
    batch.step(4)
    for _ in range(4):
        o.timestep()
    for bp in batch.pipes:
        assert O.rel_l2(state_from_dev(bp), o.state()) <= 1e-12
    batch.close()


def _err_report(gm, g64):
    s_m, s_64 = state_from_dev(gm), state_from_dev(g64)
    err = O.rel_l2(s_m, s_64)
    e_m, e_64 = gm.energy(), g64.energy()
    f_m, f_64 = gm.friction()[2], g64.friction()[2]
    return err, abs(e_m - e_64) / e_64, abs(f_m - f_64) / f_64


def test_mixed_precision_error_budget():
    import pipeflow as P
    g64 = P.Pipe(P.PipeConfig(**CFG1))
    gm = P.Pipe(P.PipeConfig(**CFG1, precision=P.PF_PREC_MIXED))
    for g in (g64, gm):
        g.vel_matrices()
        P.seeded_state(g, 1, 1e-3)
    report = {}
    done = 0
    for target in (1, 100):
        while done < target:
            g64.timestep()
            gm.timestep()
            done += 1
        report[target] = _err_report(gm, g64)
    # state rel-L2, kinetic energy and friction-velocity errors vs FP64
    assert report[1][0] < 1e-6, report
    assert report[100][0] < 1e-6, report
    assert report[100][1] < 1e-6 and report[100][2] < 1e-6, report


def test_mixed_precision_mean_mode_is_fp64():
    """The k=m=0 nonlinear term is computed in FP64 in the mixed path."""
    import pipeflow as P
    g64 = P.Pipe(P.PipeConfig(**CFG1))
    gm = P.Pipe(P.PipeConfig(**CFG1, precision=P.PF_PREC_MIXED))
    for g in (g64, gm):
        P.seeded_state(g, 2, 1e-3)
        g.vel_transform_nonlinear()
    for c in (3, 4, 5):
        n64, nm = g64.vel_field(c).download(), gm.vel_field(c).download()
        scale = np.abs(n64[0]).max() + np.abs(n64[1]).max()
        # the mode-0 column agrees to FP64 rounding, the rest to FP32 accuracy
        assert np.max(np.abs(nm[0][:, 0] - n64[0][:, 0])) <= 1e-12 * scale
        rest = max(np.abs(nm[0][:, 1:] - n64[0][:, 1:]).max(), np.abs(nm[1][:, 1:] - n64[1][:, 1:]).max())
        assert 0 < rest < 1e-5 * scale


def test_fused_transform_nonlinear_matches_oracle():
    import pipeflow as P
    from _util import from_dev, oracle_pipe, rel_coll, state_to_dev
    o, g = oracle_pipe(CFG1), P.Pipe(P.PipeConfig(**CFG1))
    st = O.seeded_state(o, 3, 1e-3)
    o.set_state(*st)
    state_to_dev(g, st)
    o.vel_transform()
    o.vel_nonlinear()
    g.vel_transform_nonlinear()
    for i, ref in enumerate((o.vel_Nr, o.vel_Nt, o.vel_Nz)):
        assert rel_coll(from_dev(g.vel_field(3 + i)), ref) < 1e-12


def test_set_state_then_batch_step_is_ordered():
    """States uploaded on the pipes' own streams right before a batch step are
    the ones the step reads (the step waits for the uploads on the device), and
    the asynchronous download returns the stepped states after a sync."""
    import ctypes as C
    import pipeflow as P
    cfgs = _cfgs()
    batch = P.Batch(cfgs)
    batch.matrices()
    for i, bp in enumerate(batch.pipes):
        _seed(bp, i)
    batch.step(3)  # graphs captured for both parities
    fresh = []
    for i, c in enumerate(cfgs):
        tmp = P.Pipe(c)
        P.seeded_state(tmp, 500 + i, 1e-3)
        fresh.append(tmp.get_state())
        tmp.close()
    for bp, st in zip(batch.pipes, fresh):
        bp.set_state(*st)
    batch.step(2)
    outs = []
    for bp in batch.pipes:
        arrs = [np.empty((bp.H, bp.N)) for _ in range(6)]
        ptrs = [a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs]
        assert bp.lib.pf_vel_get_state_async(bp.ctx, *ptrs) == 0
        outs.append(arrs)
    batch.sync()
    for c, st, arrs in zip(cfgs, fresh, outs):
        ap = P.Pipe(c)
        ap.vel_matrices()
        ap.set_state(*st)
        ap.timestep()
        ap.timestep()
        got = [np.ascontiguousarray(a.T) for a in arrs]
        want = [x for f in ap.get_state() for x in f]
        for g, w in zip(got, want):
            assert np.array_equal(g, w)
        ap.close()
    batch.close()


def _block(states):
    """State block of pf_batch_put_states: per pipe ur Re, ur Im, ut Re, ut Im,
    uz Re, uz Im, each (H, N) with n fastest."""
    return np.concatenate([np.ascontiguousarray(x.T).ravel() for st in states for f in st for x in f])


def _unblock(batch, blk):
    out, off = [], 0
    for p in batch.pipes:
        n = p.N * p.H
        a = [np.ascontiguousarray(blk[off + k * n:off + (k + 1) * n].reshape(p.H, p.N).T) for k in range(6)]
        out.append([(a[0], a[1]), (a[2], a[3]), (a[4], a[5])])
        off += 6 * n
    return out


@pytest.mark.parametrize("orbit", [False, True], ids=["main", "orbit"])
def test_batch_pipelined_state_io(orbit):
    """put_states / step_io / get_states with alternating slots: each output
    block equals its input stepped alone through pf_timestep (bit for bit), a
    zero-step pass returns its input unchanged, and a step without a block put
    into its slot is refused."""
    import pipeflow as P
    cfgs = _cfgs()
    batch = P.Batch(cfgs)
    batch.matrices()
    for i, bp in enumerate(batch.pipes):
        _seed(bp, i)
    batch.step(3, orbit=orbit)  # graphs captured for both parities
    ins = []
    for s in range(3):
        sts = []
        for i, c in enumerate(cfgs):
            tmp = P.Pipe(c)
            P.seeded_state(tmp, 700 + 10 * s + i, 1e-3)
            sts.append(tmp.get_state())
            tmp.close()
        ins.append(_block(sts))
    assert batch.io_bytes() == ins[0].nbytes
    with pytest.raises(P.PipeflowError):
        batch.step_io(1, 1)
    back = np.empty_like(ins[0])
    batch.put_states(0, ins[0])
    batch.step_io(0, 0)
    batch.get_states(0, back)
    batch.io_wait(0)
    assert np.array_equal(back, ins[0])
    outs = [np.empty_like(ins[0]) for _ in range(3)]
    batch.put_states(0, ins[0])
    for s in range(3):
        if s + 1 < 3:
            batch.put_states((s + 1) % 2, ins[s + 1])
        batch.step_io(s % 2, 2, orbit=orbit)
        batch.get_states(s % 2, outs[s])
    batch.io_sync()
    for s in range(3):
        want_all = _unblock(batch, ins[s])
        got_all = _unblock(batch, outs[s])
        for c, st, got in zip(cfgs, want_all, got_all):
            ap = P.Pipe(c)
            ap.vel_matrices()
            ap.set_state(*st)
            for _ in range(2):
                if orbit:
                    ap.steporbit(1)
                else:
                    ap.timestep()
            for (gr, gi), (wr, wi) in zip(got, ap.get_state()):
                assert np.array_equal(gr, wr) and np.array_equal(gi, wi)
            ap.close()
    batch.close()
