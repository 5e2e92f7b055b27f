"""The C++/OpenMP CPU restatement (oracle/pipeflow_cpu.cpp) against the numpy
oracle: two restatements of the same reference step, written separately (own
FFT and own banded solve in C++; numpy FFT and scipy LAPACK in Python), must
agree to rounding on identical seeded states.  CPU only."""
import json
from pathlib import Path

import numpy as np
import pytest

import pipeflow_oracle as O

PC = pytest.importorskip("pipeflow_cpu")

CASES = [
    dict(N=16, K=4, M=4, Mp=1, Re=2000.0, alpha=1.25, dt=0.01),
    dict(N=24, K=7, M=5, Mp=2, Re=3000.0, alpha=0.8, dt=0.005),  # Z = 21: radix 7
    dict(N=20, K=5, M=6, Mp=1, Re=1800.0, alpha=1.6, dt=0.01, const_flux=False),
    dict(N=40, K=24, M=16, Mp=1, Re=2000.0, alpha=1.25, dt=0.01),  # config-1 sizes
]


def _states(c):
    return [O.Coll(a, b) for a, b in c.state()]


@pytest.mark.parametrize("cfgd", CASES, ids=lambda c: "N{N}K{K}M{M}".format(**c))
@pytest.mark.parametrize("orbit", [False, True], ids=["main", "orbit"])
def test_cpp_step_matches_numpy_oracle(cfgd, orbit):
    o = O.Pipe(O.PipeConfig(**cfgd))
    o.vel_matrices()
    o.set_state(*O.seeded_state(o, 3, 1e-3))
    c = PC.CpuPipe(o)
    for _ in range(3):
        assert o.timestep(orbit=orbit) == c.timestep(orbit=orbit)
        assert O.rel_l2(_states(c), o.state()) <= 1e-13
    c.close()


def test_cpp_step_matches_golden_fixtures():
    gold = json.loads((Path(__file__).parent / "golden" / "oracle_small.json").read_text())
    for case in gold["cases"]:
        o = O.Pipe(O.PipeConfig(**case["cfg"]))
        o.vel_matrices()
        o.set_state(*O.seeded_state(o, case["seed"], case["energy"]))
        c = PC.CpuPipe(o)
        assert [c.timestep() for _ in range(case["steps"])] == case["ncorr"]
        (urr, uri), (utr, uti), (uzr, uzi) = c.state()
        for name, (re, im) in (("ur", (urr, uri)), ("ut", (utr, uti)), ("uz", (uzr, uzi))):
            cs = case["checksums"][name]
            assert abs(float(np.sum(re)) - cs[0]) <= 1e-10 * max(1.0, abs(cs[0]))
            assert abs(float(np.sum(im)) - cs[1]) <= 1e-10 * max(1.0, abs(cs[1]))
        prof = np.array(case["uz_mean_profile"])
        assert np.max(np.abs(uzr[:, 0] - prof)) <= 1e-12 * np.max(np.abs(prof))
        c.close()


def test_threads_give_the_same_result():
    cfgd = CASES[3]
    out = []
    for th in (1, max(2, PC.threads())):
        PC.set_threads(th)
        o = O.Pipe(O.PipeConfig(**cfgd))
        o.vel_matrices()
        o.set_state(*O.seeded_state(o, 5, 1e-3))
        c = PC.CpuPipe(o)
        c.timestep()
        out.append(c.state())
        c.close()
    for (a, b), (x, y) in zip(out[0], out[1]):
        assert np.array_equal(a, x) and np.array_equal(b, y)
