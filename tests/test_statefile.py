"""State files (io.f90:98-392) written and read without libnetcdf.

CPU: the product's writer against scipy's netCDF-3 reader, its reader on
files scipy writes with io_save_state's structure, interpolation and
re-truncation against the numpy restatement in the oracle, exactness of the
radial interpolation on polynomials of the right parity.  GPU: a pipe's
state saved and loaded back, and loaded onto another resolution."""
import math

import numpy as np
import pytest

import io_oracle as IO
import pipeflow_oracle as O


def _mesh(N):
    return O.default_mesh(N)


def _state(N, K, M, seed):
    rng = np.random.default_rng(seed)
    H = IO.harmonics(K, M)
    return [(rng.standard_normal((N, H)), rng.standard_normal((N, H))) for _ in range(3)]


def test_written_file_is_netcdf_with_reference_structure(tmp_path):
    from pipeflow.statefile import state_write
    N, K, M, Mp = 12, 3, 4, 2
    r = _mesh(N)
    st = _state(N, K, M, 1)
    p = tmp_path / "state0007.cdf.dat"
    state_write(p, N, K, M, Mp, r, st, t=1.25, Re=2400.0, alpha=1.1, dt=0.01, dtcor=0.02, dtcfl=0.03)
    raw = IO.read_raw(str(p))
    assert raw["dims"] == {"r": N, "H": IO.harmonics(K, M), "ReIm": 2}
    assert (raw["t"], raw["Re"], raw["alpha"], raw["dt"], raw["dtcor"], raw["dtcfl"]) == (1.25, 2400.0, 1.1, 0.01,
                                                                                            0.02, 0.03)
    assert np.array_equal(raw["r"], r)
    for nm, (re, im) in zip(("Ur", "Ut", "Uz"), st):
        data, K_, M_, Mp_, dims = raw[nm]
        assert (K_, M_, Mp_) == (K, M, Mp) and tuple(dims) == ("ReIm", "H", "r")
        assert np.array_equal(data[0].T, re) and np.array_equal(data[1].T, im)


@pytest.mark.parametrize("version", [1, 2], ids=["classic", "64bit_offset"])
def test_read_same_resolution_is_exact(tmp_path, version):
    from pipeflow.statefile import state_read
    N, K, M, Mp = 16, 4, 5, 1
    r = _mesh(N)
    st = _state(N, K, M, 2)
    p = str(tmp_path / "state.cdf.in")
    IO.write_like_reference(p, N, K, M, Mp, r, st, t=3.0, Re=2000.0, alpha=1.25, dt=0.005, version=version)
    got, sc, ch = state_read(p, N, K, M, Mp, r)
    assert ch == 0
    assert sc["t"] == 3.0 and sc["dt"] == 0.005 and sc["Re"] == 2000.0
    for (a, b), (c, d) in zip(got, st):
        assert np.array_equal(a, c) and np.array_equal(b, d)


@pytest.mark.parametrize("src,dst", [
    ((24, 6, 5, 1), (16, 4, 6, 1)),   # fewer points, fewer k, more m
    ((16, 4, 4, 2), (20, 5, 3, 2)),   # more points and k, fewer m
    ((16, 3, 2, 1), (16, 3, 2, 1)),   # same sizes, different mesh (custom r)
    ((18, 5, 3, 1), (18, 3, 5, 1)),   # fewer k and more m: the file index walk of io_load_coll
])
def test_read_other_resolution_matches_oracle(tmp_path, src, dst):
    from pipeflow.statefile import state_read
    N_, K_, M_, Mp = src
    N, K, M, _ = dst
    r_ = _mesh(N_)
    r = _mesh(N) if (N, K, M) != (N_, K_, M_) else np.sort(0.02 + 0.97 * np.random.default_rng(3).random(N))
    st = _state(N_, K_, M_, 4)
    p = str(tmp_path / "s.cdf")
    IO.write_like_reference(p, N_, K_, M_, Mp, r_, st)
    got, _, ch = state_read(p, N, K, M, Mp, r)
    want, _ = IO.load_state(p, N, K, M, Mp, r)
    assert bool(ch & 1) == (N != N_ or bool(np.max(np.abs(r - r_)) > 1e-8))
    assert bool(ch & 2) == (K != K_) and bool(ch & 4) == (M != M_)
    for (a, b), (c, d) in zip(got, want):
        assert np.max(np.abs(a - c)) <= 1e-11 * max(1.0, np.max(np.abs(c)))
        assert np.max(np.abs(b - d)) <= 1e-11 * max(1.0, np.max(np.abs(d)))


def test_interpolation_exact_on_parity_polynomials(tmp_path):
    """A field r^s * (polynomial in r^2) whose parity across the axis is that
    of (m Mp + S) is reproduced exactly (to rounding) on another mesh: the
    mirrored points extend it smoothly and 2KL+1-point Taylor interpolation
    is exact for degree <= 2KL."""
    from pipeflow.statefile import state_read
    N_, N, K, M, Mp = 24, 17, 2, 3, 1
    r_, r = _mesh(N_), _mesh(N)
    H = IO.harmonics(K, M)
    _, mm = O.harmonics(K, M)

    def field(x, S):
        out = np.empty((x.size, H))
        for nh in range(H):
            s = (mm[nh] * Mp + S) % 2  # odd in r when s == 1
            out[:, nh] = x ** s * (1.0 - 0.5 * x ** 2 + 0.25 * x ** 4 + 0.1 * nh * x ** 6)
        return out

    st = [(field(r_, S), -field(r_, S)) for S in (1, 1, 0)]
    p = str(tmp_path / "poly.cdf")
    IO.write_like_reference(p, N_, K, M, Mp, r_, st)
    got, _, _ = state_read(p, N, K, M, Mp, r)
    for (a, b), S in zip(got, (1, 1, 0)):  # the Taylor systems near the wall are ill-conditioned
        assert np.max(np.abs(a - field(r, S))) < 1e-9
        assert np.max(np.abs(b + field(r, S))) < 1e-9


def test_missing_file_and_wrong_mp_are_errors(tmp_path):
    import pipeflow as P
    from pipeflow.statefile import state_read
    with pytest.raises(P.PipeflowError, match="not found"):
        state_read(str(tmp_path / "nope.cdf"), 8, 2, 2, 1, _mesh(8))
    p = str(tmp_path / "mp.cdf")
    IO.write_like_reference(p, 8, 2, 4, 2, _mesh(8), _state(8, 2, 4, 5))
    with pytest.raises(P.PipeflowError, match="Mp"):
        state_read(p, 8, 2, 4, 1, _mesh(8))
    # a truncated file and a file that is not netCDF are errors, not crashes
    data = open(p, "rb").read()
    for k, blob in enumerate((data[:len(data) // 2], data[:40], b"not a netCDF file at all")):
        q = str(tmp_path / f"bad{k}.cdf")
        open(q, "wb").write(blob)
        with pytest.raises(P.PipeflowError):
            state_read(q, 8, 2, 4, 2, _mesh(8))


@pytest.mark.gpu
def test_pipe_save_load_round_trip_and_regrid(tmp_path):
    import pipeflow as P
    cfg = P.PipeConfig(N=24, K=6, M=5, Re=2000.0, alpha=1.25, dt=0.01)
    a = P.Pipe(cfg)
    a.vel_matrices()
    P.seeded_state(a, 11, 1e-3)
    for _ in range(3):
        a.timestep()
    p = str(tmp_path / "state0001.cdf.dat")
    a.io_save_state(p)
    b = P.Pipe(cfg)
    assert b.io_load_state(p, time_from_file=True) == 0
    assert b.tim.t == a.tim.t
    for (x, y), (u, v) in zip(a.get_state(), b.get_state()):
        assert np.array_equal(x, u) and np.array_equal(y, v)
    # onto another resolution: what pf_state_read gives, then a step runs
    cfg2 = P.PipeConfig(N=20, K=4, M=6, Re=2000.0, alpha=1.25, dt=0.01)
    c = P.Pipe(cfg2)
    assert c.io_load_state(p) & 7 == 7
    want, _ = IO.load_state(p, 20, 4, 6, 1, c.mes_D()["r"])
    for (x, y), (u, v) in zip(c.get_state(), want):
        assert np.max(np.abs(x - u)) < 1e-11 and np.max(np.abs(y - v)) < 1e-11
    c.vel_matrices()
    c.timestep()
    assert math.isfinite(c.energy())
