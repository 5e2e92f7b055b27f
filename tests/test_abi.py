"""C-ABI library checks that need no GPU: the library loads, exports every
symbol the header declares, refuses work without a device, and its host-side
radial mesh matches the oracle (meshs.f90:66-225)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import pipeflow_oracle as O

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "pipeflow_b200.h"


def _declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^(?:int|const char \*)\s*(pf_[a-z0-9_]+)\(", text, re.M)))


def test_library_loads_and_exports_header_symbols():
    from pipeflow import _lib
    lib = _lib.load()
    names = _declared()
    assert len(names) > 60
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(_lib.declared_symbols()) == names


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    import pipeflow as P
    with pytest.raises(P.PipeflowError) as e:
        P.Pipe(P.PipeConfig(N=16, K=4, M=4))
    assert e.value.status == -7


def test_bad_config_rejected():
    from pipeflow import _lib
    lib = _lib.load()
    c = _lib.pf_config()
    c.N, c.K, c.M, c.Mp = 4, 4, 4, 1
    c.Re, c.alpha = 2000.0, 1.25
    h = C.c_void_p()
    assert lib.pf_ctx_create(C.byref(c), -1, C.byref(h)) == -1
    assert b"N must exceed" in lib.pf_last_error()


@pytest.mark.parametrize("N", [16, 40, 64])
def test_host_mesh_matches_oracle(N):
    from pipeflow import _lib
    lib = _lib.load()
    KL = 4
    r = np.empty(N)
    dr = np.empty((KL, N, 2 * KL + 1))
    rl = np.empty((N, 2 * KL + 1))
    d0 = np.empty((KL + 1, KL + 1))
    d1 = np.empty((KL + 1, KL + 1))
    w = np.empty(N)
    dp = lambda a: a.ctypes.data_as(_lib.DP)
    assert lib.pf_mes_compute(N, None, dp(r), dp(dr), dp(rl), dp(d0), dp(d1), dp(w)) == 0
    D = O.mes_rdom_init(O.default_mesh(N))
    assert np.max(np.abs(r - D.r)) < 1e-15
    for i in range(KL):
        ref = D.dr[i]
        got = dr[i].T
        assert np.max(np.abs(got - ref)) <= 1e-10 * np.max(np.abs(ref))
    assert np.max(np.abs(rl.T - D.radLap)) <= 1e-10 * np.max(np.abs(D.radLap))
    assert np.max(np.abs(d0.T - D.dr0)) <= 1e-11 * np.max(np.abs(D.dr0))
    assert np.max(np.abs(d1.T - D.dr1)) <= 1e-11 * np.max(np.abs(D.dr1))
    assert np.max(np.abs(w - D.intrdr)) < 1e-14


def test_custom_mesh_validation():
    from pipeflow import _lib
    lib = _lib.load()
    N = 16
    r = np.linspace(0.05, 0.9, N)  # does not end at r=1 (meshs.f90:87-88)
    out = np.empty(N)
    st = lib.pf_mes_compute(N, r.ctypes.data_as(_lib.DP), out.ctypes.data_as(_lib.DP),
                            None, None, None, None, None)
    assert st == -1 and b"mesh.in err 3" in lib.pf_last_error()


def test_seeded_potential_matches_oracle():
    from pipeflow.ic import vector_potential_host
    p = O.Pipe(O.PipeConfig(N=20, K=5, M=6, Mp=2))
    ref = O.vector_potential(p, 7)
    got = vector_potential_host(5, 6, 2, p.mes_D.r, 7)
    for (re, im), c in zip(got, ref):
        assert np.array_equal(re, c.re) and np.array_equal(im, c.im)
