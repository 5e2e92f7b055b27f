"""The allocation-free transform entry point (pf_tra_coll2phys_noalloc).

It exists for callers of this library that cannot allocate device memory --
their memory belongs to another allocator or pool, or they must not allocate
inside their own step loop -- so it takes only device pointers the caller
owns and keeps its scratch in a static device array.  These checks call it
through the C ABI twice in a row and compare each result with the
context-based pf_tra_coll2phys on the same input, at the FP64 tolerance of
the other transform tests.  The file name makes pytest collect it last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# together these run every built transform length (3K and 3M in 12, 15, 18,
# 24, 36, 48, 72, 96, 144, 192, 288, 384) through the allocation-free kernels
CASES = [dict(N=40, K=24, M=16), dict(N=64, K=128, M=48), dict(N=16, K=5, M=4),
         dict(N=12, K=6, M=8), dict(N=20, K=12, M=32), dict(N=16, K=32, M=64), dict(N=10, K=4, M=96)]


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("dims", CASES, ids=lambda d: "N{N}K{K}M{M}".format(**d))
def test_noalloc_transform_matches_context_transform(dims):
    import torch
    import pipeflow as P
    from pipeflow import _lib as L

    lib = L.load()
    N, K, M = dims["N"], dims["K"], dims["M"]
    pipe = P.Pipe(P.PipeConfig(N=N, K=K, M=M))
    H, Z, Th = pipe.H, pipe.Z, pipe.Th
    rng = np.random.default_rng(17)
    out = torch.empty(N * Th * Z, dtype=torch.float64, device="cuda")
    for call in range(2):
        re = rng.standard_normal((N, H))
        im = rng.standard_normal((N, H))
        # the context-based entry point
        c = pipe.coll(re, im)
        p = pipe.phys()
        pipe.tra_coll2phys(c, p)
        ref = p.download()
        # the allocation-free one, on device arrays in the coll layout re[nh*N + n]
        d_re = torch.from_numpy(np.ascontiguousarray(re.T)).to("cuda")
        d_im = torch.from_numpy(np.ascontiguousarray(im.T)).to("cuda")
        out.fill_(np.nan)
        stream = torch.cuda.current_stream().cuda_stream
        st = lib.pf_tra_coll2phys_noalloc(N, K, M, C.c_void_p(d_re.data_ptr()), C.c_void_p(d_im.data_ptr()),
                                          C.c_void_p(out.data_ptr()), C.c_void_p(stream))
        assert st == 0, lib.pf_last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(N, Th, Z)
        assert np.all(np.isfinite(got))
        assert _rel(got, ref) < 1e-13, (call, _rel(got, ref))
    pipe.close()


def test_noalloc_rejects_sizes_over_the_static_scratch():
    from pipeflow import _lib as L
    lib = L.load()
    one = C.c_void_p(16)  # never dereferenced: the size check fails first
    st = lib.pf_tra_coll2phys_noalloc(128, 128, 48, one, one, one, None)
    assert st == -1
    assert b"exceeds" in lib.pf_last_error()
    st = lib.pf_tra_coll2phys_noalloc(16, 7, 4, one, one, one, None)  # 3K = 21 not built
    assert st == -1
    assert b"not among the built" in lib.pf_last_error()
