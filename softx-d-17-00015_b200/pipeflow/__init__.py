"""B200-native timestep hot path of the openpipeflow pipe-flow DNS.

The compute runs in libpipeflow_b200.so (hand-written sm_100a CUDA behind a
C ABI, include/pipeflow_b200.h); this package is the host-side mirror of the
reference's Fortran module API over that ABI.
"""
from ._lib import PF_LD_AUTO, PF_LD_PAIRED, PF_LD_REBUILT, PF_LD_STREAMED, PF_LD_WARPRING, PF_PREC_FP64, PF_PREC_MIXED, KL, load  # noqa: F401
from .api import Batch, Coll, LUMesh, Mesh, Phys, Pipe, PipeConfig, PipeflowError, Server  # noqa: F401
from .ic import seeded_state, vector_potential_host  # noqa: F401
from .tune import Tuner  # noqa: F401
