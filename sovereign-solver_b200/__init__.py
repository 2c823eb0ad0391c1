"""B200-native PDHG LP engine (drop-in for sovereign-solver's ``Pdhg::solve``).

The engine is ``libpdhg_b200.so`` (CUDA kernels + C-ABI, include/pdhg_b200.h).
This package holds its Python face (``pdhg``), the LP container (``problem``),
the seeded workload generators (``lpgen``) and the learned warm start
(``mlp``: the network, ``warmstart``: basis, training, gated starts), the
MPS reader (``mps``) and the split of a batch and of the network's training
across GPUs (``shard``).
"""
from .problem import INF, Problem  # noqa: F401
from . import lpgen  # noqa: F401
from . import mlp  # noqa: F401
from . import warmstart  # noqa: F401
from . import mps  # noqa: F401
from . import shard  # noqa: F401
from .pdhg import (  # noqa: F401
    CancellationToken, Engine, Pdhg, PdhgError, PdhgOptions, PdhgResult, csr_spmv, project_box,
    scaling,
)
