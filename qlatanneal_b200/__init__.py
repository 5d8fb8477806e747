"""qlatanneal_b200 -- qanneal's Monte Carlo sweep engine on NVIDIA B200 (sm_100a).

Drop-in for qanneal's annealer classes and ``solve()`` with ``backend="cuda"``:
the same class names, constructor arguments, result fields and error types,
running whole batched runs on the GPU through the C ABI in include/qa_gpu.h.
"""
from .models import (  # noqa: F401
    State,
    DenseIsing,
    SparseEdge,
    SparseIsing,
    QUBO,
    HigherOrderIsing,
    AnnealSchedule,
    SQASchedule,
    magnetization,
    overlap,
)
from .annealers import (  # noqa: F401
    AnnealResult,
    SQAResult,
    SQAParallelTemperingResult,
    SQAChiResult,
    RunStats,
    Annealer,
    SQAAnnealer,
    SQAParallelTemperingAnnealer,
    SQAChiAnnealer,
)

version_major, version_minor, version_patch = 2, 0, 0


def version_string() -> str:
    return f"{version_major}.{version_minor}.{version_patch}"


__version__ = "0.1.0"
