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
    ReplicaResult,
    MultiAnnealResult,
    ParallelTemperingResult,
    RunStats,
    Annealer,
    ReplicaAnnealer,
    ParallelTemperingAnnealer,
    SQAAnnealer,
    SQAParallelTemperingAnnealer,
    SQAChiAnnealer,
    BatchRunner,
    set_drift_check,
    set_update_order,
    get_update_order,
)
from ._lib import FieldDriftError  # noqa: F401
from .observers import (  # noqa: F401
    Observer,
    SweepObserver,
    MetricsObserver,
    StateTraceObserver,
    SQAObserver,
    SQASweepObserver,
    SQAMetricsObserver,
    SQAStateTraceObserver,
)

from .solver import (  # noqa: F401
    SolveResult,
    solve,
    auto_schedule_sa,
    auto_schedule_sqa,
    auto_schedule_sa_tuned,
    auto_schedule_sqa_tuned,
    auto_ladder_sqa_tuned,
    j_perp_from_beta_gamma,
    optimal_j_perp_params,
    j_rms_from_problem,
)

version_major, version_minor, version_patch = 2, 0, 0


def version_string() -> str:
    return f"{version_major}.{version_minor}.{version_patch}"


__version__ = "0.1.0"
