"""diffmpc_b200: B200-native (sm_100a) batched differentiable MPC inner solve.

Drop-in for the reference's ``diffmpc.solvers`` SQP/PCG API: the same class
and NamedTuple names (``SQPSolver``, ``SQPSolution``, ``PCGOptimalControl`` ...)
backed by hand-written CUDA kernels reached through the C ABI of
``libdmpc.so`` (``include/dmpc.h``).
"""

from .dynamics import (  # noqa: F401
    CartpoleDynamics,
    Dynamics,
    LinearDynamics,
    QuadrotorDynamics,
    SpacecraftAttitudeDynamics,
    SpacecraftDynamics,
)
from .pcg import (  # noqa: F401
    PCGDebugOutput,
    PCGOptimalControl,
    QPCostParameters,
    QPDynamicsCostPremultipliedMatrices,
    QPDynamicsParameters,
    QPParameters,
    QPSolution,
    SchurComplementMatrices,
)
from .problem import (  # noqa: F401
    OptimalControlProblem,
    check_parameters_dictionary_or_raise_errors,
    load_problem_params,
    load_solver_params,
)
from .sqp import DEFAULT_SOLVER_PARAMS, SolverReturnStatus, SQPSolution, SQPSolver  # noqa: F401
