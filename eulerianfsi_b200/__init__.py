"""B200 (sm_100a) implementation of EulerianFSI.jl's four-stage IMEX fractional step.

The public API mirrors the reference's Julia names; the step itself runs in the
CUDA library ``libefsi.so`` behind the C-ABI declared in ``include/efsi.h``.
"""
from .boundary import (AdvectiveOutflow, BoundaryConditionSetup, Dirichlet, MixedBoundary, Neumann,
                       Periodic, has_dirichlet, is_periodic_x, is_periodic_y)
from .errors import (ArgumentError, CUDAError, DimensionMismatch, DomainError, EFSIError,
                     SolverError, UnsupportedError)
from .imex import (FSIBoundaryConditions, FSIModels, FSIState, IMEXContext, IMEXWorkspace,
                   ProjectionResult, StepReport, allocate_imex_workspace, build_imex_context,
                   integrate_step, make_velocity_compatible)
from .mesh import MACGrid, MeshMetrics, build_mesh_metrics, generate_grid
from .models import *  # noqa: F401,F403  (model types mirror the reference constructors)
