"""ddhdg_b200: B200-native (sm_100a) HDG hot path of DDHDG (spiani/ddhdg) for
the Van Roosbroeck drift-diffusion system -- per-cell assembly, static
condensation onto the trace and cell reconstruction behind the reference's
``NPSolver`` / ``Problem`` API."""

from .functions import (AnalyticFunction, ConstantFunction, Function, FunctionTimesScalar,
                        PiecewiseFunction, StepDoping, as_function)
from .problem import (Adimensionalizer, BoundaryConditionHandler, BoundaryConditionType,
                      CellFaceTauNPSolverParameters, Component, DDFluxType, Displacement,
                      FixedTauNPSolverParameters, HomogeneousMobility, HomogeneousPermittivity,
                      LinearRecombinationTerm, NonlinearSolverParameters, NPSolverParameters,
                      Precision, Problem, ShockleyReadHallFixedTemperature, StructuredMesh)


def __getattr__(name):
    # the solver needs the CUDA library; import it lazily so that the problem
    # description classes stay usable on machines without a GPU
    if name in ("NPSolver", "NonlinearIterationResults"):
        from . import solver

        return getattr(solver, name)
    raise AttributeError(name)
