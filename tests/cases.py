"""Problem builders shared by the tests: restatements of the setups in the
reference's gtest suite (tests/*.cpp) and the diode workloads."""

import math

from ddhdg_b200.functions import EPSILON0, KB, Q, EV, PiecewiseFunction, StepDoping
from ddhdg_b200.problem import (Adimensionalizer, BoundaryConditionHandler,
                                BoundaryConditionType as BCT, CellFaceTauNPSolverParameters,
                                Component, DDFluxType, FixedTauNPSolverParameters,
                                HomogeneousMobility, HomogeneousPermittivity,
                                LinearRecombinationTerm, NonlinearSolverParameters, Problem,
                                ShockleyReadHallFixedTemperature, StructuredMesh)


def linear_potential(dim, max_it=1, flux=DDFluxType.use_cell):
    """tests/linear_potential.cpp:28-151."""
    mesh = StructuredMesh.hyper_cube(dim, -1, 1, refinements=3 - dim, colorize=False)
    bh = BoundaryConditionHandler()
    for i in range(2):
        bh.add_boundary_condition(i, BCT.DIRICHLET, Component.V, "x")
        bh.add_boundary_condition(i, BCT.DIRICHLET, Component.n, "0")
        bh.add_boundary_condition(i, BCT.DIRICHLET, Component.p, "0")
    pb = Problem(mesh, HomogeneousPermittivity(1.0), HomogeneousMobility(1.0, Component.n),
                 HomogeneousMobility(1.0, Component.p), LinearRecombinationTerm(0, 0, 0),
                 "q / kb", 0.0, bh, 1.0, 1.0, 0.0, 0.0)
    prm = FixedTauNPSolverParameters(2, 2, 2, NonlinearSolverParameters(1e-10, 1e-10, max_it),
                                     1, 1, 1, dd_flux_type=flux)
    return pb, prm, Adimensionalizer()


def neumann_linear(dim):
    """tests/neumann_boundary_conditions.cpp:8-158."""
    mesh = StructuredMesh.hyper_cube(dim, -1, 1, refinements=3 - dim, colorize=True)
    bh = BoundaryConditionHandler()
    for i in range(6):
        bh.add_boundary_condition(i, BCT.DIRICHLET, Component.n, 0.0)
        bh.add_boundary_condition(i, BCT.DIRICHLET, Component.p, 0.0)
    bh.add_boundary_condition(0, BCT.DIRICHLET, Component.V, -1.0)
    bh.add_boundary_condition(1, BCT.NEUMANN, Component.V, -1.0)
    for i in range(2, 6):
        bh.add_boundary_condition(i, BCT.NEUMANN, Component.V, 0.0)
    pb = Problem(mesh, HomogeneousPermittivity(1.0), HomogeneousMobility(1.0, Component.n),
                 HomogeneousMobility(1.0, Component.p), LinearRecombinationTerm(0, 0, 0),
                 "q / kb", 0.0, bh, 1.0, 1.0, 0.0, 0.0)
    prm = FixedTauNPSolverParameters(2, 2, 2)
    return pb, prm, Adimensionalizer()


def log_potential(dim, parameters, refinements=None):
    """tests/cell_face_tau_computer.cpp:8-118 (V = -2 ln x, n = 2/(x^2 q) on [1,2]^d)."""
    refinements = (4 - dim) if refinements is None else refinements
    mesh = StructuredMesh.hyper_cube(dim, 1, 2, refinements=refinements, colorize=False)
    bh = BoundaryConditionHandler()
    for i in range(2):
        bh.add_boundary_condition(i, BCT.DIRICHLET, Component.V, "-2 * log(x)")
        bh.add_boundary_condition(i, BCT.DIRICHLET, Component.n, "2 / (x^2 * q)")
        bh.add_boundary_condition(i, BCT.DIRICHLET, Component.p, 0.0)
    pb = Problem(mesh, HomogeneousPermittivity(1.0), HomogeneousMobility(1.0, Component.n),
                 HomogeneousMobility(1.0, Component.p), LinearRecombinationTerm(0, 0, 0),
                 "q / kb", 0.0, bh, 1.0, 1.0, 0.0, 0.0)
    return pb, parameters, Adimensionalizer(1, Q / KB, 1 / Q, 1)


def local_charge_neutrality_problem(refinements=4):
    """tests/local_charge_neutrality.cpp:8-118 (GaAs-like n+/i/p+ doping)."""
    dim = 2
    mesh = StructuredMesh.hyper_cube(dim, 0, 1, refinements=refinements, colorize=True)
    doping = PiecewiseFunction("0.1 - x", 1e22, PiecewiseFunction("x - 0.9", -1e23, 0.0))
    pb = Problem(mesh, HomogeneousPermittivity(12.9 * EPSILON0), HomogeneousMobility(1.0, Component.n),
                 HomogeneousMobility(1.0, Component.p), LinearRecombinationTerm(0, 0, 0),
                 300.0, doping, BoundaryConditionHandler(), 4.7e23, 9.0e24, 1.424, 0.0)
    return pb, FixedTauNPSolverParameters(1, 1, 1), Adimensionalizer(1, Q / KB, 1e23, 1)


from ddhdg_b200.workloads import (GAAS, density, diode, intrinsic_density,  # noqa: F401
                                  lcn_potential, set_bias)
