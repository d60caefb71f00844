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


# ---------------------------------------------------------------- diodes
GAAS = dict(eps_r=12.9, Nc=4.7e23, Nv=9.0e24, Ec=1.424, Ev=0.0, mu_n=0.85, mu_p=0.04, T=300.0)


def intrinsic_density(T=300.0, Nc=GAAS["Nc"], Nv=GAAS["Nv"], Ec=GAAS["Ec"], Ev=GAAS["Ev"]):
    return math.sqrt(Nc * Nv * math.exp((Ev - Ec) * EV / (KB * T)))


def lcn_potential(doping, T=300.0):
    """Local charge neutrality potential in volts (src/thermodynamic_equilibrium.cpp:31-42)."""
    Nc, Nv, Ec, Ev = GAAS["Nc"], GAAS["Nv"], GAAS["Ec"] * EV, GAAS["Ev"] * EV
    U_T = T * KB / Q
    ni2 = Nc * Nv * math.exp((Ev - Ec) / (T * KB))
    return (Ec + Ev) / (2 * Q) + U_T / 2 * math.log(Nv / Nc) + U_T * math.asinh(doping / (2 * math.sqrt(ni2)))


def density(c, qf, V, T=300.0):
    """compute_density (include/solver.h:378-412)."""
    if c == Component.n:
        return GAAS["Nc"] * math.exp((Q * (V - qf) - GAAS["Ec"] * EV) / (KB * T))
    return GAAS["Nv"] * math.exp((Q * (qf - V) + GAAS["Ev"] * EV) / (KB * T))


def diode(dim=2, m=32, k=1, bias=0.0, N_D=1e23, N_A=1e23, x_j=0.5, length=1.0,
          tau=(1.0, 1.0, 1.0), srh_tau=1e-9, scale_length=1e-6, flux=DDFluxType.use_cell,
          nonlinear=None, precision=0):
    """p-n diode on [0, length]^dim (mesh units of scale_length metres): step
    doping along x, ohmic Dirichlet contacts on the x faces (bias on the p
    side, x = length), homogeneous Neumann elsewhere, constant mobilities,
    SRH recombination (three-argument form with the physical ni)."""
    mesh = StructuredMesh(dim, [m] * dim, [0.0] * dim, [length] * dim, colorize=True)
    doping = StepDoping(x_j * length, N_D, N_A)
    Vn = lcn_potential(N_D)
    Vp = lcn_potential(-N_A) + bias
    bh = BoundaryConditionHandler()
    contact_V = {0: Vn, 1: Vp}
    contact_qf = {0: 0.0, 1: bias}
    for bid in (0, 1):
        bh.add_boundary_condition(bid, BCT.DIRICHLET, Component.V, contact_V[bid])
        bh.add_boundary_condition(bid, BCT.DIRICHLET, Component.n,
                                  density(Component.n, contact_qf[bid], contact_V[bid]))
        bh.add_boundary_condition(bid, BCT.DIRICHLET, Component.p,
                                  density(Component.p, contact_qf[bid], contact_V[bid]))
    pb = Problem(mesh, HomogeneousPermittivity(GAAS["eps_r"] * EPSILON0),
                 HomogeneousMobility(GAAS["mu_n"], Component.n),
                 HomogeneousMobility(GAAS["mu_p"], Component.p),
                 ShockleyReadHallFixedTemperature(intrinsic_density(), srh_tau, srh_tau),
                 GAAS["T"], doping, bh, GAAS["Nc"], GAAS["Nv"], GAAS["Ec"], GAAS["Ev"])
    adim = Adimensionalizer(scale_length, Q / KB, max(N_D, N_A), 1.0)
    # tau given in rescaled units -> physical values for the parameter object
    phys_tau = [tau[c] * adim.get_tau_rescaling_factor(c) for c in range(3)]
    prm = FixedTauNPSolverParameters(k, k, k, nonlinear or NonlinearSolverParameters(1e-10, 1e-10, 100),
                                     phys_tau[0], phys_tau[1], phys_tau[2],
                                     dd_flux_type=flux, precision=precision)
    return pb, prm, adim


def set_bias(problem, bias):
    """Replace the contact conditions for a new bias (replace_boundary_condition,
    src/np_solver.cpp:2160-2233); the p contact (id 1) carries the bias."""
    N_A = -problem.doping.value([[1e30, 0, 0]])[0]
    Vp = lcn_potential(-N_A) + bias
    bh = problem.boundary_handler
    bh.replace_boundary_condition(1, BCT.DIRICHLET, Component.V, Vp)
    bh.replace_boundary_condition(1, BCT.DIRICHLET, Component.n, density(Component.n, bias, Vp))
    bh.replace_boundary_condition(1, BCT.DIRICHLET, Component.p, density(Component.p, bias, Vp))
