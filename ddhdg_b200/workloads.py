"""Diode workloads: seeded synthetic p-n diodes with the shapes of the
benchmark configurations (GaAs-like material of
tests/thermodynamic_equilibrium.cpp:99-115 in the reference, mobilities of
its examples/residual.ipynb, SRH recombination with the physical intrinsic
density, ohmic contacts on the x faces as in the notebook's
copy_boundary_conditions)."""

import math

from .functions import EPSILON0, EV, KB, Q, StepDoping
from .problem import (Adimensionalizer, BoundaryConditionHandler, BoundaryConditionType as BCT,
                      Component, DDFluxType, FixedTauNPSolverParameters, HomogeneousMobility,
                      HomogeneousPermittivity, NonlinearSolverParameters, Problem,
                      ShockleyReadHallFixedTemperature, StructuredMesh)

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


def bias_sweep(solver, problem, biases, absolute_tol=None, relative_tol=None,
               max_number_of_iterations=None, callback=None):
    """Forward bias sweep with warm starts (the second diode configuration:
    0 to 0.8 V in 0.05 V steps): for every bias the contact conditions are
    replaced on the device (replace_boundary_condition,
    src/np_solver.cpp:2160-2233, without rebuilding the sparsity) and Newton
    starts from the previous bias point's solution.  Returns
    [(bias, NonlinearIterationResults)]; `callback(bias, solver, result)` is
    called after every point."""
    out = []
    for v in biases:
        set_bias(problem, float(v))
        solver.update_boundary_tables()
        res = solver.run(absolute_tol, relative_tol, max_number_of_iterations)
        out.append((float(v), res))
        if callback is not None:
            callback(float(v), solver, res)
    return out


def batch_diodes(n, seed=3, sizes=(16, 128), degrees=(1, 2, 3), doping=(1e21, 1e24), junction=(0.3, 0.7),
                 dim=2, mixed=False):
    """Seeded heterogeneous batch of diodes shaped like the batched benchmark
    configuration: mesh cells per side uniform in `sizes`, degree uniform in
    `degrees`, doping (N_D = N_A) log-uniform in `doping`, junction position
    uniform in `junction` (fraction of the length); with `mixed`, the
    devices whose degree has a mixed-precision kernel (3 (k+1)^dim <= 32)
    condense with the FP32 Jacobian, the others in FP64.  Returns a list of
    (problem, parameters, adimensionalizer, spec dict)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        m = int(rng.integers(sizes[0], sizes[1] + 1))
        k = int(rng.choice(degrees))
        N = float(10 ** rng.uniform(math.log10(doping[0]), math.log10(doping[1])))
        xj = float(rng.uniform(*junction))
        prec = 1 if mixed and 3 * (k + 1) ** dim <= 32 else 0
        pb, prm, adim = diode(dim=dim, m=m, k=k, N_D=N, N_A=N, x_j=xj, precision=prec)
        out.append((pb, prm, adim, dict(m=m, k=k, doping=N, x_j=xj, precision=prec)))
    return out
