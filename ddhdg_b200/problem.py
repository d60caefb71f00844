"""Problem description objects: the host-side mirror of the reference's
``Ddhdg::Problem`` (include/problem.h:13-46), its material classes
(include/permittivity.h, include/mobility.h, include/recombination_term.h),
``BoundaryConditionHandler`` (include/boundary_conditions.h:123-200),
``Adimensionalizer`` (include/adimensionalizer.h:11-270) and the solver
parameter classes (include/np_solver_parameters.h:34-404).

Meshes are structured Cartesian grids of segments, quadrilaterals or
hexahedra (the reference's ``GridGenerator::hyper_cube`` +
``refine_global`` and ``subdivided_hyper_rectangle`` meshes); boundary ids
follow deal.II's ``colorize`` convention (face ``2a`` at the lower end of axis
``a`` has id ``2a``, the upper end ``2a+1``) or are all ``0``.
"""

from __future__ import annotations

import enum
from dataclasses import dataclass, field
from typing import Dict, Optional, Sequence, Tuple

from .functions import KB, Q, Function, as_function


class Component(enum.IntEnum):
    """include/components.h:12-19."""

    V = 0
    n = 1
    p = 2
    phi_n = 3
    phi_p = 4


class Displacement(enum.IntEnum):
    E = 0
    Wn = 1
    Wp = 2


class BoundaryConditionType(enum.IntEnum):
    """include/boundary_conditions.h:9-14."""

    DIRICHLET = 0
    NEUMANN = 1
    ROBIN = 2


class DDFluxType(enum.IntEnum):
    """include/np_solver_parameters.h:34-39."""

    use_cell = 0
    use_trace = 1
    qiu_shi_stabilization = 2


class StructuredMesh:
    """Axis-aligned structured mesh of ``n[0] x ... x n[dim-1]`` cells on the
    box ``[lower, upper]`` (mesh coordinates are in units of the
    adimensionalizer's ``scale_length``, as in the reference)."""

    def __init__(self, dim: int, n: Sequence[int], lower: Sequence[float],
                 upper: Sequence[float], colorize: bool = True):
        if dim not in (1, 2, 3):
            raise ValueError("dim must be 1, 2 or 3")
        self.dim = int(dim)
        self.n = tuple(int(v) for v in n)[:dim]
        self.lower = tuple(float(v) for v in lower)[:dim]
        self.upper = tuple(float(v) for v in upper)[:dim]
        if len(self.n) != dim or len(self.lower) != dim or len(self.upper) != dim:
            raise ValueError("n, lower and upper need one entry per axis")
        if min(self.n) < 1:
            raise ValueError("every axis needs at least one cell")
        self.colorize = bool(colorize)

    @classmethod
    def hyper_cube(cls, dim: int, left: float = 0.0, right: float = 1.0,
                   refinements: int = 0, colorize: bool = False):
        """``GridGenerator::hyper_cube(tria, left, right, colorize)`` followed
        by ``refine_global(refinements)``."""
        m = 2 ** int(refinements)
        return cls(dim, [m] * dim, [left] * dim, [right] * dim, colorize)

    def refine_global(self, times: int = 1):
        f = 2 ** int(times)
        self.n = tuple(v * f for v in self.n)

    @property
    def h(self) -> Tuple[float, ...]:
        return tuple((u - l) / m for l, u, m in zip(self.lower, self.upper, self.n))

    @property
    def n_cells(self) -> int:
        r = 1
        for v in self.n:
            r *= v
        return r


class HomogeneousPermittivity:
    def __init__(self, epsilon: float):
        self.epsilon = float(epsilon)


class HomogeneousMobility:
    def __init__(self, mu: float, component: Component = Component.n):
        self.mu = float(mu)
        self.component = Component(component)


class LinearRecombinationTerm:
    """R = a(x) + (b(x) n + c(x) p) (src/recombination_term.cpp:116-160)."""

    kind = "linear"

    def __init__(self, constant_term=0.0, n_linear_coefficient=0.0,
                 p_linear_coefficient=0.0):
        self.constant_term = as_function(constant_term)
        self.n_linear_coefficient = as_function(n_linear_coefficient)
        self.p_linear_coefficient = as_function(p_linear_coefficient)


class ShockleyReadHallFixedTemperature:
    """SRH recombination (src/recombination_term.cpp:433-575).

    The seven-argument form stores ``Nc Nv exp((Ev-Ec)/(kB T))`` -- that is
    ni squared -- as the intrinsic concentration, exactly like the reference
    (include/recombination_term.h:219-229); the three-argument form takes ni.
    """

    kind = "srh"

    def __init__(self, intrinsic_carrier_concentration: float,
                 electron_life_time: float, hole_life_time: float):
        self.intrinsic_carrier_concentration = float(intrinsic_carrier_concentration)
        self.electron_life_time = float(electron_life_time)
        self.hole_life_time = float(hole_life_time)

    @classmethod
    def from_band_parameters(cls, conduction_band_density, valence_band_density,
                             conduction_band_edge_energy, valence_band_edge_energy,
                             temperature, electron_life_time, hole_life_time):
        import math

        ni = (conduction_band_density * valence_band_density *
              math.exp((valence_band_edge_energy - conduction_band_edge_energy) /
                       (KB * temperature)))
        return cls(ni, electron_life_time, hole_life_time)


class BoundaryConditionHandler:
    def __init__(self):
        self.dirichlet: Dict[int, Dict[Component, Function]] = {}
        self.neumann: Dict[int, Dict[Component, Function]] = {}

    def add_boundary_condition(self, boundary_id: int, bc_type, component, f):
        bc_type = BoundaryConditionType(bc_type)
        component = Component(component)
        table = self._table(bc_type)
        if component in self.dirichlet.get(boundary_id, {}) or \
                component in self.neumann.get(boundary_id, {}):
            raise ValueError("Trying to overwrite a boundary condition")
        table.setdefault(int(boundary_id), {})[component] = as_function(f)

    def replace_boundary_condition(self, boundary_id: int, bc_type, component, f) -> bool:
        """Returns True when the type of the condition changed (which forces a
        new constraint set), like the reference."""
        bc_type = BoundaryConditionType(bc_type)
        component = Component(component)
        old = None
        for t, tab in ((BoundaryConditionType.DIRICHLET, self.dirichlet),
                       (BoundaryConditionType.NEUMANN, self.neumann)):
            if component in tab.get(boundary_id, {}):
                old = t
                del tab[boundary_id][component]
        self._table(bc_type).setdefault(int(boundary_id), {})[component] = as_function(f)
        return old != bc_type

    def _table(self, bc_type):
        if bc_type == BoundaryConditionType.DIRICHLET:
            return self.dirichlet
        if bc_type == BoundaryConditionType.NEUMANN:
            return self.neumann
        raise NotImplementedError("Robin boundary conditions are not implemented by the reference either")

    def has_dirichlet_boundary_conditions(self, boundary_id: int, component) -> bool:
        return Component(component) in self.dirichlet.get(int(boundary_id), {})

    def has_neumann_boundary_conditions(self, boundary_id: int, component) -> bool:
        return Component(component) in self.neumann.get(int(boundary_id), {})

    def get_function(self, boundary_id: int, component) -> Optional[Function]:
        c = Component(component)
        if c in self.dirichlet.get(int(boundary_id), {}):
            return self.dirichlet[int(boundary_id)][c]
        if c in self.neumann.get(int(boundary_id), {}):
            return self.neumann[int(boundary_id)][c]
        return None

    def copy(self):
        h = BoundaryConditionHandler()
        h.dirichlet = {k: dict(v) for k, v in self.dirichlet.items()}
        h.neumann = {k: dict(v) for k, v in self.neumann.items()}
        return h


class Problem:
    def __init__(self, mesh: StructuredMesh, permittivity: HomogeneousPermittivity,
                 electron_mobility: HomogeneousMobility,
                 hole_mobility: HomogeneousMobility, recombination_term,
                 temperature, doping, boundary_condition_handler: BoundaryConditionHandler,
                 conduction_band_density: float, valence_band_density: float,
                 conduction_band_edge_energy: float = 0.0,
                 valence_band_edge_energy: float = 0.0):
        self.mesh = mesh
        self.permittivity = permittivity
        self.electron_mobility = electron_mobility
        self.hole_mobility = hole_mobility
        self.recombination_term = recombination_term
        self.temperature = as_function(temperature)
        self.doping = as_function(doping)
        self.boundary_handler = boundary_condition_handler
        self.band_density = {Component.n: float(conduction_band_density),
                             Component.p: float(valence_band_density)}
        self.band_edge_energy = {Component.n: float(conduction_band_edge_energy),
                                 Component.p: float(valence_band_edge_energy)}

    @property
    def dim(self):
        return self.mesh.dim


class Adimensionalizer:
    """Scaling factors of include/adimensionalizer.h:15-262."""

    def __init__(self, scale_length: float = 1.0, temperature_magnitude: float = Q / KB,
                 doping_magnitude: float = 1.0, mobility_magnitude: float = 1.0):
        self.scale_length = float(scale_length)
        self.temperature_magnitude = float(temperature_magnitude)
        self.doping_magnitude = float(doping_magnitude)
        self.mobility_magnitude = float(mobility_magnitude)

    def get_component_rescaling_factor(self, c) -> float:
        c = Component(c)
        if c == Component.V:
            return self.temperature_magnitude * KB / Q
        if c in (Component.n, Component.p):
            return self.doping_magnitude
        raise ValueError("invalid component")

    def get_displacement_rescaling_factor(self, d) -> float:
        return self.get_component_rescaling_factor(int(d)) / self.scale_length

    def get_neumann_boundary_condition_rescaling_factor(self, c) -> float:
        c = Component(c)
        if c == Component.V:
            return Q
        num = KB * self.doping_magnitude * self.temperature_magnitude * self.mobility_magnitude
        return num / (self.scale_length * self.scale_length)

    def get_permittivity_rescaling_factor(self) -> float:
        den = self.temperature_magnitude * KB
        num = self.scale_length * self.scale_length * Q * Q * self.doping_magnitude
        return num / den

    def get_thermal_voltage_rescaling_factor(self) -> float:
        return self.temperature_magnitude * KB / Q

    def get_mobility_rescaling_factor(self) -> float:
        return self.mobility_magnitude

    def get_recombination_rescaling_factor(self) -> float:
        num = KB * self.doping_magnitude * self.temperature_magnitude * self.mobility_magnitude
        den = self.scale_length * self.scale_length * Q
        return num / den

    def get_tau_rescaling_factor(self, c) -> float:
        c = Component(c)
        Tv = self.temperature_magnitude * KB / Q
        if c == Component.V:
            return Q * self.doping_magnitude / Tv
        return Tv * self.mobility_magnitude / (self.scale_length * self.scale_length)


@dataclass
class NonlinearSolverParameters:
    """include/np_solver_parameters.h:48-64."""

    absolute_tolerance: float = 1e-10
    relative_tolerance: float = 1e-10
    max_number_of_iterations: int = 100
    alpha: float = 1.0


class Precision(enum.IntEnum):
    """Arithmetic of the local condensation on the device."""

    fp64 = 0
    mixed = 1  # FP32 factorisation of the local solver, FP64 residuals


class NPSolverParameters:
    """include/np_solver_parameters.h:261-296.  Only equal degrees for V, n and
    p are supported by the device kernels."""

    tau_computer = "fixed"

    def __init__(self, V_degree: int = 1, n_degree: int = 1, p_degree: int = 1,
                 nonlinear_parameters: NonlinearSolverParameters = None,
                 iterative_linear_solver: bool = False, multithreading: bool = True,
                 dd_flux_type: DDFluxType = DDFluxType.use_cell,
                 phi_linearize: bool = False, precision: Precision = Precision.fp64,
                 consistent_drift_jacobian: bool = False,
                 consistent_recombination_jacobian: bool = False):
        if not (V_degree == n_degree == p_degree):
            raise NotImplementedError("V, n and p must share one polynomial degree")
        self.degree = {Component.V: int(V_degree), Component.n: int(n_degree),
                       Component.p: int(p_degree)}
        self.nonlinear_parameters = nonlinear_parameters or NonlinearSolverParameters()
        self.iterative_linear_solver = bool(iterative_linear_solver)
        self.multithreading = bool(multithreading)
        self.dd_flux_type = DDFluxType(dd_flux_type)
        self.phi_linearize = bool(phi_linearize)
        self.precision = Precision(precision)
        # Off by default: the reference's Jacobian.  Its cell drift term
        # couples E with the sign opposite to the residual's derivative
        # (include/assembling_methods.template.h:500 and :522 against the
        # residual at :656 and :673) and its recombination derivatives miss
        # the doping magnitude (src/recombination_term.cpp:473-475 with
        # src/adimensionalizer.cpp:476-497).  Both options only change the
        # Jacobian, never the residual, so converged solutions are the same.
        self.consistent_drift_jacobian = bool(consistent_drift_jacobian)
        self.consistent_recombination_jacobian = bool(consistent_recombination_jacobian)

    @property
    def k(self) -> int:
        return self.degree[Component.V]


class FixedTauNPSolverParameters(NPSolverParameters):
    """include/np_solver_parameters.h:298-330 (defaults tau = 1, 1, 1)."""

    tau_computer = "fixed"

    def __init__(self, V_degree: int = 1, n_degree: int = 1, p_degree: int = 1,
                 nonlinear_parameters: NonlinearSolverParameters = None,
                 V_tau: float = 1.0, n_tau: float = 1.0, p_tau: float = 1.0,
                 iterative_linear_solver: bool = False, multithreading: bool = True,
                 dd_flux_type: DDFluxType = DDFluxType.use_cell,
                 phi_linearize: bool = False, precision: Precision = Precision.fp64,
                 consistent_drift_jacobian: bool = False,
                 consistent_recombination_jacobian: bool = False):
        super().__init__(V_degree, n_degree, p_degree, nonlinear_parameters,
                         iterative_linear_solver, multithreading, dd_flux_type,
                         phi_linearize, precision, consistent_drift_jacobian,
                         consistent_recombination_jacobian)
        self.tau = {Component.V: float(V_tau), Component.n: float(n_tau),
                    Component.p: float(p_tau)}

    def get_tau(self, c) -> float:
        return self.tau[Component(c)]


class CellFaceTauNPSolverParameters(NPSolverParameters):
    """Per cell and face tau values (include/np_solver_parameters.h:332-402);
    cells are addressed by their lexicographic index."""

    tau_computer = "cell_face"

    def __init__(self, *args, **kwargs):
        super().__init__(*args, **kwargs)
        self.face_tau: Dict[Tuple[int, int], Tuple[float, float, float]] = {}

    def clear(self):
        self.face_tau.clear()

    def set_face(self, cell: int, face: int, V_tau: float, n_tau: float, p_tau: float):
        self.face_tau[(int(cell), int(face))] = (float(V_tau), float(n_tau), float(p_tau))
