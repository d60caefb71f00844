"""``NPSolver``: the host-side mirror of ``Ddhdg::NPSolver<dim, Problem>``
(include/np_solver.h:44-914) on top of the C ABI.

Device memory comes from torch (plumbing only); every numerical stage of a
Newton step runs in the CUDA library: the per-cell condensation, the global
assembly, the global trace solve and the reconstruction.  The host prepares
the coefficient tables (doping, boundary data, tau) at the quadrature points
the library reports, exactly once per problem or boundary change.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

from . import _lib
from .functions import EV, KB, Q, as_function
from .problem import (Adimensionalizer, BoundaryConditionType, Component, DDFluxType,
                      NPSolverParameters, Problem)


def _torch():
    import torch

    return torch


@dataclass
class NonlinearIterationResults:
    """include/nonlinear_iteration_results.h."""

    converged: bool
    iterations: int
    last_update_norm: float


class NPSolver:
    def __init__(self, problem: Problem, parameters: NPSolverParameters,
                 adimensionalizer: Adimensionalizer = None, verbose: bool = False,
                 device: str = "cuda:0"):
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("NPSolver needs a CUDA device (sm_100a); there is no CPU path")
        self.L = _lib.load()
        self.problem = problem
        self.parameters = parameters
        self.adim = adimensionalizer or Adimensionalizer()
        self.verbose = verbose
        self.device = torch.device(device)
        self.stream = torch.cuda.current_stream(self.device)
        mesh = problem.mesh
        self.dim = mesh.dim
        self.k = parameters.k
        self.enabled = [True, True, True]
        self._ctx = ctypes.c_void_p()
        self._geometry()
        self._create()
        n_cell = self.ncells * self.Nc_all
        self.cell_state = torch.zeros(n_cell, dtype=torch.float64, device=self.device)
        self.trace_state = torch.zeros(self.nfaces * 3 * self.nf, dtype=torch.float64, device=self.device)

    # ----------------------------------------------------------- geometry
    def _geometry(self):
        mesh = self.problem.mesh
        d, k = self.dim, self.k
        self.n = list(mesh.n) + [1] * (3 - d)
        self.h = list(mesh.h) + [1.0] * (3 - d)
        self.origin = list(mesh.lower) + [0.0] * (3 - d)
        self.nb = (k + 1) ** d
        self.nf = (k + 1) ** (d - 1)
        self.nqc, self.nqf = self.nb, self.nf
        self.F = 2 * d
        self.Nc_all = 3 * (d + 1) * self.nb
        self.ncells = int(np.prod(self.n))
        qc = np.zeros((self.nqc, 3))
        qf = np.zeros((self.F, self.nqf, 3))
        sup = np.zeros(k + 1)
        dp = ctypes.POINTER(ctypes.c_double)
        _lib.check(self.L.ddhdg_reference_points(d, k, qc.ctypes.data_as(dp), qf.ctypes.data_as(dp),
                                                 sup.ctypes.data_as(dp)), "reference_points")
        self.qref_c, self.qref_f, self.support = qc, qf, sup
        cidx = np.arange(self.ncells)
        ci = np.stack([cidx % self.n[0], (cidx // self.n[0]) % self.n[1],
                       cidx // (self.n[0] * self.n[1])], 1)
        self.cell_idx = ci
        org, hh = np.array(self.origin), np.array(self.h)
        self.cell_qp = org + (ci[:, None, :] + qc[None]) * hh
        self.cell_fqp = org + (ci[:, None, None, :] + qf[None]) * hh
        # faces
        offs, exts = [0], []
        for a in range(d):
            e = [self.n[b] + (1 if b == a else 0) for b in range(d)]
            exts.append(e)
            offs.append(offs[-1] + int(np.prod(e)))
        self.nfaces = offs[-1]
        cf = np.zeros((self.ncells, self.F), dtype=np.int64)
        for f in range(self.F):
            a, side = f // 2, f % 2
            fi = ci.copy()
            fi[:, a] += side
            idx = np.zeros(self.ncells, dtype=np.int64)
            stride = 1
            for b in range(d):
                idx += fi[:, b] * stride
                stride *= exts[a][b]
            cf[:, f] = offs[a] + idx
        self.cell_faces = cf
        self.face_qp = np.zeros((self.nfaces, self.nqf, 3))
        self.face_bid = -np.ones(self.nfaces, dtype=np.int64)
        for f in range(self.F):
            self.face_qp[cf[:, f]] = self.cell_fqp[:, f]
            a, side = f // 2, f % 2
            on_b = ci[:, a] == ((self.n[a] - 1) if side else 0)
            self.face_bid[cf[on_b, f]] = (2 * a + side) if mesh.colorize else 0

    # ------------------------------------------------------------ tables
    def _tau_rescale(self, c):
        return self.adim.get_tau_rescaling_factor(c)

    def _bc_tables(self):
        bh = self.problem.boundary_handler
        bc = np.zeros((self.nfaces, 3), dtype=np.int32)
        val = np.zeros((self.nfaces, 3, self.nqf))
        bfaces = np.nonzero(self.face_bid >= 0)[0]
        for c in range(3):
            for bid in np.unique(self.face_bid[bfaces]):
                faces = bfaces[self.face_bid[bfaces] == bid]
                pts = self.face_qp[faces].reshape(-1, 3)
                if bh.has_dirichlet_boundary_conditions(int(bid), c):
                    bc[faces, c] = 1
                    val[faces, c] = (bh.dirichlet[int(bid)][Component(c)].value(pts).reshape(-1, self.nqf) /
                                     self.adim.get_component_rescaling_factor(c))
                elif bh.has_neumann_boundary_conditions(int(bid), c):
                    bc[faces, c] = 2
                    val[faces, c] = (bh.neumann[int(bid)][Component(c)].value(pts).reshape(-1, self.nqf) /
                                     self.adim.get_neumann_boundary_condition_rescaling_factor(c))
        return np.ascontiguousarray(bc), np.ascontiguousarray(val)

    def _create(self):
        pb, prm, adim = self.problem, self.parameters, self.adim
        D = _lib.ProblemDesc()
        D.dim, D.degree = self.dim, self.k
        for a in range(3):
            D.n[a] = self.n[a]
            D.origin[a] = self.origin[a]
            D.h[a] = self.h[a]
        for c in range(3):
            D.enabled[c] = int(self.enabled[c])
        D.flux = int(prm.dd_flux_type)
        D.phi_linearize = int(prm.phi_linearize)
        D.jacobian_fix = (1 if prm.consistent_drift_jacobian else 0) | \
            (2 if prm.consistent_recombination_jacobian else 0)
        D.precision = int(prm.precision)
        T = float(pb.temperature.value(np.zeros((1, 3)))[0])
        self.T = T
        D.eps = pb.permittivity.epsilon / adim.get_permittivity_rescaling_factor()
        D.mu_n = pb.electron_mobility.mu / adim.get_mobility_rescaling_factor()
        D.mu_p = pb.hole_mobility.mu / adim.get_mobility_rescaling_factor()
        D.temperature = T
        D.thermal_voltage_rescale = adim.get_thermal_voltage_rescaling_factor()
        D.V_rescale = adim.get_component_rescaling_factor(Component.V)
        D.n_rescale = adim.get_component_rescaling_factor(Component.n)
        D.rec_rescale = adim.get_recombination_rescaling_factor()
        D.nc, D.nv = pb.band_density[Component.n], pb.band_density[Component.p]
        D.ec_eV, D.ev_eV = pb.band_edge_energy[Component.n], pb.band_edge_energy[Component.p]
        dp = ctypes.POINTER(ctypes.c_double)
        keep = []
        rt = pb.recombination_term
        pts = self.cell_qp.reshape(-1, 3)
        if getattr(rt, "kind", "linear") == "srh":
            D.rec_type = 1
            D.srh_ni = rt.intrinsic_carrier_concentration
            D.srh_tau_n = rt.electron_life_time
            D.srh_tau_p = rt.hole_life_time
        else:
            D.rec_type = 0
            for name, fn in (("rec_a_host", rt.constant_term), ("rec_b_host", rt.n_linear_coefficient),
                             ("rec_c_host", rt.p_linear_coefficient)):
                arr = np.ascontiguousarray(fn.value(pts), dtype=np.float64)
                keep.append(arr)
                setattr(D, name, arr.ctypes.data_as(dp))
        dop = np.ascontiguousarray(pb.doping.value(pts) / adim.get_component_rescaling_factor(Component.n))
        keep.append(dop)
        D.doping_host = dop.ctypes.data_as(dp)
        if prm.tau_computer == "fixed":
            for c in range(3):
                D.tau[c] = prm.get_tau(c) / self._tau_rescale(c)
        else:
            tau = np.zeros((self.ncells, self.F, 3))
            for (cell, f), vals in prm.face_tau.items():
                for c in range(3):
                    tau[cell, f, c] = vals[c] / self._tau_rescale(c)
            tau = np.ascontiguousarray(tau)
            keep.append(tau)
            D.tau_host = tau.ctypes.data_as(dp)
        bc, val = self._bc_tables()
        keep += [bc, val]
        D.face_bc_host = bc.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        D.face_bc_val_host = val.ctypes.data_as(dp)
        if self._ctx:
            self.L.ddhdg_ctx_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()
        _lib.check(self.L.ddhdg_ctx_create(ctypes.byref(D), ctypes.byref(self._ctx)), "ctx_create")
        self._desc = D
        self._keep = keep

    def __del__(self):
        try:
            if self._ctx:
                self.L.ddhdg_ctx_destroy(self._ctx)
        except Exception:
            pass

    # ------------------------------------------------------- API mirror
    def sizes(self, thermo=False):
        s = _lib.Sizes()
        _lib.check(self.L.ddhdg_get_sizes(self._ctx, int(thermo), ctypes.byref(s)), "get_sizes")
        return s

    def _sp(self):
        return ctypes.c_void_p(self.stream.cuda_stream)

    def is_enabled(self, c):
        return self.enabled[int(c)]

    def set_enabled_components(self, V, n, p):
        self.enabled = [bool(V), bool(n), bool(p)]
        _lib.check(self.L.ddhdg_set_enabled(self._ctx, int(V), int(n), int(p)), "set_enabled")

    def enable_component(self, c):
        e = list(self.enabled)
        e[int(c)] = True
        self.set_enabled_components(*e)

    def disable_component(self, c):
        e = list(self.enabled)
        e[int(c)] = False
        self.set_enabled_components(*e)

    def replace_boundary_condition(self, boundary_id, bc_type, component, f):
        """src/np_solver.cpp:2160-2233."""
        self.problem.boundary_handler.replace_boundary_condition(boundary_id, bc_type, component, f)
        self.update_boundary_tables()

    def update_boundary_tables(self):
        bc, val = self._bc_tables()
        _lib.check(self.L.ddhdg_set_boundary(self._ctx, bc.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                             val.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                   "set_boundary")

    # state as host arrays [ncells, Nc_all] and [nfaces, 3, nf]
    def get_cell_state(self):
        return self.cell_state.view(self.ncells, self.Nc_all).cpu().numpy()

    def get_trace_state(self):
        return self.trace_state.view(self.nfaces, 3, self.nf).cpu().numpy()

    def set_state(self, cell, trace):
        torch = _torch()
        self.cell_state.copy_(torch.as_tensor(np.ascontiguousarray(cell, dtype=np.float64)).reshape(-1))
        self.trace_state.copy_(torch.as_tensor(np.ascontiguousarray(trace, dtype=np.float64)).reshape(-1))

    # ---------------------------------------------- per-step primitives
    def assemble_condense(self, thermo=False):
        torch = _torch()
        s = self.sizes(thermo)
        nc, Nt = self.ncells, s.Nt
        tt = torch.empty(nc * Nt * Nt, dtype=torch.float64, device=self.device)
        rhs = torch.empty(nc * Nt, dtype=torch.float64, device=self.device)
        dflag = torch.empty(nc * Nt, dtype=torch.int32, device=self.device)
        dval = torch.empty(nc * Nt, dtype=torch.float64, device=self.device)
        _lib.check(self.L.ddhdg_assemble_condense(self._ctx, self.cell_state.data_ptr(),
                                                  self.trace_state.data_ptr(), int(thermo),
                                                  tt.data_ptr(), rhs.data_ptr(), dflag.data_ptr(),
                                                  dval.data_ptr(), self._sp()), "assemble_condense")
        return tt.view(nc, Nt, Nt), rhs.view(nc, Nt), dflag.view(nc, Nt), dval.view(nc, Nt)

    def reconstruct(self, update_trace, thermo=False):
        torch = _torch()
        ut = update_trace if isinstance(update_trace, torch.Tensor) else \
            torch.as_tensor(np.ascontiguousarray(update_trace, dtype=np.float64), device=self.device)
        ut = ut.reshape(-1).contiguous()
        out = torch.empty(self.ncells * self.Nc_all, dtype=torch.float64, device=self.device)
        _lib.check(self.L.ddhdg_reconstruct(self._ctx, self.cell_state.data_ptr(), self.trace_state.data_ptr(),
                                            ut.data_ptr(), out.data_ptr(), int(thermo), self._sp()),
                   "reconstruct")
        return out.view(self.ncells, self.Nc_all)

    def get_local_cell_system(self, cells, thermo=False):
        """get_local_cell_system (src/np_solver.cpp:2337-2445) for a list of
        cells (indices into the lexicographic cell order): the local system
        before the Schur complement, assembled on the device.  Returns a dict
        of arrays with a leading cell axis: cc [Nc][Nc], ct [Nc][Nt],
        tc [Nt][Nc], tt [Nt][Nt], c [Nc], t [Nt] (Nc: enabled cell dofs)."""
        torch = _torch()
        s = self.sizes(thermo)
        ncomp = 1 if thermo else sum(self.enabled)
        Nc, Nt = ncomp * (self.dim + 1) * self.nb, s.Nt
        idx = torch.as_tensor(np.asarray(cells, dtype=np.int64).ravel(), device=self.device)
        n = int(idx.numel())
        shapes = dict(cc=(Nc, Nc), ct=(Nc, Nt), tc=(Nt, Nc), tt=(Nt, Nt), c=(Nc,), t=(Nt,))
        out = {k: torch.empty((n,) + v, dtype=torch.float64, device=self.device) for k, v in shapes.items()}
        _lib.check(self.L.ddhdg_local_cell_system(self._ctx, self.cell_state.data_ptr(),
                                                  self.trace_state.data_ptr(), int(thermo), n,
                                                  idx.data_ptr(), 0,
                                                  *[out[k].data_ptr() for k in ("cc", "ct", "tc", "tt", "c", "t")],
                                                  self._sp()), "local_cell_system")
        return {k: v.cpu().numpy() for k, v in out.items()}

    def assemble_condense_plain(self, thermo=False):
        """The same outputs as assemble_condense from the plain FP64 device
        path: the full local systems and an LU of cc per cell, as the
        reference computes them."""
        torch = _torch()
        s = self.sizes(thermo)
        nc, Nt = self.ncells, s.Nt
        tt = torch.empty(nc * Nt * Nt, dtype=torch.float64, device=self.device)
        rhs = torch.empty(nc * Nt, dtype=torch.float64, device=self.device)
        dflag = torch.empty(nc * Nt, dtype=torch.int32, device=self.device)
        dval = torch.empty(nc * Nt, dtype=torch.float64, device=self.device)
        _lib.check(self.L.ddhdg_assemble_condense_plain(self._ctx, self.cell_state.data_ptr(),
                                                        self.trace_state.data_ptr(), int(thermo),
                                                        tt.data_ptr(), rhs.data_ptr(), dflag.data_ptr(),
                                                        dval.data_ptr(), self._sp()), "assemble_condense_plain")
        return tt.view(nc, Nt, Nt), rhs.view(nc, Nt), dflag.view(nc, Nt), dval.view(nc, Nt)

    def reconstruct_plain(self, update_trace, thermo=False):
        """The cell update from the plain FP64 device path (cell systems
        assembled again with the trace update, then solved)."""
        torch = _torch()
        ut = update_trace if isinstance(update_trace, torch.Tensor) else \
            torch.as_tensor(np.ascontiguousarray(update_trace, dtype=np.float64), device=self.device)
        ut = ut.reshape(-1).contiguous()
        out = torch.empty(self.ncells * self.Nc_all, dtype=torch.float64, device=self.device)
        _lib.check(self.L.ddhdg_reconstruct_plain(self._ctx, self.cell_state.data_ptr(),
                                                  self.trace_state.data_ptr(), ut.data_ptr(),
                                                  out.data_ptr(), int(thermo), self._sp()),
                   "reconstruct_plain")
        return out.view(self.ncells, self.Nc_all)

    # ------------------------------------------- global linear system
    def assemble_system(self, thermo=False):
        """assemble_system(false, thermo_eq) + copy_local_to_global
        (include/assembling_methods.template.h:10-89, src/np_solver.cpp:
        1293-1322) on the device: the Newton system of the trace at the
        current state, kept as a CSR matrix (rows and columns in the
        restricted trace order: face, enabled component, face node).
        Dirichlet-constrained dofs are identity rows whose right-hand side is
        the projected Dirichlet increment."""
        torch = _torch()
        s = self.sizes(thermo)
        tt, rhs, flag, val = self.assemble_condense(thermo)
        vals = torch.zeros(s.nnz, dtype=torch.float64, device=self.device)
        grhs = torch.zeros(s.n_trace_dofs, dtype=torch.float64, device=self.device)
        _lib.check(self.L.ddhdg_scatter(self._ctx, tt.data_ptr(), rhs.data_ptr(), flag.data_ptr(),
                                        val.data_ptr(), vals.data_ptr(), grhs.data_ptr(), int(thermo),
                                        self._sp()), "scatter")
        self._system = dict(thermo=bool(thermo), blocks=(tt, rhs, flag, val), values=vals, rhs=grhs)
        return self._system

    def _need_system(self):
        if getattr(self, "_system", None) is None:
            self.assemble_system()
        return self._system

    def _component_dofs(self, thermo=False):
        """restricted trace dof indices of every enabled component"""
        comps = [0] if thermo else [c for c in range(3) if self.enabled[c]]
        nc = len(comps)
        idx = np.arange(self.nfaces * nc * self.nf).reshape(self.nfaces, nc, self.nf)
        return {Component(c): idx[:, i, :].ravel() for i, c in enumerate(comps)}

    def _csr_structure(self, thermo=False):
        rp, ci = ctypes.c_void_p(), ctypes.c_void_p()
        _lib.check(self.L.ddhdg_get_csr(self._ctx, int(thermo), ctypes.byref(rp), ctypes.byref(ci)), "get_csr")
        s = self.sizes(thermo)
        rowptr = np.empty(s.n_trace_dofs + 1, dtype=np.int32)
        colind = np.empty(s.nnz, dtype=np.int32)
        cudart = ctypes.CDLL("libcudart.so")
        self.stream.synchronize()
        for host, ptr in ((rowptr, rp), (colind, ci)):
            if cudart.cudaMemcpy(host.ctypes.data_as(ctypes.c_void_p), ptr, ctypes.c_size_t(host.nbytes), 2):
                raise RuntimeError("cudaMemcpy of the trace sparsity failed")
        return rowptr, colind

    def get_residual(self):
        """pyddhdg NPSolver::get_residual (src/pyddhdg/pyddhdg.cpp:1601-1666):
        the right-hand side of the assembled system, one array per enabled
        component (dofs in the restricted trace order)."""
        sysm = self._need_system()
        b = sysm["rhs"].cpu().numpy()
        return {c: b[d] for c, d in self._component_dofs(sysm["thermo"]).items()}

    def get_jacobian(self):
        """pyddhdg NPSolver::get_jacobian (src/pyddhdg/pyddhdg.cpp:1852-1935):
        the assembled matrix split into blocks per pair of enabled
        components, as scipy CSR matrices."""
        import scipy.sparse as sp

        sysm = self._need_system()
        rowptr, colind = self._csr_structure(sysm["thermo"])
        n = len(rowptr) - 1
        A = sp.csr_matrix((sysm["values"].cpu().numpy(), colind, rowptr), shape=(n, n))
        dofs = self._component_dofs(sysm["thermo"])
        return {(c1, c2): A[d1][:, d2].tocsr() for c1, d1 in dofs.items() for c2, d2 in dofs.items()}

    def get_linear_system_solution_vector(self):
        """pyddhdg NPSolver::get_linear_system_solution_vector
        (src/pyddhdg/pyddhdg.cpp:1670-1735): the solution of the assembled
        system (nested-dissection solve on the device), per enabled
        component."""
        torch = _torch()
        sysm = self._need_system()
        tt, rhs, flag, val = sysm["blocks"]
        x = torch.empty(sysm["rhs"].numel(), dtype=torch.float64, device=self.device)
        _lib.check(self.L.ddhdg_solve_condensed(self._ctx, tt.data_ptr(), rhs.data_ptr(), flag.data_ptr(),
                                                val.data_ptr(), x.data_ptr(), int(sysm["thermo"]),
                                                self._sp()), "solve_condensed")
        xs = x.cpu().numpy()
        return {c: xs[d] for c, d in self._component_dofs(sysm["thermo"]).items()}

    def set_solver_graphs(self, enable: bool):
        """Capture the trace solve's launch sequence in a CUDA graph on the
        second solve with the same buffers and replay it afterwards (on by
        default); off: every solve launches its kernels directly."""
        _lib.check(self.L.ddhdg_set_solver_graphs(self._ctx, int(bool(enable))), "set_solver_graphs")

    def private_run(self, abs_tol, rel_tol, max_it, thermo=False, alpha=None):
        alpha = self.parameters.nonlinear_parameters.alpha if alpha is None else alpha
        it = ctypes.c_int()
        nrm = ctypes.c_double()
        code = self.L.ddhdg_newton(self._ctx, self.cell_state.data_ptr(), self.trace_state.data_ptr(),
                                   int(thermo), float(abs_tol), float(rel_tol), int(max_it), float(alpha),
                                   ctypes.byref(it), ctypes.byref(nrm), self._sp())
        if code not in (0, 7):
            _lib.check(code, "newton")
        return NonlinearIterationResults(code == 0, it.value, nrm.value)

    def run(self, absolute_tol=None, relative_tol=None, max_number_of_iterations=None):
        """NPSolver::run (src/np_solver.cpp:1565-1597)."""
        nl = self.parameters.nonlinear_parameters
        return self.private_run(nl.absolute_tolerance if absolute_tol is None else absolute_tol,
                                nl.relative_tolerance if relative_tol is None else relative_tol,
                                nl.max_number_of_iterations if max_number_of_iterations is None
                                else max_number_of_iterations)

    def last_timings(self):
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        st = ctypes.c_int()
        self.L.ddhdg_last_timings(self._ctx, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(st))
        return dict(condense_ms=a.value, solve_ms=b.value, reconstruct_ms=c.value, steps=st.value)

    # -------------------------------------------------- projections
    def _lcn_potential(self, doping):
        pb = self.problem
        Nc, Nv = pb.band_density[Component.n], pb.band_density[Component.p]
        Ec, Ev = pb.band_edge_energy[Component.n] * EV, pb.band_edge_energy[Component.p] * EV
        T = self.T
        U_T = T * KB / Q
        twice_ni = 2 * np.sqrt(Nc * Nv * np.exp((Ev - Ec) / (T * KB)))
        return ((Ec + Ev) / (2 * Q) + U_T / 2 * np.log(Nv / Nc) + U_T * np.arcsinh(doping / twice_ni)) / \
            self.adim.get_component_rescaling_factor(Component.V)

    def compute_local_charge_neutrality(self):
        """src/thermodynamic_equilibrium.cpp:9-351: potential of local charge
        neutrality projected on the cells and on every face."""
        torch = _torch()
        pb = self.problem
        vc = self._lcn_potential(pb.doping.value(self.cell_qp.reshape(-1, 3)))
        vf = self._lcn_potential(pb.doping.value(self.cell_fqp.reshape(-1, 3)))
        vt = self._lcn_potential(pb.doping.value(self.face_qp.reshape(-1, 3)))
        dvc = torch.as_tensor(np.ascontiguousarray(vc), device=self.device)
        dvf = torch.as_tensor(np.ascontiguousarray(vf), device=self.device)
        dvt = torch.as_tensor(np.ascontiguousarray(vt), device=self.device)
        _lib.check(self.L.ddhdg_project_cell(self._ctx, dvc.data_ptr(), dvf.data_ptr(), 0,
                                             self.cell_state.data_ptr(), self._sp()), "project_cell")
        _lib.check(self.L.ddhdg_project_trace(self._ctx, dvt.data_ptr(), 0, self.trace_state.data_ptr(),
                                              self._sp()), "project_trace")
        self.stream.synchronize()

    def compute_thermodynamic_equilibrium(self, absolute_tol=None, relative_tol=None,
                                          max_number_of_iterations=None, generate_first_guess=True):
        """src/thermodynamic_equilibrium.cpp:365-405."""
        nl = self.parameters.nonlinear_parameters
        if generate_first_guess:
            self.compute_local_charge_neutrality()
        res = self.private_run(nl.absolute_tolerance if absolute_tol is None else absolute_tol,
                               nl.relative_tolerance if relative_tol is None else relative_tol,
                               nl.max_number_of_iterations if max_number_of_iterations is None
                               else max_number_of_iterations, thermo=True)
        for c in (1, 2):
            _lib.check(self.L.ddhdg_project_density(self._ctx, c, 0.0, self.cell_state.data_ptr(),
                                                    self.trace_state.data_ptr(), self._sp()),
                       "project_density")
        return res

    def set_component(self, c, f, use_projection=False):
        """Solver::set_component: interpolation at the support points (or L2
        projection), scalar, flux = -grad f, and trace values."""
        torch = _torch()
        f = as_function(f)
        c = int(c)
        scale = self.adim.get_component_rescaling_factor(c)
        if use_projection:
            vc = np.ascontiguousarray(f.value(self.cell_qp.reshape(-1, 3)) / scale)
            vf = np.ascontiguousarray(f.value(self.cell_fqp.reshape(-1, 3)) / scale)
            vt = np.ascontiguousarray(f.value(self.face_qp.reshape(-1, 3)) / scale)
            _lib.check(self.L.ddhdg_project_cell(self._ctx, torch.as_tensor(vc, device=self.device).data_ptr(),
                                                 torch.as_tensor(vf, device=self.device).data_ptr(), c,
                                                 self.cell_state.data_ptr(), self._sp()), "project_cell")
            _lib.check(self.L.ddhdg_project_trace(self._ctx, torch.as_tensor(vt, device=self.device).data_ptr(),
                                                  c, self.trace_state.data_ptr(), self._sp()), "project_trace")
            self.stream.synchronize()
            return
        cs = self.get_cell_state()
        ts = self.get_trace_state()
        d = self.dim
        nodes = self.support
        ref = np.zeros((self.nb, 3))
        r = np.arange(self.nb)
        for a in range(d):
            ref[:, a] = nodes[r % (self.k + 1)]
            r = r // (self.k + 1)
        pts = (np.array(self.origin) + (self.cell_idx[:, None, :] + ref[None]) * np.array(self.h)).reshape(-1, 3)
        blk = cs[:, c * (d + 1) * self.nb:(c + 1) * (d + 1) * self.nb].reshape(self.ncells, d + 1, self.nb)
        blk[:, d] = (f.value(pts) / scale).reshape(self.ncells, self.nb)
        g = f.gradient(pts) / scale
        for s in range(d):
            blk[:, s] = -g[:, s].reshape(self.ncells, self.nb)
        cs[:, c * (d + 1) * self.nb:(c + 1) * (d + 1) * self.nb] = blk.reshape(self.ncells, -1)
        # trace support points
        fpts = np.zeros((self.nfaces, self.nf, 3))
        for f_ in range(self.F):
            a, side = f_ // 2, f_ % 2
            fr = np.zeros((self.nf, 3))
            fr[:, a] = side
            mm = np.arange(self.nf)
            for t in range(d - 1):
                fr[:, (a + 1 + t) % d] = nodes[mm % (self.k + 1)]
                mm = mm // (self.k + 1)
            fpts[self.cell_faces[:, f_]] = np.array(self.origin) + \
                (self.cell_idx[:, None, :] + fr[None]) * np.array(self.h)
        ts[:, c, :] = (f.value(fpts.reshape(-1, 3)) / scale).reshape(self.nfaces, self.nf)
        self.set_state(cs, ts)

    def get_solution_on_a_point(self, point, c):
        """NPSolver::get_solution_on_a_point (src/np_solver.cpp:1637-1700):
        V, n, p (physical units) or the quasi Fermi potential phi_n / phi_p
        (volts) at one point, evaluated on the device."""
        return float(self.evaluate(c, np.atleast_2d(point))[0])

    def evaluate(self, c, points):
        """The same at many points [N, dim] (one device launch)."""
        torch = _torch()
        pts = np.atleast_2d(np.asarray(points, dtype=np.float64))
        if pts.shape[1] < 3:
            pts = np.concatenate([pts, np.zeros((pts.shape[0], 3 - pts.shape[1]))], 1)
        c = Component(c)
        what = {Component.V: 0, Component.n: 1, Component.p: 2, Component.phi_n: 3, Component.phi_p: 4}[c]
        dpts = torch.as_tensor(np.ascontiguousarray(pts), device=self.device)
        out = torch.empty(pts.shape[0], dtype=torch.float64, device=self.device)
        _lib.check(self.L.ddhdg_sample_points(self._ctx, self.cell_state.data_ptr(), pts.shape[0],
                                              dpts.data_ptr(), what, out.data_ptr(), self._sp()),
                   "sample_points")
        return out.cpu().numpy()
