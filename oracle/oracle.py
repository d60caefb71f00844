"""ORACLE -- test infrastructure only.

CPU FP64 restatement of the reference's Newton solver around the per-cell HDG
kernel (the per-cell kernel itself is ``hdg_oracle.cpp``).  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py`` use it,
and only as the checker / the reported CPU baseline.

What it restates (reference file:line):
  * Newton loop ``private_run``                 src/np_solver.cpp:1452-1561
  * global assembly ``copy_local_to_global``     src/np_solver.cpp:1293-1322
    (Dirichlet rows constrained, values filled after the solve,
     src/np_solver.cpp:1502-1513)
  * global solve (UMFPACK there, SuperLU here)  src/np_solver.cpp:1326-1354
  * local charge neutrality first guess          src/thermodynamic_equilibrium.cpp:9-351
  * thermodynamic equilibrium driver             src/thermodynamic_equilibrium.cpp:365-405
  * phi -> n, p projection                       src/project_component.cpp:268-420,575-654
  * l2_average trace projection                  src/copy_on_trace.cpp:631-1010
  * interpolation of a component                 src/np_solver.cpp:876-980
  * rescaling factors                            include/adimensionalizer.h:28-262
  * tau rescaling                                src/np_solver_parameters.cpp:13-28
  * Einstein relation / quasi Fermi potential    include/solver.h:343-412
The global UMFPACK factorisation is replaced by SuperLU (scipy 1.18); both
are direct LU solvers, so the results agree to round-off.
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

KB = 1.380649e-23
Q = 1.602176634e-19
EV = 1.602176565e-19

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build():
    """Compile the C++ oracle (make) if needed."""
    src = os.path.join(_HERE, "hdg_oracle.cpp")
    if (not os.path.exists(_LIB_PATH)) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.POINTER(OrProblem)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.oracle_sizes.argtypes = [P, ip]
        L.oracle_tables.argtypes = [P] + [dp] * 8
        L.oracle_local_cell_system.argtypes = [P, dp, dp, ctypes.c_long, ctypes.c_int] + [dp] * 6
        L.oracle_assemble_condense.argtypes = [P, dp, dp, ctypes.c_int, dp, dp, ip, dp, ctypes.c_int]
        L.oracle_local_cell_systems.argtypes = [P, dp, dp, dp, ctypes.c_int] + [dp] * 6 + [ctypes.c_int]
        L.oracle_reconstruct.argtypes = [P, dp, dp, dp, ctypes.c_int, dp, ctypes.c_int]
        L.oracle_srh.argtypes = [ctypes.c_double] * 6 + [dp] * 3
        L.oracle_srh_intrinsic.argtypes = [ctypes.c_double] * 5
        L.oracle_srh_intrinsic.restype = ctypes.c_double
        _lib = L
    return _lib


class OrProblem(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int), ("k", ctypes.c_int),
        ("n", ctypes.c_int * 3),
        ("origin", ctypes.c_double * 3), ("h", ctypes.c_double * 3),
        ("enabled", ctypes.c_int * 3),
        ("flux", ctypes.c_int), ("phi_linearize", ctypes.c_int), ("rec_type", ctypes.c_int),
        ("eps", ctypes.c_double), ("mu_n", ctypes.c_double), ("mu_p", ctypes.c_double),
        ("temperature", ctypes.c_double), ("thermal_voltage_rescale", ctypes.c_double),
        ("V_rescale", ctypes.c_double), ("n_rescale", ctypes.c_double), ("rec_rescale", ctypes.c_double),
        ("nc", ctypes.c_double), ("nv", ctypes.c_double), ("ec_eV", ctypes.c_double), ("ev_eV", ctypes.c_double),
        ("srh_ni", ctypes.c_double), ("srh_tau_n", ctypes.c_double), ("srh_tau_p", ctypes.c_double),
        ("rec_a", ctypes.POINTER(ctypes.c_double)), ("rec_b", ctypes.POINTER(ctypes.c_double)),
        ("rec_c", ctypes.POINTER(ctypes.c_double)),
        ("doping", ctypes.POINTER(ctypes.c_double)), ("tau", ctypes.POINTER(ctypes.c_double)),
        ("face_bc", ctypes.POINTER(ctypes.c_int)), ("face_bc_val", ctypes.POINTER(ctypes.c_double)),
        ("jacobian_fix", ctypes.c_int),
    ]


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


# --------------------------------------------------------------- 1D bases
def lobatto_points(k):
    if k == 0:
        return np.array([0.5])
    from numpy.polynomial import legendre as L

    c = np.zeros(k + 1)
    c[-1] = 1.0
    inner = L.legroots(L.legder(c)) if k > 1 else np.array([])
    return np.sort(np.concatenate([[0.0], 0.5 * (1 + inner), [1.0]]))


def lagrange_eval(nodes, x):
    """values [len(x), len(nodes)] and derivatives of the Lagrange basis."""
    x = np.asarray(x, dtype=np.float64)
    m = len(nodes)
    V = np.ones((x.size, m))
    D = np.zeros((x.size, m))
    for a in range(m):
        for b in range(m):
            if b != a:
                V[:, a] *= (x - nodes[b]) / (nodes[a] - nodes[b])
        for mm in range(m):
            if mm == a:
                continue
            r = np.full(x.size, 1.0 / (nodes[a] - nodes[mm]))
            for b in range(m):
                if b != a and b != mm:
                    r *= (x - nodes[b]) / (nodes[a] - nodes[b])
            D[:, a] += r
    return V, D


# ----------------------------------------------------------- the solver
@dataclass
class NewtonResult:
    converged: bool
    iterations: int
    last_update_norm: float


class OracleSolver:
    """Restatement of ``Ddhdg::NPSolver`` on a structured mesh (CPU, FP64)."""

    def __init__(self, problem, parameters, adimensionalizer, nthreads=0):
        self.problem = problem
        self.parameters = parameters
        self.adim = adimensionalizer
        self.nthreads = int(nthreads)
        mesh = problem.mesh
        self.dim = mesh.dim
        self.k = parameters.k
        self.enabled = [True, True, True]
        self._geometry()
        self.cell_state = np.zeros((self.ncells, self.Nc_all))
        self.trace_state = np.zeros((self.nfaces, 3, self.nf))
        self.newton_history = []

    # ------------------------------------------------------------ geometry
    def _geometry(self):
        mesh = self.problem.mesh
        d, k = self.dim, self.k
        self.n = list(mesh.n) + [1] * (3 - d)
        self.h = list(mesh.h) + [1.0] * (3 - d)
        self.origin = list(mesh.lower) + [0.0] * (3 - d)
        self.nb = (k + 1) ** d
        self.nf = (k + 1) ** (d - 1)
        self.nqc, self.nqf = self.nb, self.nf
        self.Nc_all = 3 * (d + 1) * self.nb
        self.ncells = int(np.prod(self.n))
        self.F = 2 * d
        # faces: for each axis a, lexicographic with extent n_a + 1 along a
        self.axis_offset = [0]
        self.axis_extent = []
        for a in range(d):
            ext = [self.n[b] + (1 if b == a else 0) for b in range(d)]
            self.axis_extent.append(ext)
            self.axis_offset.append(self.axis_offset[-1] + int(np.prod(ext)))
        self.nfaces = self.axis_offset[-1]
        c = np.arange(self.ncells)
        ci = np.stack([c % self.n[0], (c // self.n[0]) % self.n[1], c // (self.n[0] * self.n[1])], 1)
        self.cell_idx = ci
        cf = np.zeros((self.ncells, self.F), dtype=np.int64)
        for f in range(self.F):
            a, side = f // 2, f % 2
            fi = ci.copy()
            fi[:, a] += side
            ext = self.axis_extent[a]
            idx = np.zeros(self.ncells, dtype=np.int64)
            stride = 1
            for b in range(d):
                idx += fi[:, b] * stride
                stride *= ext[b]
            cf[:, f] = self.axis_offset[a] + idx
        self.cell_faces = cf
        # face -> (cell, local face) of the first / second neighbour
        owner = -np.ones((self.nfaces, 2), dtype=np.int64)
        owner_f = -np.ones((self.nfaces, 2), dtype=np.int64)
        for f in range(self.F):
            slot = f % 2  # lower-face side (f even) is the cell "after" the face
            owner[cf[:, f], 1 - slot] = c
            owner_f[cf[:, f], 1 - slot] = f
        self.face_cells = owner
        self.face_local = owner_f
        # boundary id per face (-1 interior)
        bid = -np.ones(self.nfaces, dtype=np.int64)
        for f in range(self.F):
            a, side = f // 2, f % 2
            on_b = ci[:, a] == (self.n[a] - 1 if side else 0)
            faces = cf[on_b, f]
            bid[faces] = (2 * a + side) if mesh.colorize else 0
        self.face_bid = bid

        # tables from the C++ geometry (reference coordinates, weights, bases)
        P = self._struct(probe=True)
        L = lib()
        nqc, nqf, nb, nf = self.nqc, self.nqf, self.nb, self.nf
        self.t_cqref = np.zeros((nqc, 3))
        self.t_cJxW = np.zeros(nqc)
        self.t_fqref = np.zeros((self.F, nqf, 3))
        self.t_fJxW = np.zeros((self.F, nqf))
        self.t_cphi = np.zeros((nqc, nb))
        self.t_fxi = np.zeros((nqf, nf))
        self.t_fphi = np.zeros((self.F, nqf, nb))
        self.t_cgrad = np.zeros((nqc, nb, 3))
        L.oracle_tables(ctypes.byref(P), _dp(self.t_cqref), _dp(self.t_cJxW), _dp(self.t_fqref),
                        _dp(self.t_fJxW), _dp(self.t_cphi), _dp(self.t_fxi), _dp(self.t_fphi),
                        _dp(self.t_cgrad))
        org = np.array(self.origin)
        hh = np.array(self.h)
        self.cell_qp = org + (ci[:, None, :] + self.t_cqref[None, :, :]) * hh  # [ncells, nqc, 3]
        self.cell_fqp = org + (ci[:, None, None, :] + self.t_fqref[None]) * hh  # [ncells, F, nqf, 3]
        # face quadrature points by global face (from the cell after the face
        # or the one before at the upper boundary)
        self.face_qp = np.zeros((self.nfaces, nqf, 3))
        for s in (0, 1):
            cells = self.face_cells[:, s]
            ok = cells >= 0
            self.face_qp[ok] = self.cell_fqp[cells[ok], self.face_local[ok, s]]
        self.normals = np.zeros((self.F, 3))
        for f in range(self.F):
            self.normals[f, f // 2] = 1.0 if f % 2 else -1.0

    # --------------------------------------------------------- rescaling
    def _rescale(self):
        a = self.adim
        T_mag, N, L_, M = a.temperature_magnitude, a.doping_magnitude, a.scale_length, a.mobility_magnitude
        r = {}
        r["V"] = T_mag * KB / Q
        r["n"] = N
        r["thermal"] = T_mag * KB / Q
        r["eps"] = L_ * L_ * Q * Q * N / (T_mag * KB)
        r["mu"] = M
        r["rec"] = KB * N * T_mag * M / (L_ * L_ * Q)
        Tv = T_mag * KB / Q
        r["tau"] = [Q * N / Tv, Tv * M / (L_ * L_), Tv * M / (L_ * L_)]
        r["neumann"] = [Q, KB * N * T_mag * M / (L_ * L_), KB * N * T_mag * M / (L_ * L_)]
        return r

    def _struct(self, probe=False, thermo=False):
        pb, prm = self.problem, self.parameters
        P = OrProblem()
        P.dim, P.k = self.dim, self.k
        for a in range(3):
            P.n[a] = self.n[a]
            P.origin[a] = self.origin[a]
            P.h[a] = self.h[a]
        en = [True, False, False] if thermo else self.enabled
        for c in range(3):
            P.enabled[c] = int(en[c])
        P.flux = int(prm.dd_flux_type)
        P.phi_linearize = int(prm.phi_linearize)
        P.jacobian_fix = (1 if getattr(prm, "consistent_drift_jacobian", False) else 0) | \
            (2 if getattr(prm, "consistent_recombination_jacobian", False) else 0)
        if probe:
            return P
        r = self._rescale()
        T = pb.temperature.value(np.zeros((1, 3)))[0]
        self.T = T
        P.rec_type = 1 if getattr(pb.recombination_term, "kind", "linear") == "srh" else 0
        P.eps = pb.permittivity.epsilon / r["eps"]
        P.mu_n = pb.electron_mobility.mu / r["mu"]
        P.mu_p = pb.hole_mobility.mu / r["mu"]
        P.temperature = T
        P.thermal_voltage_rescale = r["thermal"]
        P.V_rescale = r["V"]
        P.n_rescale = r["n"]
        P.rec_rescale = r["rec"]
        P.nc = pb.band_density[1]
        P.nv = pb.band_density[2]
        P.ec_eV = pb.band_edge_energy[1]
        P.ev_eV = pb.band_edge_energy[2]
        keep = []
        if P.rec_type == 1:
            rt = pb.recombination_term
            P.srh_ni = rt.intrinsic_carrier_concentration
            P.srh_tau_n = rt.electron_life_time
            P.srh_tau_p = rt.hole_life_time
        else:
            rt = pb.recombination_term
            pts = self.cell_qp.reshape(-1, 3)
            for name, fn in (("rec_a", rt.constant_term), ("rec_b", rt.n_linear_coefficient),
                             ("rec_c", rt.p_linear_coefficient)):
                arr = np.ascontiguousarray(fn.value(pts), dtype=np.float64)
                keep.append(arr)
                setattr(P, name, _dp(arr))
        dop = np.ascontiguousarray(pb.doping.value(self.cell_qp.reshape(-1, 3)) / r["n"])
        keep.append(dop)
        P.doping = _dp(dop)
        tau = np.zeros((self.ncells, self.F, 3))
        if prm.tau_computer == "fixed":
            for c in range(3):
                tau[:, :, c] = prm.tau[c] / r["tau"][c]
        else:
            for (cell, f), vals in prm.face_tau.items():
                for c in range(3):
                    tau[cell, f, c] = vals[c] / r["tau"][c]
        tau = np.ascontiguousarray(tau)
        keep.append(tau)
        P.tau = _dp(tau)
        bc, bcv = self._bc_tables(r)
        keep += [bc, bcv]
        P.face_bc = _ip(bc)
        P.face_bc_val = _dp(bcv)
        self._keep = keep
        return P

    def _bc_tables(self, r):
        bh = self.problem.boundary_handler
        bc = np.zeros((self.nfaces, 3), dtype=np.int32)
        val = np.zeros((self.nfaces, 3, self.nqf))
        bfaces = np.nonzero(self.face_bid >= 0)[0]
        for c in range(3):
            for bid in np.unique(self.face_bid[bfaces]):
                faces = bfaces[self.face_bid[bfaces] == bid]
                if bh.has_dirichlet_boundary_conditions(int(bid), c):
                    fn = bh.dirichlet[int(bid)][c]
                    bc[faces, c] = 1
                    val[faces, c] = fn.value(self.face_qp[faces].reshape(-1, 3)).reshape(-1, self.nqf) / \
                        (r["V"] if c == 0 else r["n"])
                elif bh.has_neumann_boundary_conditions(int(bid), c):
                    fn = bh.neumann[int(bid)][c]
                    bc[faces, c] = 2
                    val[faces, c] = fn.value(self.face_qp[faces].reshape(-1, 3)).reshape(-1, self.nqf) / \
                        r["neumann"][c]
        return np.ascontiguousarray(bc), np.ascontiguousarray(val)

    # --------------------------------------------------------- components
    def set_enabled_components(self, V, n, p):
        self.enabled = [bool(V), bool(n), bool(p)]

    def enabled_list(self, thermo=False):
        en = [True, False, False] if thermo else self.enabled
        return [c for c in range(3) if en[c]]

    def cell_block(self, c):
        """view [ncells, d+1, nb] of component c (displacement comps then scalar)."""
        d, nb = self.dim, self.nb
        return self.cell_state[:, c * (d + 1) * nb:(c + 1) * (d + 1) * nb].reshape(self.ncells, d + 1, nb)

    # ------------------------------------------------- per-cell primitives
    def local_cell_system(self, cell, thermo=False):
        P = self._struct(thermo=thermo)
        sizes = np.zeros(9, dtype=np.int32)
        lib().oracle_sizes(ctypes.byref(P), _ip(sizes))
        Nc, Nt = int(sizes[1]), int(sizes[2])
        cc = np.zeros((Nc, Nc))
        ct = np.zeros((Nc, Nt))
        tc = np.zeros((Nt, Nc))
        tt = np.zeros((Nt, Nt))
        crhs = np.zeros(Nc)
        trhs = np.zeros(Nt)
        cs = np.ascontiguousarray(self.cell_state)
        ts = np.ascontiguousarray(self.trace_state)
        lib().oracle_local_cell_system(ctypes.byref(P), _dp(cs), _dp(ts), int(cell), int(thermo),
                                       _dp(cc), _dp(ct), _dp(tc), _dp(tt), _dp(crhs), _dp(trhs))
        return dict(cc=cc, ct=ct, tc=tc, tt=tt, c=crhs, t=trhs)

    def local_cell_systems(self, thermo=False, update_trace=None, cells=None):
        """Local systems (cc, ct, tc, tt, cc_rhs, tt_rhs) of every cell (or of
        the listed `cells`, in that order), as assembled term by term before
        the Schur complement."""
        P = self._struct(thermo=thermo)
        sizes = np.zeros(9, dtype=np.int32)
        lib().oracle_sizes(ctypes.byref(P), _ip(sizes))
        Nc, Nt, n = int(sizes[1]), int(sizes[2]), self.ncells
        if cells is not None:
            assert update_trace is None
            cells = np.asarray(cells, dtype=np.int64)
            out = [np.zeros((len(cells),) + s) for s in ((Nc, Nc), (Nc, Nt), (Nt, Nc), (Nt, Nt), (Nc,), (Nt,))]
            cs = np.ascontiguousarray(self.cell_state)
            ts = np.ascontiguousarray(self.trace_state)
            for i, cell in enumerate(cells):
                bufs = [np.zeros(a.shape[1:]) for a in out]
                lib().oracle_local_cell_system(ctypes.byref(P), _dp(cs), _dp(ts), int(cell), int(thermo),
                                               *[_dp(b) for b in bufs])
                for a, b in zip(out, bufs):
                    a[i] = b
            return tuple(out)
        cc = np.zeros((n, Nc, Nc))
        ct = np.zeros((n, Nc, Nt))
        tc = np.zeros((n, Nt, Nc))
        tt = np.zeros((n, Nt, Nt))
        cr = np.zeros((n, Nc))
        tr = np.zeros((n, Nt))
        cs = np.ascontiguousarray(self.cell_state)
        ts = np.ascontiguousarray(self.trace_state)
        ut = None if update_trace is None else np.ascontiguousarray(update_trace, dtype=np.float64)
        lib().oracle_local_cell_systems(ctypes.byref(P), _dp(cs), _dp(ts),
                                        None if ut is None else _dp(ut), int(thermo), _dp(cc), _dp(ct),
                                        _dp(tc), _dp(tt), _dp(cr), _dp(tr), self.nthreads)
        return cc, ct, tc, tt, cr, tr

    @staticmethod
    def _refined_solve(A, B, sweeps=3):
        """Row-equilibrated LU solve of the batched systems A X = B, followed
        by iterative refinement with residuals in long double: the result is
        the FP64 rounding of the exact solution even where the cell system is
        ill-conditioned (3D Dirichlet cells), so it serves as the parity
        target of any FP64 implementation."""
        d = 1.0 / np.abs(A).max(2, keepdims=True)
        Ad, Bd = A * d, B * d
        X = np.linalg.solve(Ad, Bd)
        Al, Bl, Xl = Ad.astype(np.longdouble), Bd.astype(np.longdouble), X.astype(np.longdouble)
        for _ in range(sweeps):
            R = (Bl - Al @ Xl).astype(np.float64)
            Xl = Xl + np.linalg.solve(Ad, R)
        return Xl

    def reconstruct_accurate(self, update_trace, thermo=False):
        """Reconstruction-pass local systems solved accurately (row-
        equilibrated LU refined with long-double residuals)."""
        cc, _, _, _, cr, _ = self.local_cell_systems(thermo, update_trace)
        cr0 = self.local_cell_systems(thermo)[4]
        x = self._refined_solve(cc, cr[:, :, None])[:, :, 0].astype(np.float64)
        # magnitude of the summed terms through the local solve: |cc^-1| times
        # (|residual part| + |trace-update part|) of the right-hand side
        mag = (np.abs(np.linalg.inv(cc)) @ (np.abs(cr0) + np.abs(cr - cr0))[:, :, None])[:, :, 0]
        out = np.zeros((self.ncells, self.Nc_all))
        sc = np.zeros((self.ncells, self.Nc_all))
        en = [True, False, False] if thermo else self.enabled
        idx = [i for i in range(self.Nc_all) if en[i // ((self.dim + 1) * self.nb)]]
        out[:, idx] = x
        sc[:, idx] = mag
        # [3 components][flux, scalar] magnitude of the summed terms
        d, nb = self.dim, self.nb
        blk = sc.reshape(self.ncells, 3, d + 1, nb)
        self.reconstruct_block_scale = np.stack([np.abs(blk[:, :, :d]).max((0, 2, 3)),
                                                 np.abs(blk[:, :, d]).max((0, 2))], 1)
        return out

    def condense_accurate(self, thermo=False, cells=None):
        """Schur complement tt + tc cc^-1 [ct | cc_rhs] of the term-by-term
        local systems, with cc^-1 applied by a row-equilibrated LU refined in
        long double (so the result does not carry the round-off of any one
        inversion) and the products summed in long double.  Used to separate
        round-off of the reference's inversion from assembly, and as the
        parity target.  `cells` restricts it to a subset (in that order).

        Sets ``condense_term_scale`` (global magnitudes of the summed terms of
        tt and rhs), ``condense_block_scale`` = (tt [ncomp][ncomp],
        rhs [ncomp]): the magnitude of the summed terms (tt or tt_rhs and the
        Schur product) inside each (row component, column component) block of
        the restricted trace order [face][component][node], and
        ``condense_solve_scale``, the same with the terms summed inside the
        local solve counted too (|tt| + |tc| |cc^-1| |ct|, |tr| + |tc| |cc^-1|
        |cc_rhs|)."""
        cc, ct, tc, tt, cr, tr = self.local_cell_systems(thermo, cells=cells)
        rhs = np.concatenate([cr[:, :, None], ct], 2)
        Xl = self._refined_solve(cc, rhs)
        tcXl = tc.astype(np.longdouble) @ Xl
        tcX = tcXl.astype(np.float64)
        S = (tt + tcXl[:, :, 1:]).astype(np.float64)
        g = (tr + tcXl[:, :, 0]).astype(np.float64)
        # magnitude of the summed terms (round-off scale of S and g)
        self.condense_term_scale = (max(np.abs(tt).max(), np.abs(tcX[:, :, 1:]).max()),
                                    max(np.abs(tr).max(), np.abs(tcX[:, :, 0]).max()))
        ncomp = len(self.enabled_list(thermo))
        comp = (np.arange(tt.shape[1]) // self.nf) % ncomp
        # magnitudes through the local solve as well: |tt| + |tc| |cc^-1| |ct|
        # and |tr| + |tc| |cc^-1| |cc_rhs| (the componentwise bound of any
        # backward-stable solve; in 3D Dirichlet cells cc^-1 cc_rhs is a
        # cancellation of terms 1e6 times larger than the result)
        aTC = np.abs(tc) @ np.abs(np.linalg.inv(cc))
        s3t = np.abs(tt) + aTC @ np.abs(ct)
        s3r = np.abs(tr) + (aTC @ np.abs(cr)[:, :, None])[:, :, 0]
        bt = np.zeros((ncomp, ncomp))
        br = np.zeros(ncomp)
        st = np.zeros((ncomp, ncomp))
        sr = np.zeros(ncomp)
        for a in range(ncomp):
            ra = comp == a
            br[a] = max(np.abs(tr[:, ra]).max(), np.abs(tcX[:, ra, 0]).max())
            sr[a] = s3r[:, ra].max()
            for b in range(ncomp):
                cb = np.flatnonzero(comp == b) + 1
                bt[a, b] = max(np.abs(tt[:, ra][:, :, cb - 1]).max(), np.abs(tcX[:, ra][:, :, cb]).max())
                st[a, b] = s3t[:, ra][:, :, cb - 1].max()
        self.condense_block_scale = (bt, br)
        self.condense_solve_scale = (st, sr)
        return S, g

    def assemble_condense(self, thermo=False):
        P = self._struct(thermo=thermo)
        ncomp = len(self.enabled_list(thermo))
        Nt = self.F * ncomp * self.nf
        tt = np.zeros((self.ncells, Nt, Nt))
        rhs = np.zeros((self.ncells, Nt))
        flag = np.zeros((self.ncells, Nt), dtype=np.int32)
        val = np.zeros((self.ncells, Nt))
        cs = np.ascontiguousarray(self.cell_state)
        ts = np.ascontiguousarray(self.trace_state)
        lib().oracle_assemble_condense(ctypes.byref(P), _dp(cs), _dp(ts), int(thermo), _dp(tt), _dp(rhs),
                                       _ip(flag), _dp(val), self.nthreads)
        return tt, rhs, flag, val

    def reconstruct(self, update_trace, thermo=False):
        P = self._struct(thermo=thermo)
        out = np.zeros((self.ncells, self.Nc_all))
        cs = np.ascontiguousarray(self.cell_state)
        ts = np.ascontiguousarray(self.trace_state)
        ut = np.ascontiguousarray(update_trace)
        lib().oracle_reconstruct(ctypes.byref(P), _dp(cs), _dp(ts), _dp(ut), int(thermo), _dp(out), self.nthreads)
        return out

    # ---------------------------------------------------------- global
    def local_to_global(self, ncomp):
        """[ncells, Nt] global restricted trace dof of each cell-local dof."""
        nf = self.nf
        lt = np.arange(self.F * ncomp * nf)
        f = lt // (ncomp * nf)
        ce = (lt // nf) % ncomp
        m = lt % nf
        return (self.cell_faces[:, f] * ncomp + ce[None, :]) * nf + m[None, :]

    def global_system(self, tt, rhs, flag, val, ncomp):
        g = self.local_to_global(ncomp)
        N = self.nfaces * ncomp * self.nf
        Nt = g.shape[1]
        rows = np.repeat(g, Nt, axis=1).ravel()
        cols = np.tile(g, (1, Nt)).ravel()
        A = sp.coo_matrix((tt.ravel(), (rows, cols)), shape=(N, N)).tocsr()
        b = np.zeros(N)
        np.add.at(b, g.ravel(), rhs.ravel())
        dmask = flag.ravel() != 0
        ddofs = g.ravel()[dmask]
        dvals = val.ravel()[dmask]
        # constrained rows/columns carry no couplings (condensed); a unit
        # diagonal with zero rhs is what the constraint leaves behind
        diag = np.zeros(N)
        diag[ddofs] = 1.0
        A = A + sp.diags(diag)
        b[ddofs] = 0.0
        return A.tocsc(), b, ddofs, dvals

    # ----------------------------------------------------------- Newton
    def private_run(self, abs_tol, rel_tol, max_it, thermo=False, record=False):
        comps = self.enabled_list(thermo)
        ncomp = len(comps)
        alpha = self.parameters.nonlinear_parameters.alpha
        converged = False
        step = 0
        update_cell_norm = 0.0
        self.newton_history = []
        while max_it < 0 or step < max_it:
            step += 1
            tt, rhs, flag, val = self.assemble_condense(thermo)
            A, b, ddofs, dvals = self.global_system(tt, rhs, flag, val, ncomp)
            x = spla.splu(A).solve(b)
            x[ddofs] = dvals
            upd_trace = np.zeros((self.nfaces, 3, self.nf))
            xx = x.reshape(self.nfaces, ncomp, self.nf)
            for i, c in enumerate(comps):
                upd_trace[:, c, :] = xx[:, i, :]
            upd_cell = self.reconstruct(upd_trace, thermo)
            update_cell_norm = np.abs(upd_cell).max()
            update_trace_norm = np.abs(upd_trace).max()
            cur_norm = max(np.abs(self.cell_state).max(), np.abs(self.trace_state).max())
            update_norm = max(update_cell_norm, update_trace_norm)
            self.trace_state += alpha * upd_trace
            self.cell_state += alpha * upd_cell
            if record:
                self.newton_history.append((self.cell_state.copy(), self.trace_state.copy()))
            if update_norm < abs_tol or update_norm < rel_tol * cur_norm:
                converged = True
                break
        return NewtonResult(converged, step, float(update_cell_norm))

    def run(self, abs_tol=None, rel_tol=None, max_it=None, record=False):
        nl = self.parameters.nonlinear_parameters
        return self.private_run(nl.absolute_tolerance if abs_tol is None else abs_tol,
                                nl.relative_tolerance if rel_tol is None else rel_tol,
                                nl.max_number_of_iterations if max_it is None else max_it,
                                thermo=False, record=record)

    # ----------------------------------------------------- projections
    def _mass(self):
        M = np.einsum("q,qa,qb->ab", self.t_cJxW, self.t_cphi, self.t_cphi)
        Mf = np.einsum("q,qa,qb->ab", self.t_fJxW[0] if self.dim > 1 else np.ones(1), self.t_fxi, self.t_fxi)
        return M, Mf

    def _project_cell(self, vals_cell, vals_face):
        """L2 projection of a scalar given at cell qps [ncells,nqc] and cell-face
        qps [ncells,F,nqf]: scalar coefficients and the weak gradient
        displacement (src/project_component.cpp:268-420)."""
        M, _ = self._mass()
        d = self.dim
        rc = np.einsum("cq,q,qa->ca", vals_cell, self.t_cJxW, self.t_cphi)
        coef = np.linalg.solve(M, rc.T).T
        disp = np.zeros((self.ncells, d, self.nb))
        for s in range(d):
            rd = np.einsum("cq,q,qa->ca", vals_cell, self.t_cJxW, self.t_cgrad[:, :, s])
            for f in range(self.F):
                ns = self.normals[f, s]
                if ns == 0.0:
                    continue
                rd -= np.einsum("cq,q,qa->ca", vals_face[:, f], self.t_fJxW[f], self.t_fphi[f]) * ns
            disp[:, s] = np.linalg.solve(M, rd.T).T
        return coef, disp

    def _cell_values_at(self, c, where="cell"):
        blk = self.cell_block(c)
        if where == "cell":
            return np.einsum("ca,qa->cq", blk[:, self.dim], self.t_cphi)
        return np.einsum("ca,fqa->cfq", blk[:, self.dim], self.t_fphi)

    def _lcn_potential(self, doping, T):
        pb = self.problem
        r = self._rescale()
        Nc, Nv = pb.band_density[1], pb.band_density[2]
        Ec, Ev = pb.band_edge_energy[1] * EV, pb.band_edge_energy[2] * EV
        U_T = T * KB / Q
        ni2 = Nc * Nv * np.exp((Ev - Ec) / (T * KB))
        twice_ni = 2 * np.sqrt(ni2)
        return ((Ec + Ev) / (2 * Q) + U_T / 2 * np.log(Nv / Nc) + U_T * np.arcsinh(doping / twice_ni)) / r["V"]

    def compute_local_charge_neutrality(self):
        """src/thermodynamic_equilibrium.cpp:9-351 (cells, then every face)."""
        pb = self.problem
        T = pb.temperature.value(np.zeros((1, 3)))[0]
        vc = self._lcn_potential(pb.doping.value(self.cell_qp.reshape(-1, 3)).reshape(self.ncells, -1), T)
        vf = self._lcn_potential(pb.doping.value(self.cell_fqp.reshape(-1, 3)).reshape(self.ncells, self.F, -1), T)
        coef, disp = self._project_cell(vc, vf)
        blk = self.cell_block(0)
        blk[:, self.dim] = coef
        blk[:, :self.dim] = disp
        # trace: L2 projection of the potential on every face
        _, Mf = self._mass()
        vtf = self._lcn_potential(pb.doping.value(self.face_qp.reshape(-1, 3)).reshape(self.nfaces, -1), T)
        w = self.t_fJxW[0] if self.dim > 1 else np.ones(1)
        rhs = np.einsum("Fq,q,qm->Fm", vtf, w, self.t_fxi)
        self.trace_state[:, 0, :] = np.linalg.solve(Mf, rhs.T).T

    def _l2_average_trace(self, c):
        """src/copy_on_trace.cpp:631-1010 with TraceProjectionStrategy::l2_average."""
        _, Mf = self._mass()
        vals = self._cell_values_at(c, "face")  # [ncells, F, nqf]
        acc = np.zeros((self.nfaces, self.nqf))
        cnt = np.zeros(self.nfaces)
        for f in range(self.F):
            np.add.at(acc, self.cell_faces[:, f], vals[:, f])
            np.add.at(cnt, self.cell_faces[:, f], 1.0)
        avg = acc / cnt[:, None]
        w = self.t_fJxW[0] if self.dim > 1 else np.ones(1)
        rhs = np.einsum("Fq,q,qm->Fm", avg, w, self.t_fxi)
        self.trace_state[:, c, :] = np.linalg.solve(Mf, rhs.T).T

    def density_from_qf(self, c, qf, V, T):
        """compute_density (include/solver.h:378-412)."""
        pb = self.problem
        KbT = KB * T
        if c == 1:
            return pb.band_density[1] * np.exp((Q * (V - qf) - pb.band_edge_energy[1] * EV) / KbT)
        return pb.band_density[2] * np.exp((Q * (qf - V) + pb.band_edge_energy[2] * EV) / KbT)

    def project_quasi_fermi(self, c, qf_value=0.0):
        """project_component(phi_n / phi_p, qf) (src/project_component.cpp:268-420)."""
        r = self._rescale()
        T = self.problem.temperature.value(np.zeros((1, 3)))[0]
        Vc = self._cell_values_at(0, "cell") * r["V"]
        Vf = self._cell_values_at(0, "face") * r["V"]
        nc = self.density_from_qf(c, qf_value, Vc, T) / r["n"]
        nf = self.density_from_qf(c, qf_value, Vf, T) / r["n"]
        coef, disp = self._project_cell(nc, nf)
        blk = self.cell_block(c)
        blk[:, self.dim] = coef
        blk[:, :self.dim] = disp
        self._l2_average_trace(c)

    def compute_thermodynamic_equilibrium(self, abs_tol=None, rel_tol=None, max_it=None,
                                          generate_first_guess=True):
        nl = self.parameters.nonlinear_parameters
        saved = list(self.enabled)
        if generate_first_guess:
            self.compute_local_charge_neutrality()
        res = self.private_run(nl.absolute_tolerance if abs_tol is None else abs_tol,
                               nl.relative_tolerance if rel_tol is None else rel_tol,
                               nl.max_number_of_iterations if max_it is None else max_it,
                               thermo=True)
        self.project_quasi_fermi(1)
        self.project_quasi_fermi(2)
        self.enabled = saved
        return res

    def set_component(self, c, f, use_projection=False):
        """Solver::set_component (src/solver.cpp:26-35): projection or
        interpolation (src/np_solver.cpp:876-980)."""
        from ddhdg_b200.functions import as_function

        f = as_function(f)
        r = self._rescale()
        scale = r["V"] if c == 0 else r["n"]
        if use_projection:
            vc = f.value(self.cell_qp.reshape(-1, 3)).reshape(self.ncells, -1) / scale
            vf = f.value(self.cell_fqp.reshape(-1, 3)).reshape(self.ncells, self.F, -1) / scale
            coef, disp = self._project_cell(vc, vf)
            blk = self.cell_block(c)
            blk[:, self.dim] = coef
            blk[:, :self.dim] = disp
            self._l2_average_trace(c)
            return
        pts = self.cell_support_points().reshape(-1, 3)
        blk = self.cell_block(c)
        blk[:, self.dim] = (f.value(pts) / scale).reshape(self.ncells, self.nb)
        g = f.gradient(pts) / scale
        for s in range(self.dim):
            blk[:, s] = -g[:, s].reshape(self.ncells, self.nb)
        fp = self.face_support_points().reshape(-1, 3)
        self.trace_state[:, c, :] = (f.value(fp) / scale).reshape(self.nfaces, self.nf)

    def cell_support_points(self):
        nodes = lobatto_points(self.k)
        d = self.dim
        idx = np.arange(self.nb)
        ref = np.zeros((self.nb, 3))
        r = idx.copy()
        for a in range(d):
            ref[:, a] = nodes[r % (self.k + 1)]
            r //= (self.k + 1)
        return np.array(self.origin) + (self.cell_idx[:, None, :] + ref[None]) * np.array(self.h)

    def face_support_points(self):
        nodes = lobatto_points(self.k)
        d = self.dim
        pts = np.zeros((self.nfaces, self.nf, 3))
        for s in (0, 1):
            cells = self.face_cells[:, s]
            ok = cells >= 0
            lf = self.face_local[ok, s]
            a = lf // 2
            ref = np.zeros((ok.sum(), self.nf, 3))
            ref[np.arange(ok.sum()), :, a] = (lf % 2)[:, None]
            for m in range(self.nf):
                r = m
                for t in range(d - 1):
                    ax = (a + 1 + t) % d
                    ref[np.arange(ok.sum()), m, ax] = nodes[r % (self.k + 1)]
                    r //= (self.k + 1)
            pts[ok] = np.array(self.origin) + (self.cell_idx[cells[ok]][:, None, :] + ref) * np.array(self.h)
        return pts

    # ------------------------------------------------------- evaluation
    def evaluate(self, c, points):
        """Scalar component c (physical units) at points [N,3] (get_solution_on_a_point)."""
        pts = np.atleast_2d(np.asarray(points, dtype=np.float64))
        if pts.shape[1] < 3:
            pts = np.concatenate([pts, np.zeros((pts.shape[0], 3 - pts.shape[1]))], 1)
        r = self._rescale()
        scale = r["V"] if c == 0 else r["n"]
        return self._eval_blk(c, self.dim, pts) * scale

    def _eval_blk(self, c, sub, pts):
        nodes = lobatto_points(self.k)
        d = self.dim
        rel = (pts[:, :d] - np.array(self.origin[:d])) / np.array(self.h[:d])
        ci = np.clip(np.floor(rel).astype(np.int64), 0, np.array(self.n[:d]) - 1)
        xi = rel - ci
        cell = ci[:, 0]
        if d > 1:
            cell = cell + self.n[0] * ci[:, 1]
        if d > 2:
            cell = cell + self.n[0] * self.n[1] * ci[:, 2]
        phi = np.ones((pts.shape[0], self.nb))
        for a in range(d):
            V, _ = lagrange_eval(nodes, xi[:, a])
            idx = (np.arange(self.nb) // (self.k + 1) ** a) % (self.k + 1)
            phi *= V[:, idx]
        blk = self.cell_block(c)[cell, sub]
        return np.einsum("na,na->n", phi, blk)

    def l2_error(self, c, exact, extra_points=2):
        """Cell-wise Gauss integration of (u_h - u)^2 in physical units of c."""
        from ddhdg_b200.functions import as_function

        exact = as_function(exact)
        m = self.k + 1 + extra_points
        g, w = np.polynomial.legendre.leggauss(m)
        g = 0.5 * (g + 1)
        w = 0.5 * w
        d = self.dim
        grids = np.meshgrid(*([g] * d), indexing="ij")
        ref = np.zeros((m ** d, 3))
        for a in range(d):
            ref[:, a] = grids[a].transpose(*reversed(range(d))).ravel() if d > 1 else grids[a].ravel()
        wg = np.ones(m ** d)
        wgrids = np.meshgrid(*([w] * d), indexing="ij")
        for a in range(d):
            wg = wg * (wgrids[a].transpose(*reversed(range(d))).ravel() if d > 1 else wgrids[a].ravel())
        vol = np.prod(self.h[:d])
        pts = np.array(self.origin) + (self.cell_idx[:, None, :] + ref[None]) * np.array(self.h)
        uh = self.evaluate(c, pts.reshape(-1, 3)).reshape(self.ncells, -1)
        ue = exact.value(pts.reshape(-1, 3)).reshape(self.ncells, -1)
        return math.sqrt(float(np.einsum("cq,q->", (uh - ue) ** 2, wg) * vol))


def srh(ni, tau_n, tau_p, n, p, rescaling=1.0):
    r = ctypes.c_double()
    dn = ctypes.c_double()
    dp = ctypes.c_double()
    lib().oracle_srh(ni, tau_n, tau_p, n, p, rescaling, ctypes.byref(r), ctypes.byref(dn), ctypes.byref(dp))
    return r.value, dn.value, dp.value


def srh_intrinsic(Nc, Nv, Ec, Ev, T):
    return lib().oracle_srh_intrinsic(Nc, Nv, Ec, Ev, T)
