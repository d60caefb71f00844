"""Batched condensation: many devices (diodes) of different mesh sizes and
polynomial degrees condensed in ONE persistent launch per Newton step, and
reconstructed in one more (``ddhdg_batch_*`` of the C ABI).

The reference condenses one device at a time, its per-cell worker run over
that device's cells by WorkStream (include/assembling_methods.template.h:
67-88).  ``CondenseBatch`` hands a work list of tiles (device, range of its
cells) to the CTAs of one grid; the tile sizes per degree and the CTAs per SM
come from ``autotune()``, which times the batch's own launch.  Every device's
outputs are bitwise those of its own ``NPSolver.assemble_condense`` /
``reconstruct``.
"""

from __future__ import annotations

import ctypes

from . import _lib


class CondenseBatch:
    """One launch per Newton step over the contexts of `solvers`
    (``NPSolver`` objects of one dimension, FP64 or mixed precision, each
    condensed in its own precision).  The outputs of solver i
    are ``tt[i]``, ``rhs[i]``, ``dflag[i]``, ``dval[i]`` (shaped like
    ``NPSolver.assemble_condense``); the reconstruction reads
    ``update_trace[i]`` ([nfaces * 3 * nf]) and writes ``update_cell[i]``.
    The solvers' state tensors must stay in place (the launches are replayed
    from CUDA graphs)."""

    def __init__(self, solvers, thermo=False, buffers=None):
        self.solvers = list(solvers)
        self.thermo = bool(thermo)
        self.L = _lib.load()
        if buffers is None:
            buffers = [self.buffers_for(g, thermo) for g in self.solvers]
        self.buffers = buffers
        self.tt = [b["tt"] for b in buffers]
        self.rhs = [b["rhs"] for b in buffers]
        self.dflag = [b["dflag"] for b in buffers]
        self.dval = [b["dval"] for b in buffers]
        self.update_trace = [b["update_trace"] for b in buffers]
        self.update_cell = [b["update_cell"] for b in buffers]
        items = (_lib.BatchItem * len(self.solvers))()
        for i, g in enumerate(self.solvers):
            it = items[i]
            it.ctx = g._ctx
            it.cell_state = g.cell_state.data_ptr()
            it.trace_state = g.trace_state.data_ptr()
            it.tt = self.tt[i].data_ptr()
            it.rhs = self.rhs[i].data_ptr()
            it.dflag = self.dflag[i].data_ptr()
            it.dval = self.dval[i].data_ptr()
            it.update_trace = self.update_trace[i].data_ptr()
            it.update_cell = self.update_cell[i].data_ptr()
        self._items = items
        self._b = ctypes.c_void_p()
        _lib.check(self.L.ddhdg_batch_create(items, len(self.solvers), int(self.thermo), ctypes.byref(self._b)),
                   "batch_create")
        self.stream = self.solvers[0].stream
        self.cells = sum(g.ncells for g in self.solvers)

    @staticmethod
    def buffers_for(g, thermo=False):
        """Output and update buffers of one solver in a batch (kept by a
        caller that rebuilds batches over the same solvers, so that the
        solvers' trace-solve graphs stay valid)."""
        import torch

        s = g.sizes(thermo)
        nc, Nt, dev = g.ncells, s.Nt, g.device
        return {"tt": torch.empty((nc, Nt, Nt), dtype=torch.float64, device=dev),
                "rhs": torch.empty((nc, Nt), dtype=torch.float64, device=dev),
                "dflag": torch.empty((nc, Nt), dtype=torch.int32, device=dev),
                "dval": torch.empty((nc, Nt), dtype=torch.float64, device=dev),
                "update_trace": torch.zeros(g.nfaces * 3 * g.nf, dtype=torch.float64, device=dev),
                "update_cell": torch.empty((nc, g.Nc_all), dtype=torch.float64, device=dev)}

    def _sp(self):
        return ctypes.c_void_p(self.stream.cuda_stream)

    def newton_step(self, alphas):
        """One Newton step of every solver (batched condensation, the trace
        solves overlapped on side streams, batched reconstruction, damped
        update in place).  Returns (norms [n][4]: max |update_cell|,
        max |update_trace|, max |cell_state|, max |trace_state| before the
        update, statuses [n])."""
        import numpy as np

        n = len(self.solvers)
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(alphas, dtype=np.float64), (n,)))
        norms = np.zeros((n, 4))
        status = (ctypes.c_int * n)()
        dp = ctypes.POINTER(ctypes.c_double)
        code = self.L.ddhdg_batch_newton_step(self._b, a.ctypes.data_as(dp), norms.ctypes.data_as(dp), status,
                                              self._sp())
        if code not in (0, 3, 8):
            _lib.check(code, "batch_newton_step")
        return norms, list(status)

    def newton_step_begin(self, alphas):
        """Enqueue one Newton step of every solver (as ``newton_step``) and
        return at once."""
        import numpy as np

        n = len(self.solvers)
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(alphas, dtype=np.float64), (n,)))
        dp = ctypes.POINTER(ctypes.c_double)
        _lib.check(self.L.ddhdg_batch_newton_step_begin(self._b, a.ctypes.data_as(dp), self._sp()),
                   "batch_newton_step_begin")

    def newton_step_end(self, wait=True):
        """The result of the step in flight: (norms, statuses) as
        ``newton_step`` returns them, or None while it is still running
        (wait=False)."""
        import numpy as np

        n = len(self.solvers)
        norms = np.zeros((n, 4))
        status = (ctypes.c_int * n)()
        done = ctypes.c_int()
        dp = ctypes.POINTER(ctypes.c_double)
        code = self.L.ddhdg_batch_newton_step_end(self._b, int(bool(wait)), norms.ctypes.data_as(dp), status,
                                                  ctypes.byref(done))
        if code not in (0, 3, 8):
            _lib.check(code, "batch_newton_step_end")
        if not done.value:
            return None
        return norms, list(status)

    def condense(self):
        _lib.check(self.L.ddhdg_batch_condense(self._b, self._sp()), "batch_condense")

    def reconstruct(self):
        _lib.check(self.L.ddhdg_batch_reconstruct(self._b, self._sp()), "batch_reconstruct")

    def autotune(self, reps=3):
        """Pick the cells per tile of every degree and the CTAs per SM by
        timing this batch's condensation launch; returns the best time (ms)."""
        ms = ctypes.c_float()
        _lib.check(self.L.ddhdg_batch_autotune(self._b, int(reps), ctypes.byref(ms), self._sp()),
                   "batch_autotune")
        return float(ms.value)

    def shape(self):
        cpt = (ctypes.c_int * 3)()
        cps, grid, nt = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.check(self.L.ddhdg_batch_get_shape(self._b, cpt, ctypes.byref(cps), ctypes.byref(grid),
                                                ctypes.byref(nt)), "batch_get_shape")
        return {"cells_per_tile": {1: cpt[0], 2: cpt[1], 3: cpt[2]}, "ctas_per_sm": cps.value,
                "grid": grid.value, "tiles": nt.value}

    def set_shape(self, cells_per_tile, ctas_per_sm):
        """cells_per_tile: {degree: cells} for degrees 1..3."""
        cpt = (ctypes.c_int * 3)(*[int(cells_per_tile[k]) for k in (1, 2, 3)])
        _lib.check(self.L.ddhdg_batch_set_shape(self._b, cpt, int(ctas_per_sm)), "batch_set_shape")

    def close(self):
        if self._b:
            self.L.ddhdg_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
