"""Scalar functions of position used for doping, temperature, boundary data and
exact solutions.

They play the part of the deal.II ``Function`` objects that the reference
passes around (``dealii::FunctionParser`` strings, ``ConstantFunction``,
``Ddhdg::PiecewiseFunction`` in src/function_tools.cpp:409-479,
``FunctionTimesScalar``).  Every function is evaluated on the host, vectorised
over an ``(N, 3)`` array of points, and the results are handed to the device
as tables at quadrature points.
"""

from __future__ import annotations

import math
from typing import Callable, Union

import numpy as np

# Physical constants of include/constants.h:12-15
PI = math.pi
E = math.e
EPSILON0 = 8.85418781762e-12
Q = 1.602176634e-19
KB = 1.380649e-23
EV = 1.602176565e-19

_PARSER_CONSTANTS = {
    "pi": PI,
    "e": E,
    "eps0": EPSILON0,
    "epsilon0": EPSILON0,
    "q": Q,
    "kb": KB,
    "eV": EV,
}

_PARSER_FUNCS = {
    "exp": np.exp,
    "log": np.log,
    "ln": np.log,
    "sqrt": np.sqrt,
    "sin": np.sin,
    "cos": np.cos,
    "tan": np.tan,
    "tanh": np.tanh,
    "sinh": np.sinh,
    "cosh": np.cosh,
    "asinh": np.arcsinh,
    "atan": np.arctan,
    "abs": np.abs,
    "pow": np.power,
}


class Function:
    """Base class: ``value(points)`` with ``points`` of shape ``(N, 3)``."""

    def value(self, points: np.ndarray) -> np.ndarray:  # pragma: no cover
        raise NotImplementedError

    def gradient(self, points: np.ndarray) -> np.ndarray:
        """Central finite differences (the AutoDerivativeFunction scheme that
        deal.II's FunctionParser uses), step 1e-8 scaled by |x|."""
        pts = np.asarray(points, dtype=np.float64)
        g = np.zeros_like(pts)
        for a in range(3):
            h = 1e-8 * np.maximum(1.0, np.abs(pts[:, a]))
            pp = pts.copy()
            pm = pts.copy()
            pp[:, a] += h
            pm[:, a] -= h
            g[:, a] = (self.value(pp) - self.value(pm)) / (2 * h)
        return g

    def __call__(self, points):
        return self.value(points)


class ConstantFunction(Function):
    def __init__(self, c: float):
        self.c = float(c)

    def value(self, points):
        return np.full(np.asarray(points).shape[0], self.c, dtype=np.float64)

    def gradient(self, points):
        return np.zeros((np.asarray(points).shape[0], 3), dtype=np.float64)


class AnalyticFunction(Function):
    """A FunctionParser-like expression in ``x, y, z`` (``^`` is a power) or
    a Python callable ``f(x, y, z)`` working on numpy arrays."""

    def __init__(self, expr: Union[str, Callable], gradient: Callable = None):
        self.expr = expr
        self._grad = gradient
        if isinstance(expr, str):
            self._code = compile(expr.replace("^", "**"), "<ddhdg-function>", "eval")
        else:
            self._code = None

    def value(self, points):
        pts = np.asarray(points, dtype=np.float64)
        x, y, z = pts[:, 0], pts[:, 1], pts[:, 2]
        if self._code is not None:
            ns = dict(_PARSER_FUNCS)
            ns.update(_PARSER_CONSTANTS)
            ns.update({"x": x, "y": y, "z": z})
            v = eval(self._code, {"__builtins__": {}}, ns)
        else:
            v = self.expr(x, y, z)
        v = np.asarray(v, dtype=np.float64)
        if v.ndim == 0:
            v = np.full(pts.shape[0], float(v))
        return v

    def gradient(self, points):
        if self._grad is not None:
            pts = np.asarray(points, dtype=np.float64)
            g = np.asarray(self._grad(pts[:, 0], pts[:, 1], pts[:, 2]), dtype=np.float64)
            return np.moveaxis(np.broadcast_to(g, (3, pts.shape[0])), 0, 1).copy()
        return super().gradient(points)


class PiecewiseFunction(Function):
    """``f1`` where ``condition > 0`` and ``f2`` elsewhere: the ``value_list``
    semantics of Ddhdg::PiecewiseFunction (src/function_tools.cpp:459-479),
    which is what the assembly evaluates through."""

    def __init__(self, condition, f1, f2):
        self.condition = as_function(condition)
        self.f1 = as_function(f1)
        self.f2 = as_function(f2)

    def value(self, points):
        c = self.condition.value(points)
        return np.where(c > 0, self.f1.value(points), self.f2.value(points))


class FunctionTimesScalar(Function):
    def __init__(self, f, s: float):
        self.f = as_function(f)
        self.s = float(s)

    def value(self, points):
        return self.f.value(points) * self.s

    def gradient(self, points):
        return self.f.gradient(points) * self.s


class StepDoping(Function):
    """Two-sided step along axis ``axis``: ``+N_D`` for ``x < x_j`` and
    ``-N_A`` for ``x >= x_j`` (the p-n junction profile of the diode
    workloads)."""

    def __init__(self, x_j: float, N_D: float, N_A: float, axis: int = 0):
        self.x_j = float(x_j)
        self.N_D = float(N_D)
        self.N_A = float(N_A)
        self.axis = int(axis)

    def value(self, points):
        x = np.asarray(points, dtype=np.float64)[:, self.axis]
        return np.where(x < self.x_j, self.N_D, -self.N_A)


def as_function(f) -> Function:
    if isinstance(f, Function):
        return f
    if isinstance(f, (int, float, np.floating, np.integer)):
        return ConstantFunction(float(f))
    if isinstance(f, str) or callable(f):
        return AnalyticFunction(f)
    raise TypeError(f"cannot build a Function from {type(f)!r}")
