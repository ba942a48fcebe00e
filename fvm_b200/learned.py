"""Learned error correction for the AMG solve (no reference counterpart).

A message-passing network on the finest level's cell graph (width 32,
three layers) maps the FP64 residual to a correction of the solution. It is
trained on the GPU, by the library's own forward/backward kernels and Adam,
on (residual, error) pairs harvested from the plain solver's own runs, and
used by ThermalModelA.advance() as a flexible step after every AMG
refinement iteration that is kept only when it lowers the FP64 L1 residual
norm (the plain AMG step stands otherwise).

    lc = LearnedCorrection(seed=0)
    lc.harvest(plain_model, nOuter=20, perSolve=4)   # plain solves of training instances
    losses = lc.train(steps=2000, lr=1e-3)
    model.setLearnedCorrection(lc)                   # used by the next advance()
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import c_double_p, c_float_p, c_int_p, check


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class LearnedCorrection:
    def __init__(self, seed: int = 0):
        lib = _lib.load()
        h = lib.fvm_learned_create(int(seed))
        if not h:
            raise _lib.FvmError(5, lib.fvm_last_error().decode())
        self._h = ctypes.c_void_p(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().fvm_learned_destroy(h)
            except Exception:
                pass
            self._h = None

    def handle(self):
        return self._h

    @staticmethod
    def numParams() -> int:
        return int(_lib.load().fvm_learned_num_params())

    def getParams(self) -> np.ndarray:
        p = np.zeros(self.numParams(), np.float32)
        check(_lib.load().fvm_learned_get_params(self._h, p.ctypes.data_as(c_float_p), len(p)))
        return p

    def setParams(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(_lib.load().fvm_learned_set_params(self._h, p.ctypes.data_as(c_float_p), len(p)))

    def save(self, path: str) -> None:
        np.savez(path, params=self.getParams())

    def load(self, path: str) -> None:
        self.setParams(np.load(path)["params"])

    @property
    def tensorCores(self) -> bool:
        """Dense layers on the tensor cores (tcgen05, TF32 operands, FP32
        sums; the default) or in FP32 on the CUDA cores."""
        v = ctypes.c_int(0)
        check(_lib.load().fvm_learned_tensor_cores(self._h, ctypes.byref(v)))
        return bool(v.value)

    @tensorCores.setter
    def tensorCores(self, on: bool) -> None:
        check(_lib.load().fvm_learned_set_tensor_cores(self._h, 1 if on else 0))

    ERROR, RESIDUAL = 0, 1

    def setObjective(self, objective: int) -> None:
        """Training objective: ERROR (relative squared error of the
        predicted error, the default) or RESIDUAL (|r + A d|^2 / |r|^2, the
        residual the correction leaves)."""
        check(_lib.load().fvm_learned_set_objective(self._h, int(objective)))

    def setUsefulFactor(self, f: float) -> None:
        """The solve retires the step after three tries if fewer than a
        quarter cut the residual below f times its value (default 0.5)."""
        check(_lib.load().fvm_learned_set_useful_factor(self._h, float(f)))

    def residualFactor(self) -> float:
        """sqrt(mean |r + A d|^2 / |r|^2) on the pairs at the last
        evaluate() with the RESIDUAL objective (-1 if none since training);
        a solve skips the network when it is above the useful factor."""
        v = ctypes.c_double(0)
        check(_lib.load().fvm_learned_residual_factor(self._h, ctypes.byref(v)))
        return v.value

    def harvest(self, model, nOuter: int = 20, perSolve: int = 4, relativeTolerance: float = 1e-10,
                maxCycles: int = 200) -> int:
        """Outer iterations of `model` (a ThermalModelA with a plain AMG
        linear solver, after init() and its fields), each linear system
        solved to relativeTolerance; returns the pairs added."""
        model._push()
        n = ctypes.c_int(0)
        check(_lib.load().fvm_learned_harvest(self._h, model._h, int(nOuter), int(perSolve),
                                              float(relativeTolerance), int(maxCycles), ctypes.byref(n)))
        return n.value

    def numPairs(self) -> int:
        return int(_lib.load().fvm_learned_num_pairs(self._h))

    def train(self, steps: int, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        losses = np.zeros(max(int(steps), 1))
        check(_lib.load().fvm_learned_train(self._h, int(steps), float(lr), int(seed), losses.ctypes.data_as(c_double_p)))
        return losses[: int(steps)]

    def evaluate(self) -> float:
        v = ctypes.c_double(0)
        check(_lib.load().fvm_learned_evaluate(self._h, ctypes.byref(v)))
        return v.value

    # --- kernels on a plain CSR graph (checks against a CPU restatement) ---------
    def forward_csr(self, row, col, diag, off, r) -> np.ndarray:
        row, col, diag, off, r = _i32(row), _i32(col), _f64(diag), _f64(off), _f64(r)
        out = np.zeros(len(diag))
        check(_lib.load().fvm_learned_forward_csr(self._h, len(diag), row.ctypes.data_as(c_int_p),
                                                  col.ctypes.data_as(c_int_p), diag.ctypes.data_as(c_double_p),
                                                  off.ctypes.data_as(c_double_p), r.ctypes.data_as(c_double_p),
                                                  out.ctypes.data_as(c_double_p)))
        return out

    def gradient_csr(self, row, col, diag, off, r, e):
        row, col, diag, off, r, e = _i32(row), _i32(col), _f64(diag), _f64(off), _f64(r), _f64(e)
        g = np.zeros(self.numParams(), np.float32)
        loss = ctypes.c_double(0)
        check(_lib.load().fvm_learned_gradient_csr(self._h, len(diag), row.ctypes.data_as(c_int_p),
                                                   col.ctypes.data_as(c_int_p), diag.ctypes.data_as(c_double_p),
                                                   off.ctypes.data_as(c_double_p), r.ctypes.data_as(c_double_p),
                                                   e.ctypes.data_as(c_double_p), g.ctypes.data_as(c_float_p),
                                                   ctypes.byref(loss)))
        return g, loss.value
