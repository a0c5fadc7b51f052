"""Many formulas integrated together in one pack (persistent tile kernels, CUDA graphs)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import BatchStats, Report, Tuning, check, lib, ptr
from .cnf import Formula
from .instance import Result


class Batch:
    """Capacities bound the device arrays, which are allocated once."""

    def __init__(self, max_instances: int, max_vars: int, max_clauses: int, max_lits: int,
                 precision: str = "fp32", device: int = 0):
        h = ctypes.c_void_p()
        check(lib().dmm_batch_create(_lib.PRECISIONS[precision], int(device), int(max_instances),
                                     int(max_vars), int(max_clauses), int(max_lits),
                                     ctypes.byref(h)))
        self._h = h
        self.formulas: list[Formula] = []

    @classmethod
    def for_formulas(cls, formulas, precision="fp32", device=0):
        return cls(len(formulas), sum(f.n for f in formulas), sum(f.m for f in formulas),
                   sum(f.nlits for f in formulas), precision, device)

    def close(self):
        if getattr(self, "_h", None):
            lib().dmm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_tuning(self, **kw):
        t = Tuning(**{k: int(v) for k, v in kw.items()})
        check(lib().dmm_batch_set_tuning(self._h, ctypes.byref(t)))

    def add(self, f: Formula, x0, params=None, max_steps: int = 0) -> int:
        x0 = np.ascontiguousarray(x0, dtype=np.float64)
        if x0.shape != (f.state_size(),):
            raise ValueError("x0 must have n + 2m entries")
        idx = ctypes.c_int32()
        p = None if params is None else ctypes.byref(params)
        check(lib().dmm_batch_add(self._h, ptr(f.lits, ctypes.c_int32),
                                  ptr(f.clause_off, ctypes.c_int64), f.n, f.m, p,
                                  ptr(x0, ctypes.c_double), int(max_steps), ctypes.byref(idx)))
        self.formulas.append(f)
        return idx.value

    def run(self, wall_s: float = 0.0) -> dict:
        s = BatchStats()
        check(lib().dmm_batch_run(self._h, float(wall_s), ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in s._fields_}

    def result(self, index: int):
        r = Report()
        post = np.zeros(self.formulas[index].n, dtype=np.int8)
        check(lib().dmm_batch_result(self._h, int(index), ctypes.byref(r),
                                     ptr(post, ctypes.c_int8)))
        return Result.from_report(r), post

    def set_state_at(self, index: int, x, t: float, step: int = 0) -> None:
        """Restarts formula `index` from state x at time t after `step` steps (a resume
        from a checkpoint, dynex.cc:2521-2532)."""
        f = self.formulas[index]
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.shape != (f.state_size(),):
            raise ValueError("x must have n + 2m entries")
        check(lib().dmm_batch_set_state_at(self._h, int(index), ptr(x, ctypes.c_double),
                                           float(t), int(step)))

    def state(self, index: int):
        f = self.formulas[index]
        x = np.zeros(f.state_size(), dtype=np.float64)
        t = ctypes.c_double()
        check(lib().dmm_batch_state(self._h, int(index), ptr(x, ctypes.c_double), ctypes.byref(t)))
        return x, t.value
