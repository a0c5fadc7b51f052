"""One formula on one GPU: the host-side mirror of the reference integrator.

The reference's integrator is the function pair ``dmm_generate_dxdt`` (dynex.cc:332) and
``dmm_dostep`` (dynex.cc:301) driven by the adaptive loop of ``dmm()`` (dynex.cc:1381-1459).
:class:`Instance` offers the same three operations (``generate_dxdt``, ``dostep``,
``solve``) on device-resident state, plus ``step`` for a fixed number of accepted steps.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import Limits, Report, Tuning, check, lib, ptr
from .cnf import Formula


@dataclass
class Result:
    status: int
    status_name: str
    steps: int
    t: float
    loc: int
    best_loc: int
    energy: float
    solved_step: int
    solved_t: float
    wall_s: float

    @property
    def solved(self) -> bool:
        return self.status == _lib.SOLVED

    @classmethod
    def from_report(cls, r: Report) -> "Result":
        return cls(**r.as_dict())


class Instance:
    """A formula resident on a GPU with its integration state.

    precision: "fp32" (production) or "fp64" (the reference's arithmetic, bit-exact).
    """

    def __init__(self, formula: Formula, precision: str = "fp32", device: int = 0):
        self.formula = formula
        self.precision = precision
        self.n, self.m = formula.n, formula.m
        h = ctypes.c_void_p()
        check(lib().dmm_instance_create(ptr(formula.lits, ctypes.c_int32),
                                        ptr(formula.clause_off, ctypes.c_int64), formula.n,
                                        formula.m, _lib.PRECISIONS[precision], int(device),
                                        ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().dmm_instance_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- configuration -------------------------------------------------------------------
    def set_params(self, params=None, alpha_cm=None, **over) -> None:
        """Parameters (defaults of dynex.cc:132-140, overridable by keyword)."""
        p = params if params is not None else _lib.default_params(**over)
        a = None if alpha_cm is None else np.ascontiguousarray(alpha_cm, dtype=np.float64)
        check(lib().dmm_instance_set_params(self._h, ctypes.byref(p), ptr(a, ctypes.c_double)))

    @property
    def tuning(self) -> dict:
        t = Tuning()
        check(lib().dmm_instance_get_tuning(self._h, ctypes.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw) -> None:
        t = Tuning()
        check(lib().dmm_instance_get_tuning(self._h, ctypes.byref(t)))
        for k, v in kw.items():
            setattr(t, k, int(v))
        check(lib().dmm_instance_set_tuning(self._h, ctypes.byref(t)))

    # -- state ---------------------------------------------------------------------------
    def set_state(self, x) -> None:
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.shape != (self.n + 2 * self.m,):
            raise ValueError("state must have n + 2m entries")
        check(lib().dmm_instance_set_state(self._h, ptr(x, ctypes.c_double)))

    def set_state_at(self, x, t: float, step: int) -> None:
        """Sets the state with the integration continuing at time t after `step` steps."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.shape != (self.n + 2 * self.m,):
            raise ValueError("state must have n + 2m entries")
        check(lib().dmm_instance_set_state_at(self._h, ptr(x, ctypes.c_double), float(t),
                                              int(step)))

    def get_state(self):
        x = np.zeros(self.n + 2 * self.m, dtype=np.float64)
        t = ctypes.c_double()
        check(lib().dmm_instance_get_state(self._h, ptr(x, ctypes.c_double), ctypes.byref(t)))
        return x, t.value

    # -- the reference function pair -----------------------------------------------------
    def generate_dxdt(self, x):
        """dmm_generate_dxdt (dynex.cc:332): (dxdt, loc, energy).  Leaves the instance at x."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        d = np.zeros_like(x)
        loc = ctypes.c_int32()
        e = ctypes.c_double()
        check(lib().dmm_instance_rhs(self._h, ptr(x, ctypes.c_double), ptr(d, ctypes.c_double),
                                     ctypes.byref(loc), ctypes.byref(e)))
        return d, loc.value, e.value

    def dostep(self, x, dxdt, h: float):
        """dmm_dostep (dynex.cc:301): x + h*dxdt with unit pin and clamps."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        dxdt = np.ascontiguousarray(dxdt, dtype=np.float64)
        o = np.zeros_like(x)
        check(lib().dmm_instance_dostep(self._h, ptr(x, ctypes.c_double),
                                        ptr(dxdt, ctypes.c_double), float(h),
                                        ptr(o, ctypes.c_double)))
        return o

    # -- integration ---------------------------------------------------------------------
    def step(self, nsteps: int) -> Result:
        r = Report()
        check(lib().dmm_instance_step(self._h, int(nsteps), ctypes.byref(r)))
        return Result.from_report(r)

    def solve(self, max_steps: int = 0, wall_s: float = 0.0) -> Result:
        """dmm() (dynex.cc:1182-1474): integrate until solved or a limit is hit."""
        lim = Limits(int(max_steps), 0, float(wall_s))
        r = Report()
        check(lib().dmm_instance_solve(self._h, ctypes.byref(lim), ctypes.byref(r)))
        return Result.from_report(r)

    def report(self) -> Result:
        r = Report()
        check(lib().dmm_instance_report(self._h, ctypes.byref(r)))
        return Result.from_report(r)

    def assignment(self, pre: bool = True):
        """(pre, post): sign of V when the solution was found (0 for V == 0) and the
        reported assignment after the final step (+1/-1).  pre is None when unsolved."""
        post = np.zeros(self.n, dtype=np.int8)
        if pre:
            p = np.zeros(self.n, dtype=np.int8)
            st = lib().dmm_instance_assignment(self._h, ptr(p, ctypes.c_int8),
                                               ptr(post, ctypes.c_int8))
            if st == 10:  # DMM_ERR_STATE: not solved
                p = None
                check(lib().dmm_instance_assignment(self._h, None, ptr(post, ctypes.c_int8)))
            else:
                check(st)
            return p, post
        check(lib().dmm_instance_assignment(self._h, None, ptr(post, ctypes.c_int8)))
        return None, post

    def profile(self, nsteps: int, flush_bytes: int = 0):
        """Device time (ms) of the clause and variable kernels over nsteps plain-launched
        steps, each after flush_bytes of L2-evicting writes."""
        a = ctypes.c_double()
        b = ctypes.c_double()
        check(lib().dmm_instance_profile(self._h, int(nsteps), int(flush_bytes), ctypes.byref(a),
                                         ctypes.byref(b)))
        return a.value, b.value

    def time_steps(self, nsteps: int) -> float:
        """Device time (ms) of nsteps steps launched as the solver launches them."""
        ms = ctypes.c_double()
        check(lib().dmm_instance_time_steps(self._h, int(nsteps), ctypes.byref(ms)))
        return ms.value

    def time_steps_flushed(self, nsteps: int, flush_bytes: int) -> float:
        """Summed device time (ms) of nsteps steps, each launched alone after an L2 flush."""
        ms = ctypes.c_double()
        check(lib().dmm_instance_time_steps_flushed(self._h, int(nsteps), int(flush_bytes),
                                                    ctypes.byref(ms)))
        return ms.value

    LAUNCH_FORMS = {1: "two-kernel", 2: "cooperative", 3: "cooperative-single",
                    4: "staged", 5: "one-block-per-formula", 6: "staged-multi"}

    @property
    def launch_form(self) -> str:
        """Kernel that step/solve launch with the current tuning (see LAUNCH_FORMS)."""
        f = lib().dmm_instance_launch_form(self._h)
        if f < 0:
            check(f)
        return self.LAUNCH_FORMS[f]

    def trace_phases(self, nsteps: int) -> dict:
        """Per-step microseconds (mean, max over blocks) between the cooperative kernel's
        trace points, averaged over one launch of nsteps steps."""
        out = (ctypes.c_double * 23)()
        check(lib().dmm_instance_trace_phases(self._h, int(nsteps), out))
        keys = ("a_load", "a_gather", "a_eval", "barrier1", "b_load", "b_gather", "b_reduce",
                "barrier2", "decide", "barrier3")
        r = {k: (out[2 * i], out[2 * i + 1]) for i, k in enumerate(keys)}
        r["sm_mhz"] = out[20]
        r["launch_prologue"] = out[21]
        r["launch_epilogue"] = out[22]
        return r
