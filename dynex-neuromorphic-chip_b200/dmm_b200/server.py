"""Continuous-batching server: formulas arrive, are admitted by device-memory footprint,
integrate together with everything resident, and retire when solved or out of steps."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import ServerConfig, ServerResult, check, lib, ptr
from .cnf import Formula
from .instance import Result


class Server:
    def __init__(self, budget_bytes: int, max_slots: int = 4096, steps_per_launch: int = 32,
                 precision: str = "fp32", device: int = 0):
        cfg = ServerConfig(_lib.PRECISIONS[precision], int(device), int(budget_bytes),
                           int(max_slots), int(steps_per_launch))
        h = ctypes.c_void_p()
        check(lib().dmm_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self.n_of: dict[int, int] = {}

    def close(self):
        if getattr(self, "_h", None):
            lib().dmm_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def clock(self) -> float:
        return lib().dmm_server_clock(self._h)

    def submit(self, f: Formula, x0=None, seed: int = 0, max_steps: int = 0, params=None) -> int:
        x = None if x0 is None else np.ascontiguousarray(x0, dtype=np.float64)
        t = ctypes.c_int64()
        p = None if params is None else ctypes.byref(params)
        check(lib().dmm_server_submit(self._h, ptr(f.lits, ctypes.c_int32),
                                      ptr(f.clause_off, ctypes.c_int64), f.n, f.m, p,
                                      ptr(x, ctypes.c_double), ctypes.c_uint64(seed),
                                      int(max_steps), ctypes.byref(t)))
        self.n_of[t.value] = f.n
        return t.value

    def pump(self):
        """One scheduling round: (resident, queued)."""
        r = ctypes.c_int32()
        q = ctypes.c_int32()
        check(lib().dmm_server_pump(self._h, ctypes.byref(r), ctypes.byref(q)))
        return r.value, q.value

    def take(self, cap: int = 1024):
        """Finished results: list of dicts with ticket, Result, submit/admit/finish times
        and the reported assignment."""
        buf = (ServerResult * cap)()
        cnt = ctypes.c_int32()
        check(lib().dmm_server_take(self._h, buf, int(cap), ctypes.byref(cnt)))
        out = []
        for i in range(cnt.value):
            r = buf[i]
            n = self.n_of.pop(r.ticket)
            post = np.zeros(n, dtype=np.int8)
            check(lib().dmm_server_assignment(self._h, r.ticket, ptr(post, ctypes.c_int8), n))
            out.append({"ticket": r.ticket, "result": Result.from_report(r.report),
                        "submit_s": r.submit_s, "admit_s": r.admit_s, "finish_s": r.finish_s,
                        "assignment": post})
        return out
