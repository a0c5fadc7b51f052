"""Formulas on the host: DIMACS I/O, the planted generator, the strict-sign checker and
initial states (all implemented in libdmm.so)."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from ._lib import Cnf, check, lib, ptr


@dataclass
class Formula:
    """A CNF formula: clause i is lits[clause_off[i]:clause_off[i+1]] (DIMACS numbering)."""

    n: int
    m: int
    lits: np.ndarray        # int32
    clause_off: np.ndarray  # int64, m+1
    max_occurrence: int = 0

    @property
    def nlits(self) -> int:
        return int(self.clause_off[-1])

    def state_size(self) -> int:
        return self.n + 2 * self.m


def _from_cnf(c: "ctypes.POINTER(Cnf)") -> Formula:
    cc = c.contents
    lits = np.ctypeslib.as_array(cc.lits, shape=(max(cc.nlits, 1),))[: cc.nlits].copy()
    off = np.ctypeslib.as_array(cc.clause_off, shape=(cc.m + 1,)).copy()
    f = Formula(int(cc.n), int(cc.m), lits.astype(np.int32), off.astype(np.int64),
                int(cc.max_occurrence))
    lib().dmm_cnf_free(c)
    return f


def read_cnf(path: str) -> Formula:
    """DIMACS reader (the reference loader, dynex.cc:2306-2392)."""
    c = ctypes.POINTER(Cnf)()
    check(lib().dmm_cnf_read(path.encode(), ctypes.byref(c)))
    return _from_cnf(c)


def from_arrays(lits, clause_off, n: int) -> Formula:
    lits = np.ascontiguousarray(lits, dtype=np.int32)
    off = np.ascontiguousarray(clause_off, dtype=np.int64)
    m = len(off) - 1
    c = ctypes.POINTER(Cnf)()
    check(lib().dmm_cnf_from_arrays(ptr(lits, ctypes.c_int32), ptr(off, ctypes.c_int64), int(n),
                                    int(m), ctypes.byref(c)))
    return _from_cnf(c)


def write_cnf(f: Formula, path: str, planted=None) -> None:
    c = Cnf(f.n, f.m, f.nlits, ptr(f.lits, ctypes.c_int32), ptr(f.clause_off, ctypes.c_int64),
            f.max_occurrence, 0)
    pl = None if planted is None else np.ascontiguousarray(planted, dtype=np.int8)
    check(lib().dmm_cnf_write(ctypes.byref(c), path.encode(), ptr(pl, ctypes.c_int8)))


def write_state(path: str, x, n: int, m: int, t: float) -> None:
    """State checkpoint in the reference's `<cnf>.assignment.txt` format (dynex.cc:2131-2135):
    the n + 2m values [V | Xs | Xl] as "%.15f, ", then t as "%.15f "."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    if x.shape != (n + 2 * m,):
        raise ValueError("x must have n + 2m entries")
    check(lib().dmm_state_write(path.encode(), ptr(x, ctypes.c_double), int(n), int(m), float(t)))


def read_state(path: str, n: int, m: int, reference_rounding: bool = False):
    """(x, t) from a state checkpoint file (dynex.cc:2521-2532); reference_rounding rounds
    every value to float as the reference's loader does."""
    x = np.zeros(n + 2 * m, dtype=np.float64)
    t = ctypes.c_double()
    check(lib().dmm_state_read(path.encode(), int(n), int(m), int(bool(reference_rounding)),
                               ptr(x, ctypes.c_double), ctypes.byref(t)))
    return x, t.value


def generate_planted(n: int, m: int, p0: float = 0.08, p1: float = 0.46, seed: int = 0):
    """Planted 3-SAT: (Formula, planted +1/-1 assignment).  p0/p1: probability that 3 / 1
    literals of a clause agree with the planted assignment (else 2)."""
    c = ctypes.POINTER(Cnf)()
    planted = np.zeros(n, dtype=np.int8)
    check(lib().dmm_cnf_generate_planted(int(n), int(m), float(p0), float(p1),
                                         ctypes.c_uint64(seed & (2**64 - 1)), ctypes.byref(c),
                                         ptr(planted, ctypes.c_int8)))
    return _from_cnf(c), planted


def check_assignment(f: Formula, assign) -> int:
    """Number of clauses with no literal whose sign matches assign (+1/-1/0)."""
    a = np.ascontiguousarray(assign, dtype=np.int8)
    if a.shape != (f.n,):
        raise ValueError("assignment length must be n")
    r = lib().dmm_check_assignment(ptr(f.lits, ctypes.c_int32), ptr(f.clause_off, ctypes.c_int64),
                                   f.m, f.n, ptr(a, ctypes.c_int8))
    if r < 0:
        raise ValueError("bad formula or assignment")
    return int(r)


def initial_state_reference(f: Formula, seed: int = 0, replica: int = 0):
    """Initial state of the reference CLI for seed/replica (dynex.cc:2635-2700):
    (x, alpha_divisor)."""
    x = np.zeros(f.state_size(), dtype=np.float64)
    div = ctypes.c_int32()
    check(lib().dmm_initial_state_reference(ptr(f.lits, ctypes.c_int32),
                                            ptr(f.clause_off, ctypes.c_int64), f.n, f.m,
                                            int(seed), int(replica), ptr(x, ctypes.c_double),
                                            ctypes.byref(div)))
    return x, int(div.value)


def initial_state_uniform(f: Formula, seed: int):
    """V ~ U[-1,1], Xs ~ U[0,1], Xl = 1 (unit-clause variables pinned)."""
    x = np.zeros(f.state_size(), dtype=np.float64)
    check(lib().dmm_initial_state_uniform(ptr(f.lits, ctypes.c_int32),
                                          ptr(f.clause_off, ctypes.c_int64), f.n, f.m,
                                          ctypes.c_uint64(seed & (2**64 - 1)),
                                          ptr(x, ctypes.c_double)))
    return x
