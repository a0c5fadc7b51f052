"""ctypes access to the parity oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/, tests/golden/make_golden.py,
__graft_entry__.smoke() and bench.py's CPU-baseline leg; never by the product.

* :class:`Oracle` wraps ``_build/liboracle.so`` (``dmm_oracle.cc``), the project's CPU
  restatement of the reference integrator (FP64 reference mode and FP32 production mode).
* :class:`Reference` wraps ``_ref/libdynex_ref.so`` (``ref_harness.cc``), the unmodified
  reference ``dynex.cc`` driven per step.  The reference keeps its formula in process
  globals, so only one :class:`Reference` can be live per process.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libdynex_ref.so")
REF_CLI = os.path.join(HERE, "_ref", "dynex_ref")
REF_GPU_SO = os.path.join(HERE, "_ref", "libdynex_gpu_ref.so")

DEFAULT_PARAMS = (2.5, 20.0, 0.25, 0.05, 0.1, 0.1)  # dynex.cc:132-138
DEFAULT_XL_MAX = 10000  # dynex.cc:140


class RunResult(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_int),
        ("solved", ctypes.c_int),
        ("solve_step", ctypes.c_int),
        ("pad", ctypes.c_int),
        ("t", ctypes.c_double),
        ("solve_t", ctypes.c_double),
    ]


# Where the reference sources are read from when the harness is built (DYNEX_REFERENCE_DIR
# overrides); a machine without them uses the prebuilt _ref/ files as they are.
REF_DIR = os.environ.get("DYNEX_REFERENCE_DIR", "/root/reference")


def build(quiet: bool = True) -> None:
    """Builds the oracle (and the reference harness where the reference sources exist)."""
    out = subprocess.run(["make", "-C", HERE, "all", f"REF_DIR={REF_DIR}"], capture_output=True,
                         text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def _ptr(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t)) if a is not None else None


_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_I32 = ctypes.POINTER(ctypes.c_int32)
_I64 = ctypes.POINTER(ctypes.c_int64)
_S8 = ctypes.POINTER(ctypes.c_byte)

_oracle_lib = None


def _load_oracle():
    global _oracle_lib
    if _oracle_lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        lib = ctypes.CDLL(ORACLE_SO)
        lib.oracle_create.restype = ctypes.c_void_p
        lib.oracle_create.argtypes = [ctypes.c_int, ctypes.c_int, _I32, _I64, _D, ctypes.c_int, _D,
                                      ctypes.c_int]
        lib.oracle_destroy.argtypes = [ctypes.c_void_p]
        lib.oracle_xl_max.restype = ctypes.c_double
        lib.oracle_xl_max.argtypes = [ctypes.c_void_p]
        lib.oracle_rhs.argtypes = [ctypes.c_void_p, _D, _D, _I, _D]
        lib.oracle_dostep.argtypes = [ctypes.c_void_p, _D, _D, ctypes.c_double, _D]
        lib.oracle_run.argtypes = [ctypes.c_void_p, _D, ctypes.c_int, _D, ctypes.c_int, _I, _D,
                                   _S8, _S8, ctypes.POINTER(RunResult)]
        lib.oracle_check.argtypes = [ctypes.c_void_p, _S8]
        lib.oracle_init_state.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _D]
        _oracle_lib = lib
    return _oracle_lib


def _as_formula(lits, coff):
    lits = np.ascontiguousarray(lits, dtype=np.int32)
    coff = np.ascontiguousarray(coff, dtype=np.int64)
    return lits, coff


class _Common:
    n: int
    m: int

    def _run_common(self, fn, x0, max_steps, dump_every):
        N = self.n + 2 * self.m
        x0 = np.ascontiguousarray(x0, dtype=np.float64)
        assert x0.shape == (N,)
        dump = None
        if dump_every:
            dump = np.zeros((max_steps // dump_every + 1, N), dtype=np.float64)
        loc = np.full(max_steps + 1, -1, dtype=np.int32)
        energy = np.full(max_steps + 1, np.nan, dtype=np.float64)
        pre = np.zeros(self.n, dtype=np.int8)
        post = np.zeros(self.n, dtype=np.int8)
        res = RunResult()
        rc = fn(_ptr(x0, ctypes.c_double), int(max_steps), _ptr(dump, ctypes.c_double),
                int(dump_every or 0), _ptr(loc, ctypes.c_int), _ptr(energy, ctypes.c_double),
                _ptr(pre, ctypes.c_byte), _ptr(post, ctypes.c_byte), ctypes.byref(res))
        if rc != 0:
            raise RuntimeError("run failed")
        s = res.steps
        return {
            "steps": res.steps, "solved": bool(res.solved), "solve_step": res.solve_step,
            "t": res.t, "solve_t": res.solve_t, "dump": dump, "loc": loc[:s], "energy": energy[:s],
            "pre": pre, "post": post,
        }


class Oracle(_Common):
    """CPU restatement of the reference integrator for one formula."""

    def __init__(self, n, m, lits, coff, params=DEFAULT_PARAMS, xl_max=DEFAULT_XL_MAX,
                 alpha_cm=None, precision="fp64"):
        self.lib = _load_oracle()
        self.n, self.m = int(n), int(m)
        self.lits, self.coff = _as_formula(lits, coff)
        p = np.ascontiguousarray(params, dtype=np.float64)
        a = None if alpha_cm is None else np.ascontiguousarray(alpha_cm, dtype=np.float64)
        prec = {"fp64": 1, "fp32": 0}[precision]
        self.h = self.lib.oracle_create(self.n, self.m, _ptr(self.lits, ctypes.c_int32),
                                        _ptr(self.coff, ctypes.c_int64), _ptr(p, ctypes.c_double),
                                        int(xl_max), _ptr(a, ctypes.c_double), prec)
        if not self.h:
            raise ValueError("literal out of range")

    def close(self):
        if self.h:
            self.lib.oracle_destroy(self.h)
            self.h = None

    __del__ = close

    @property
    def xl_max(self) -> float:
        return self.lib.oracle_xl_max(self.h)

    def rhs(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        d = np.zeros_like(x)
        loc = ctypes.c_int()
        e = ctypes.c_double()
        self.lib.oracle_rhs(self.h, _ptr(x, ctypes.c_double), _ptr(d, ctypes.c_double),
                            ctypes.byref(loc), ctypes.byref(e))
        return d, loc.value, e.value

    def dostep(self, x, dxdt, h):
        x = np.ascontiguousarray(x, dtype=np.float64)
        dxdt = np.ascontiguousarray(dxdt, dtype=np.float64)
        o = np.zeros_like(x)
        self.lib.oracle_dostep(self.h, _ptr(x, ctypes.c_double), _ptr(dxdt, ctypes.c_double),
                               float(h), _ptr(o, ctypes.c_double))
        return o

    def run(self, x0, max_steps, dump_every=0):
        return self._run_common(lambda *a: self.lib.oracle_run(self.h, *a), x0, max_steps,
                                dump_every)

    def init_state(self, seed=0, replica=0):
        x = np.zeros(self.n + 2 * self.m, dtype=np.float64)
        self.lib.oracle_init_state(self.h, int(seed), int(replica), _ptr(x, ctypes.c_double))
        return x

    def check(self, assign) -> int:
        a = np.ascontiguousarray(assign, dtype=np.int8)
        return int(self.lib.oracle_check(self.h, _ptr(a, ctypes.c_byte)))


_ref_lib = None


def reference_available() -> bool:
    return os.path.exists(REF_SO)


def _load_ref():
    global _ref_lib
    if _ref_lib is None:
        lib = ctypes.CDLL(REF_SO)
        lib.ref_setup.argtypes = [ctypes.c_int, ctypes.c_int, _I32, _I64, _D, ctypes.c_int]
        lib.ref_xl_max.restype = ctypes.c_double
        lib.ref_rhs.argtypes = [_D, ctypes.c_double, _D, _I, _D]
        lib.ref_dostep.argtypes = [_D, _D, ctypes.c_double, _D]
        lib.ref_run.argtypes = [_D, ctypes.c_int, _D, ctypes.c_int, _I, _D, _S8, _S8,
                                ctypes.POINTER(RunResult)]
        lib.ref_generate_planted.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_ulonglong, _I32, _I64, _S8]
        lib.ref_initial_state_uniform.argtypes = [_I32, _I64, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_ulonglong, _D]
        _ref_lib = lib
    return _ref_lib


def planted_instance(n, m, p0=0.08, p1=0.46, seed=0, init_seed=None):
    """(lits, clause_off, planted, x0) of the library's planted generator and uniform initial
    state for these arguments, built by the reference harness library (instance_gen.h) so
    that the process needs nothing else; x0 is None without init_seed."""
    lib = _load_ref()
    lits = np.zeros(3 * int(m), dtype=np.int32)
    off = np.zeros(int(m) + 1, dtype=np.int64)
    sigma = np.zeros(int(n), dtype=np.int8)
    if lib.ref_generate_planted(int(n), int(m), float(p0), float(p1), int(seed) & (2**64 - 1),
                                _ptr(lits, ctypes.c_int32), _ptr(off, ctypes.c_int64),
                                _ptr(sigma, ctypes.c_byte)) != 0:
        raise ValueError("bad generator arguments")
    x0 = None
    if init_seed is not None:
        x0 = np.zeros(int(n) + 2 * int(m), dtype=np.float64)
        lib.ref_initial_state_uniform(_ptr(lits, ctypes.c_int32), _ptr(off, ctypes.c_int64),
                                      int(n), int(m), int(init_seed) & (2**64 - 1),
                                      _ptr(x0, ctypes.c_double))
    return lits, off, sigma, x0


class Reference(_Common):
    """The unmodified reference dynex.cc (per-step harness).  One live instance per process."""

    def __init__(self, n, m, lits, coff, params=DEFAULT_PARAMS, xl_max=DEFAULT_XL_MAX):
        self.lib = _load_ref()
        self.n, self.m = int(n), int(m)
        self.lits, self.coff = _as_formula(lits, coff)
        p = np.ascontiguousarray(params, dtype=np.float64)
        rc = self.lib.ref_setup(self.n, self.m, _ptr(self.lits, ctypes.c_int32),
                                _ptr(self.coff, ctypes.c_int64), _ptr(p, ctypes.c_double),
                                int(xl_max))
        if rc != 0:
            raise ValueError("reference rejected the formula")

    @property
    def xl_max(self) -> float:
        return self.lib.ref_xl_max()

    def rhs(self, x, t=0.0):
        x = np.ascontiguousarray(x, dtype=np.float64)
        d = np.zeros_like(x)
        loc = ctypes.c_int()
        e = ctypes.c_double()
        self.lib.ref_rhs(_ptr(x, ctypes.c_double), float(t), _ptr(d, ctypes.c_double),
                         ctypes.byref(loc), ctypes.byref(e))
        return d, loc.value, e.value

    def dostep(self, x, dxdt, h):
        x = np.ascontiguousarray(x, dtype=np.float64)
        dxdt = np.ascontiguousarray(dxdt, dtype=np.float64)
        o = np.zeros_like(x)
        self.lib.ref_dostep(_ptr(x, ctypes.c_double), _ptr(dxdt, ctypes.c_double), float(h),
                            _ptr(o, ctypes.c_double))
        return o

    def run(self, x0, max_steps, dump_every=0):
        return self._run_common(self.lib.ref_run, x0, max_steps, dump_every)


class GpuPriorArt:
    """The reference's GPU prior art (dynex.cu, unmodified, sm_100a) driven by its own host
    loop with a step cap (ref_gpu_harness.cu).  For timing only: its arithmetic differs from
    dynex.cc (atomics in arbitrary order, its own step-size rule).  One per process."""

    def __init__(self, n, m, lits, coff, params=DEFAULT_PARAMS, xl_max=DEFAULT_XL_MAX):
        lib = ctypes.CDLL(REF_GPU_SO)
        lib.refgpu_setup.argtypes = [ctypes.c_int, ctypes.c_int, _I32, _I64, _D, ctypes.c_int]
        lib.refgpu_run.argtypes = [_D, ctypes.c_int, _D, _I, _I]
        self.lib = lib
        self.n, self.m = int(n), int(m)
        lits, coff = _as_formula(lits, coff)
        p = np.ascontiguousarray(params, dtype=np.float64)
        if lib.refgpu_setup(self.n, self.m, _ptr(lits, ctypes.c_int32), _ptr(coff, ctypes.c_int64),
                            _ptr(p, ctypes.c_double), int(xl_max)) != 0:
            raise RuntimeError("reference GPU set-up failed")

    def run(self, x0, max_steps):
        """(wall ms, steps done, last unsatisfied count) of up to max_steps steps from x0."""
        x0 = np.ascontiguousarray(x0, dtype=np.float64)
        ms = ctypes.c_double()
        steps = ctypes.c_int()
        loc = ctypes.c_int()
        if self.lib.refgpu_run(_ptr(x0, ctypes.c_double), int(max_steps), ctypes.byref(ms),
                               ctypes.byref(steps), ctypes.byref(loc)) != 0:
            raise RuntimeError("reference GPU run failed")
        return ms.value, steps.value, loc.value

    def close(self):
        self.lib.refgpu_teardown()


def read_cnf(path):
    """Minimal DIMACS reader for tests: (n, m, lits int32, clause_off int64)."""
    n = m = None
    lits, coff = [], [0]
    cur = 0
    with open(path) as f:
        for line in f:
            tok = line.split()
            if not tok:
                continue
            if tok[0] == "c":
                continue
            if tok[0] == "p":
                n, m = int(tok[2]), int(tok[3])
                continue
            for t in tok:
                v = int(t)
                if v == 0:
                    coff.append(coff[-1] + cur)
                    cur = 0
                else:
                    lits.append(v)
                    cur += 1
    return n, m, np.array(lits, dtype=np.int32), np.array(coff[: m + 1], dtype=np.int64)
