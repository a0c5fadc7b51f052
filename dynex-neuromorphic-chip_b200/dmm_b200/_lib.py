"""ctypes binding of include/dmm.h (libdmm.so).

The library is required: there is no CPU fallback.  Loading fails loudly when
``lib/libdmm.so`` has not been built (``python dynex-neuromorphic-chip_b200/build.py``).
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libdmm.so")
CLI_PATH = os.path.join(PKG_ROOT, "bin", "dynex")

# dmm_status
OK = 0
STATUS_NAMES = {
    0: "DMM_OK", 1: "DMM_ERR_ARG", 2: "DMM_ERR_CUDA", 3: "DMM_ERR_NOMEM", 4: "DMM_ERR_NO_DEVICE",
    5: "DMM_ERR_LITERAL", 6: "DMM_ERR_CLAUSE_LEN", 7: "DMM_ERR_PARSE", 8: "DMM_ERR_IO",
    9: "DMM_ERR_BUDGET", 10: "DMM_ERR_STATE", 11: "DMM_ERR_BUILD",
}
# dmm_run_status
RUNNING, SOLVED, STEP_LIMIT, TIME_LIMIT, CANCELLED = 0, 1, 2, 3, 4
RUN_STATUS_NAMES = {0: "RUNNING", 1: "SOLVED", 2: "STEP_LIMIT", 3: "TIME_LIMIT", 4: "CANCELLED"}
PRECISIONS = {"fp32": 0, "fp64": 1}


class DmmError(RuntimeError):
    def __init__(self, status: int, text: str, detail: str):
        self.status = status
        self.name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{self.name}: {text}" + (f" ({detail})" if detail else ""))


class Params(ctypes.Structure):
    _fields_ = [("alpha", ctypes.c_double), ("beta", ctypes.c_double), ("gamma", ctypes.c_double),
                ("delta", ctypes.c_double), ("epsilon", ctypes.c_double), ("zeta", ctypes.c_double),
                ("xl_max", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class Report(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("steps", ctypes.c_int32), ("t", ctypes.c_double),
                ("loc", ctypes.c_int32), ("best_loc", ctypes.c_int32), ("energy", ctypes.c_double),
                ("solved_step", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("solved_t", ctypes.c_double), ("wall_s", ctypes.c_double)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}
        d["status_name"] = RUN_STATUS_NAMES.get(self.status, str(self.status))
        return d


class Limits(ctypes.Structure):
    _fields_ = [("max_steps", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("wall_s", ctypes.c_double)]


class Tuning(ctypes.Structure):
    _fields_ = [("clause_tile", ctypes.c_int32), ("var_group", ctypes.c_int32),
                ("var_tile", ctypes.c_int32), ("steps_per_graph", ctypes.c_int32),
                ("blocks_per_sm", ctypes.c_int32), ("launch_mode", ctypes.c_int32),
                ("u_layout", ctypes.c_int32), ("l2_policy", ctypes.c_int32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Cnf(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("m", ctypes.c_int32), ("nlits", ctypes.c_int64),
                ("lits", ctypes.POINTER(ctypes.c_int32)),
                ("clause_off", ctypes.POINTER(ctypes.c_int64)),
                ("max_occurrence", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class BatchStats(ctypes.Structure):
    _fields_ = [("clause_updates", ctypes.c_int64), ("steps_launched", ctypes.c_int64),
                ("solved", ctypes.c_int32), ("unsolved", ctypes.c_int32),
                ("wall_s", ctypes.c_double), ("device_ms", ctypes.c_double)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int32), ("device", ctypes.c_int32),
                ("budget_bytes", ctypes.c_int64), ("max_slots", ctypes.c_int32),
                ("steps_per_launch", ctypes.c_int32)]


class ServerResult(ctypes.Structure):
    _fields_ = [("ticket", ctypes.c_int64), ("report", Report), ("submit_s", ctypes.c_double),
                ("admit_s", ctypes.c_double), ("finish_s", ctypes.c_double)]


_P = ctypes.POINTER
_vp = ctypes.c_void_p
_i32, _i64, _u64, _d = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_double
_pi32, _pi64, _pi8, _pd = _P(ctypes.c_int32), _P(ctypes.c_int64), _P(ctypes.c_int8), _P(ctypes.c_double)

# name -> (restype, argtypes); every entry point declared in include/dmm.h
SIGNATURES = {
    "dmm_abi_version": (_i32, []),
    "dmm_status_string": (ctypes.c_char_p, [_i32]),
    "dmm_last_error": (ctypes.c_char_p, []),
    "dmm_params_default": (None, [_P(Params)]),
    "dmm_device_count": (_i32, []),
    "dmm_release_cached_memory": (None, []),
    "dmm_cnf_read": (_i32, [ctypes.c_char_p, _P(_P(Cnf))]),
    "dmm_cnf_from_arrays": (_i32, [_pi32, _pi64, _i32, _i32, _P(_P(Cnf))]),
    "dmm_cnf_free": (None, [_P(Cnf)]),
    "dmm_cnf_write": (_i32, [_P(Cnf), ctypes.c_char_p, _pi8]),
    "dmm_state_write": (_i32, [ctypes.c_char_p, _pd, _i32, _i32, _d]),
    "dmm_state_read": (_i32, [ctypes.c_char_p, _i32, _i32, _i32, _pd, _pd]),
    "dmm_cnf_generate_planted": (_i32, [_i32, _i32, _d, _d, _u64, _P(_P(Cnf)), _pi8]),
    "dmm_check_assignment": (_i64, [_pi32, _pi64, _i32, _i32, _pi8]),
    "dmm_initial_state_reference": (_i32, [_pi32, _pi64, _i32, _i32, _i32, _i32, _pd, _pi32]),
    "dmm_initial_state_uniform": (_i32, [_pi32, _pi64, _i32, _i32, _u64, _pd]),
    "dmm_instance_create": (_i32, [_pi32, _pi64, _i32, _i32, _i32, _i32, _P(_vp)]),
    "dmm_instance_destroy": (None, [_vp]),
    "dmm_instance_set_params": (_i32, [_vp, _P(Params), _pd]),
    "dmm_instance_set_tuning": (_i32, [_vp, _P(Tuning)]),
    "dmm_instance_get_tuning": (_i32, [_vp, _P(Tuning)]),
    "dmm_instance_set_state": (_i32, [_vp, _pd]),
    "dmm_instance_set_state_at": (_i32, [_vp, _pd, _d, _i32]),
    "dmm_instance_get_state": (_i32, [_vp, _pd, _pd]),
    "dmm_instance_rhs": (_i32, [_vp, _pd, _pd, _pi32, _pd]),
    "dmm_instance_dostep": (_i32, [_vp, _pd, _pd, _d, _pd]),
    "dmm_instance_step": (_i32, [_vp, _i32, _P(Report)]),
    "dmm_instance_solve": (_i32, [_vp, _P(Limits), _P(Report)]),
    "dmm_instance_report": (_i32, [_vp, _P(Report)]),
    "dmm_instance_assignment": (_i32, [_vp, _pi8, _pi8]),
    "dmm_instance_profile": (_i32, [_vp, _i32, _i64, _pd, _pd]),
    "dmm_instance_time_steps": (_i32, [_vp, _i32, _pd]),
    "dmm_instance_time_steps_flushed": (_i32, [_vp, _i32, _i64, _pd]),
    "dmm_instance_trace_phases": (_i32, [_vp, _i32, _pd]),
    "dmm_instance_launch_form": (_i32, [_vp]),
    "dmm_instance_test_barrier_timeout": (_i32, [_vp]),
    "dmm_rhs3_f32_noalloc": (_i32, [_vp, _i32, _i32, _vp, _P(Params), _vp, _vp, _vp]),
    "dmm_batch_create": (_i32, [_i32, _i32, _i32, _i64, _i64, _i64, _P(_vp)]),
    "dmm_batch_destroy": (None, [_vp]),
    "dmm_batch_set_tuning": (_i32, [_vp, _P(Tuning)]),
    "dmm_batch_add": (_i32, [_vp, _pi32, _pi64, _i32, _i32, _P(Params), _pd, _i32, _pi32]),
    "dmm_batch_run": (_i32, [_vp, _d, _P(BatchStats)]),
    "dmm_batch_run_until": (_i32, [_vp, _d, _i32, _P(BatchStats)]),
    "dmm_batch_result": (_i32, [_vp, _i32, _P(Report), _pi8]),
    "dmm_batch_assignment": (_i32, [_vp, _i32, _pi8, _pi8]),
    "dmm_batch_state": (_i32, [_vp, _i32, _pd, _pd]),
    "dmm_batch_set_state_at": (_i32, [_vp, _i32, _pd, _d, _i32]),
    "dmm_server_create": (_i32, [_P(ServerConfig), _P(_vp)]),
    "dmm_server_destroy": (None, [_vp]),
    "dmm_server_submit": (_i32, [_vp, _pi32, _pi64, _i32, _i32, _P(Params), _pd, _u64, _i32,
                                 _pi64]),
    "dmm_server_pump": (_i32, [_vp, _pi32, _pi32]),
    "dmm_server_take": (_i32, [_vp, _P(ServerResult), _i32, _pi32]),
    "dmm_server_assignment": (_i32, [_vp, _i64, _pi8, _i32]),
    "dmm_server_clock": (_d, [_vp]),
}

_lib = None


def lib():
    """The loaded libdmm.so (raises if it is missing; there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libdmm.so is not built ({LIB_PATH}); run "
                              "python dynex-neuromorphic-chip_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != OK:
        L = lib()
        text = L.dmm_status_string(status).decode()
        detail = (L.dmm_last_error() or b"").decode()
        raise DmmError(status, text, detail)


def ptr(a, ctype):
    """Pointer to a contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def default_params(**over) -> Params:
    p = Params()
    lib().dmm_params_default(ctypes.byref(p))
    for k, v in over.items():
        setattr(p, k, v)
    return p
