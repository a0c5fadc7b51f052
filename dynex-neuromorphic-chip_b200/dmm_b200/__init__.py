"""B200-native digital-memcomputing (DMM) SAT integrator: Python host mirror of the C ABI.

The compute path is ``lib/libdmm.so`` (hand-written sm_100a kernels behind include/dmm.h);
this package only binds it.  Importing works without a GPU; creating an instance needs one.
"""
from ._lib import (CANCELLED, RUNNING, SOLVED, STEP_LIMIT, TIME_LIMIT, DmmError, Params,
                   default_params, lib)
from .batch import Batch
from .cnf import (Formula, check_assignment, from_arrays, generate_planted,
                  initial_state_reference, initial_state_uniform, read_cnf, read_state,
                  write_cnf, write_state)
from .instance import Instance, Result
from .server import Server

__all__ = [
    "Batch", "CANCELLED", "DmmError", "Formula", "Instance", "Params", "RUNNING", "Result",
    "SOLVED", "STEP_LIMIT", "Server", "TIME_LIMIT", "check_assignment", "default_params",
    "from_arrays", "generate_planted", "initial_state_reference", "initial_state_uniform", "lib",
    "read_cnf", "read_state", "write_cnf", "write_state",
]
