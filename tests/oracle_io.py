"""The oracle (oracle/solve_stage.cpp) as the tests call it: the checker, never the product."""
import ctypes as C
import os

from bearing_b200 import _ffi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(os.path.join(ROOT, "oracle", "_build", "liboracle.so"))
        _lib.oracle_solve_step.argtypes = [C.POINTER(_ffi.Bodies), C.POINTER(_ffi.Rows), C.POINTER(_ffi.Step), C.c_int32]
        _lib.oracle_solve_step.restype = C.c_int32
        _lib.oracle_atan2.argtypes = [C.c_double, C.c_double]
        _lib.oracle_atan2.restype = C.c_double
    return _lib


def solver(workers=0):
    """(function address, user) of the oracle as a bw_solver, for World(solver=...)."""
    return C.cast(lib().oracle_solver, C.c_void_p).value, workers


def solve(copy, workers=0):
    B, R, S = copy.views()
    rc = lib().oracle_solve_step(C.byref(B), C.byref(R), C.byref(S), workers)
    assert rc == 0
    return copy
