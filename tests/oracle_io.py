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
        _pd = C.POINTER(C.c_double)
        _lib.oracle_dual_create.restype = C.c_void_p
        _lib.oracle_dual_create.argtypes = [C.POINTER(_ffi.Bodies), _pd, _pd]
        _lib.oracle_dual_destroy.argtypes = [C.c_void_p]
        _lib.oracle_dual_seed.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32]
        _lib.oracle_dual_step.argtypes = [C.c_void_p, C.POINTER(_ffi.Bodies), C.POINTER(_ffi.Rows),
                                          C.POINTER(_ffi.Step), C.POINTER(_ffi.RowMemory)]
        _lib.oracle_dual_pose.argtypes = [C.c_void_p, C.c_int32, _pd, _pd]
        _lib.oracle_stage_jvp.argtypes = [C.POINTER(_ffi.Bodies), C.POINTER(_ffi.Rows), C.POINTER(_ffi.Step),
                                          C.POINTER(_ffi.Bodies), C.POINTER(_ffi.Rows)]
    return _lib


def solver(workers=0):
    """(function address, user) of the oracle as a bw_solver, for World(solver=...)."""
    return C.cast(lib().oracle_solver, C.c_void_p).value, workers


def solve(copy, workers=0):
    B, R, S = copy.views()
    rc = lib().oracle_solve_step(C.byref(B), C.byref(R), C.byref(S), workers)
    assert rc == 0
    return copy


class DualWorld:
    """A World stepped with the oracle's solve stage, carrying derivatives along five directions
    (oracle_dual_*): every body's friction, every body's restitution, and the three components of
    one body's initial velocity.  The world's own double state follows the dual run's real parts."""

    def __init__(self, world, friction, restitution, launched):
        import numpy as np
        self.world = world
        self.lib = lib()
        B, _, _ = world.views()
        n = world._count
        self._fr = np.full(n, float(friction))
        self._re = np.full(n, float(restitution))
        pd = C.POINTER(C.c_double)
        self.h = self.lib.oracle_dual_create(C.byref(B), self._fr.ctypes.data_as(pd), self._re.ctypes.data_as(pd))
        self.lib.oracle_dual_seed(self.h, 1, 0, 0, 0)
        self.lib.oracle_dual_seed(self.h, 2, 0, 0, 1)
        for k in range(3):
            self.lib.oracle_dual_seed(self.h, 0, launched, k, 2 + k)

    def step(self, dt):
        from bearing_b200.adjoint import _Memory
        w = self.world
        w.begin_step(dt)
        B, R, S = w.views()
        mem = _Memory(R.count)
        assert _ffi.host().bw_row_memory_get(w._w, C.byref(mem.s)) == 0
        rc = self.lib.oracle_dual_step(self.h, C.byref(B), C.byref(R), C.byref(S), C.byref(mem.s))
        assert rc == 0, f"oracle_dual_step: {rc}"
        w.end_step()

    def pose(self, slot):
        """(position and rotation, 7; their derivatives, 7 x 5)."""
        import numpy as np
        v, t = np.zeros(7), np.zeros(35)
        pd = C.POINTER(C.c_double)
        self.lib.oracle_dual_pose(self.h, slot, v.ctypes.data_as(pd), t.ctypes.data_as(pd))
        return v, t.reshape(7, 5)

    def close(self):
        if self.h:
            self.lib.oracle_dual_destroy(self.h)
            self.h = None
