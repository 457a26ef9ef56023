"""The CUDA library as the GPU tests call it, through its C ABI."""
import ctypes as C

from bearing_b200 import _ffi

_ctx = {}
PATHS = {"auto": 0, "grid": _ffi.BG_FLAG_GRID, "block": _ffi.BG_FLAG_BLOCK}


def ctx(path="auto"):
    if path not in _ctx:
        c = _ffi.gpu().bg_create(0, PATHS[path])
        assert c, "bg_create(0) failed"
        _ctx[path] = c
    return _ctx[path]


def error(path="auto"):
    return _ffi.gpu().bg_last_error(ctx(path)).decode()


def solve(copy, path="auto"):
    B, R, S = copy.views()
    rc = _ffi.gpu().bg_solve_step(ctx(path), C.byref(B), C.byref(R), C.byref(S))
    assert rc == 0, f"bg_solve_step: {rc} {error(path)}"
    return copy
