"""The C ABI: both libraries load and export every function their headers declare, and the
host side's checks refuse bad input without changing anything.  No GPU is needed here."""
import ctypes as C
import os
import re

import pytest

from bearing_b200 import _ffi
from bearing_b200.world import BearingError, World

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b((?:bg|bw)_[a-z_]+)\s*\(", text, flags=re.M)))


def test_headers_declare_what_the_bindings_know():
    assert declared("bearing_gpu.h") == sorted(_ffi.GPU_SYMBOLS)
    assert declared("bearing_world.h") == sorted(_ffi.HOST_SYMBOLS)


def test_gpu_library_loads_and_exports_every_declared_function():
    lib = C.CDLL(_ffi.lib_path("libbearing_gpu.so"))
    for name in declared("bearing_gpu.h"):
        assert hasattr(lib, name), name
    assert _ffi.gpu().bg_version() >> 16 == 1


def test_host_library_loads_and_exports_every_declared_function():
    lib = C.CDLL(_ffi.lib_path("libbearing_host.so"))
    for name in declared("bearing_world.h"):
        assert hasattr(lib, name), name


def test_oracle_library_loads():
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_build", "liboracle.so"))
    for name in ("oracle_solve_step", "oracle_solver", "oracle_atan2", "oracle_release_threads"):
        assert hasattr(lib, name)


def test_calls_on_a_null_context_are_refused():
    g = _ffi.gpu()
    assert g.bg_solve(None, None) == _ffi.BG_EINVAL
    assert g.bg_restore(None) == _ffi.BG_EINVAL
    assert g.bg_upload(None, None, None) == _ffi.BG_EINVAL
    assert g.bg_register_host(None, None, None, 0) == _ffi.BG_EINVAL
    assert g.bg_unregister_host(None) == _ffi.BG_EINVAL
    assert g.bg_registered_bytes(None) == 0
    assert g.bg_last_error(None) == b"no context"
    g.bg_destroy(None)


def test_bg_create_on_a_missing_device_returns_null():
    g = _ffi.gpu()
    assert not g.bg_create(999, 0)
    assert not g.bg_create(-1, 0)


def test_world_refuses_what_is_not_on_this_path():
    w = World({}, solver=(1, 0))
    with pytest.raises(BearingError):
        w.addBody({"shape": "hull"})
    with pytest.raises(BearingError):
        w.addBody({"rotation": (0, 0, 0, 0)})
    with pytest.raises(BearingError):
        w.addBody({"colour": 3})
    with pytest.raises(BearingError):
        w.step(0)
    with pytest.raises(BearingError):
        w.step(float("inf"))
    with pytest.raises(BearingError):
        World({"sleeping": True}, solver=(1, 0))
    with pytest.raises(BearingError):
        World({"substeps": 0}, solver=(1, 0))
    assert w.stats()["bodies"] == 0
    w.destroy()


def test_world_without_a_solver_refuses_to_step():
    lib = _ffi.host()
    opts = _ffi.Options((C.c_double * 3)(0, -9.81, 0), 8)
    w = lib.bw_create(C.byref(opts))
    assert lib.bw_step(w, C.c_double(1 / 60)) == _ffi.BG_EUNSUPPORTED
    assert b"no solve stage" in lib.bw_last_error(w)
    lib.bw_destroy(w)


def test_rotation_is_normalised_on_the_way_in():
    # src/core/check.js:106-117: scaled by the largest component, then normalised.
    w = World({}, solver=(1, 0))
    s = w.addBody({"rotation": (0.0, 0.0, 3.0, 4.0)})
    q = w.state()["rotation"][4 * s:4 * s + 4]
    x, y, z, ww = 0.0, 0.0, 3.0 / 4.0, 1.0
    k = 1 / (x * x + y * y + z * z + ww * ww) ** 0.5
    assert list(q) == [x * k, y * k, z * k, ww * k]
    w.destroy()


def test_mass_and_inertia_follow_the_shape():
    # src/shapes.js:14-56 and src/world.js:2152-2274
    import math
    w = World({}, solver=(1, 0))
    box = w.addBody({"size": (1.0, 2.0, 3.0), "density": 2.0})
    ball = w.addBody({"shape": "sphere", "radius": 0.5})
    cap = w.addBody({"shape": "capsule", "radius": 0.25, "height": 1.5})
    B, _, _ = w.views()
    inv_mass = [B.inv_mass[i] for i in range(3)]
    assert inv_mass[box] == 1 / 12.0
    vol = (4 / 3) * math.pi * 0.5 * 0.5 * 0.5
    assert inv_mass[ball] == 1 / (1000 * vol)
    m = 12.0
    assert [B.inertia[3 * box + k] for k in range(3)] == [m * (4 + 9) / 12, m * (1 + 9) / 12, m * (1 + 4) / 12]
    assert B.dims[3 * cap] == 0.25 and B.dims[3 * cap + 1] == 1.5
    w.destroy()


def test_static_entry_point_refuses_bad_counts_and_starts_before_touching_a_device():
    # bg_solve_step_static checks the counts and the colour starts on the host, as bg_solve_step
    # does, and returns before any CUDA call: these run without a GPU.
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_io
    from bearing_b200 import scenes
    from stage_io import StageCopy
    w = World({}, solver=oracle_io.solver(0))
    scenes.pyramid(w, rows=6)
    for _ in range(3):
        w.step(1 / 60)
    w.begin_step(1 / 60)
    base = StageCopy(w)
    g = _ffi.gpu()
    for bad in ("starts[0]", "decreasing", "past count", "solved", "bodies", "rows", "dt", "null column"):
        work = base.copy()
        B, R, S = work.views()
        if bad == "starts[0]":
            R.starts[0] = 1
        elif bad == "decreasing":
            R.starts[1] = R.starts[2] + 1
        elif bad == "past count":
            R.starts[34] = R.count + 5000
        elif bad == "solved":
            R.solved = R.starts[33] + 1
        elif bad == "bodies":
            B.capacity = _ffi.BG_STATIC_MAX_BODIES + 1
        elif bad == "rows":
            R.count = _ffi.BG_STATIC_MAX_ROWS + 1
        elif bad == "dt":
            S.dt = 0.0
        else:
            R.normal = None
        assert g.bg_solve_step_static(C.byref(B), C.byref(R), C.byref(S), None) == _ffi.BG_EINVAL, bad
    w.destroy()
