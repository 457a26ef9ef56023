"""World: the reference's World API (src/world.js, src/bearing.d.ts:512-575) for boxes, spheres
and capsules, with the contact solve stage on a B200.

The host side of each step (bounds, pair finding, narrowphase, colouring, warm-start memory,
store, transforms) runs in ``libbearing_host.so``; the solve stage (src/world.js:962-1032) runs
in ``libbearing_gpu.so`` through its C ABI.  ``world.step(dt)``, ``world.transforms`` and
``world.workers`` mean what they mean in the reference.  There is no CPU fallback for the solve
stage: a World made with the GPU solver fails loudly if the CUDA library cannot run.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

from . import _ffi, check

SHAPES = {"box": _ffi.BG_BOX, "sphere": _ffi.BG_SPHERE, "capsule": _ffi.BG_CAPSULE}
TYPES = {"dynamic": _ffi.BG_DYNAMIC, "static": _ffi.BG_STATIC, "kinematic": _ffi.BG_KINEMATIC}

# Defaults: src/world.js:205-221.
DEFAULTS = dict(
    type="dynamic", shape="box", size=(1.0, 1.0, 1.0), radius=0.5, height=2.0, density=1000.0, mass=0.0,
    friction=0.5, restitution=0.0, damping=0.0, angularDamping=0.0, gravityScale=1.0,
    position=(0.0, 0.0, 0.0), rotation=(0.0, 0.0, 0.0, 1.0), velocity=(0.0, 0.0, 0.0),
    angularVelocity=(0.0, 0.0, 0.0),
)
# The reference's option lists (src/world.js:57-82, 190-196), for its messages; this path covers
# boxes, spheres and capsules that are dynamic, static or kinematic.
REFERENCE_BODY_OPTIONS = [
    "type", "shape", "size", "radius", "height", "vertices", "indices", "heights", "columns", "spacing", "parts",
    "density", "mass", "inertia", "centerOfMass",
    "friction", "restitution", "damping", "angularDamping", "gravityScale", "layers", "mask", "sensor",
    "lockRotation", "maxSlope", "stepHeight",
    "position", "rotation", "velocity", "angularVelocity",
]
REFERENCE_SHAPES = ["box", "sphere", "capsule", "hull", "compound", "mesh", "heightfield"]
REFERENCE_TYPES = ["dynamic", "static", "kinematic", "character"]
SHAPE_SIZES = {"box": ["size"], "sphere": ["radius"], "capsule": ["radius", "height"], "hull": ["vertices"],
               "compound": ["parts"], "mesh": ["vertices", "indices"], "heightfield": ["heights", "columns", "spacing"]}
SIZES = ["size", "radius", "height", "vertices", "indices", "heights", "columns", "spacing", "parts"]
BODY_OPTIONS = set(DEFAULTS)
WORLD_OPTIONS = ["gravity", "substeps", "sleeping", "workers", "reuse"]


class BearingError(RuntimeError):
    """A step or a setter failed; the message is the library's."""


class GpuSolver:
    """The solve stage on one CUDA device, through bg_solve_step (bearing_gpu.h)."""

    def __init__(self, device: int = 0, flags: int = 0):
        self.lib = _ffi.gpu()
        self.ctx = self.lib.bg_create(device, flags)
        if not self.ctx:
            raise BearingError(f"bg_create({device}) failed: no usable CUDA device")
        self.fn = C.cast(self.lib.bg_solve_step, C.c_void_p).value
        # bw_solver takes (user, bodies, rows, step); bg_solve_step takes (ctx, bodies, rows, step).
        self.user = self.ctx
        # bw_narrowphase takes (user, bodies, gravity, pairs, out), bg_collide (ctx, ...) alike.
        self.collide_fn = C.cast(self.lib.bg_collide, C.c_void_p).value
        # bw_contact_solver and bg_contact_step alike.
        self.contact_fn = C.cast(self.lib.bg_contact_step, C.c_void_p).value

    def contact_ms(self):
        """The last bg_contact_step's device times in ms: narrowphase, rows/colours/order, stage, store."""
        ms = (C.c_double * 4)()
        if self.lib.bg_last_contact_ms(self.ctx, ms) != 0:
            return None
        return list(ms)

    def error(self) -> str:
        return self.lib.bg_last_error(self.ctx).decode()

    def close(self):
        if self.ctx:
            self.lib.bg_destroy(self.ctx)
            self.ctx = None


def _workers(name, value):
    """'auto' or a whole number from 0 (src/world.js _setWorkers): `name` is "World" for the
    option, "world.workers" for the property."""
    if value != "auto" and (isinstance(value, bool) or not isinstance(value, int) or value < 0):
        text = f"must be 'auto' or a whole number, 0 or more, got {check.show(value)}"
        check.fail("", f"World: workers {text}" if name == "World" else f"world.workers {text}")
    return value


def _not_here(caller, what):
    check.fail(caller, f"{what} is not on this path (boxes, spheres and capsules, dynamic, static or kinematic)")


def _resolve(caller, given_):
    """addBody's options checked in the reference's order (src/world.js:2328-2462, from DEFAULTS),
    the ones this path does not cover refused where the reference would first meet them."""
    given = check.options(caller, given_)
    check.known(caller, given, REFERENCE_BODY_OPTIONS)

    def has(k):
        return k in given

    shape = check.one_of(caller, "shape", given["shape"], REFERENCE_SHAPES) if has("shape") else "box"
    level = shape in ("mesh", "heightfield")
    ttype = check.one_of(caller, "type", given["type"], REFERENCE_TYPES) if has("type") else \
        ("static" if level else "dynamic")
    for k in SIZES:
        if has(k) and k not in SHAPE_SIZES[shape]:
            check.fail(caller, f"a {shape} has no {k}")
    if level and ttype in ("dynamic", "character"):
        check.fail(caller, f"type must be 'static' or 'kinematic' for a {shape}, got '{ttype}'")
    if shape in ("hull", "compound") and ttype == "character":
        check.fail(caller, f"type must be 'dynamic', 'static' or 'kinematic' for a {shape}, got 'character'")
    if shape not in SHAPES:
        _not_here(caller, f"a {shape}")
    if ttype not in TYPES:
        _not_here(caller, f"a {ttype} body")
    size = check.positive3(caller, "size", given["size"]) if has("size") else DEFAULTS["size"]
    radius = check.positive(caller, "radius", given["radius"]) if has("radius") else DEFAULTS["radius"]
    height = check.positive(caller, "height", given["height"]) if has("height") else DEFAULTS["height"]
    if shape == "capsule" and height < 2 * radius:
        check.fail(caller, f"height must be at least twice radius ({check.js_number(2 * radius)}), "
                           f"got {check.js_number(height)}")
    if has("mass") and has("density"):
        check.fail(caller, "give mass or density, not both")
    mass = check.positive(caller, "mass", given["mass"]) if has("mass") else 0.0
    density = check.positive(caller, "density", given["density"]) if has("density") else DEFAULTS["density"]
    for k in ("inertia", "centerOfMass"):
        if has(k):
            _not_here(caller, f"{k} given")
    friction = check.at_least_zero(caller, "friction", given["friction"]) if has("friction") else DEFAULTS["friction"]
    restitution = DEFAULTS["restitution"]
    if has("restitution"):
        r = given["restitution"]
        if isinstance(r, bool) or not isinstance(r, (int, float)) or not (0 <= r <= 1):
            check.fail(caller, f"restitution must be from 0 to 1, got {check.show(r)}")
        restitution = float(r)
    damping = check.at_least_zero(caller, "damping", given["damping"]) if has("damping") else DEFAULTS["damping"]
    angular_damping = check.at_least_zero(caller, "angularDamping", given["angularDamping"]) \
        if has("angularDamping") else DEFAULTS["angularDamping"]
    gravity_scale = check.finite(caller, "gravityScale", given["gravityScale"]) if has("gravityScale") \
        else DEFAULTS["gravityScale"]
    for k in ("layers", "mask", "sensor", "lockRotation"):
        if has(k):
            _not_here(caller, f"{k}")
    if ttype != "character":
        for k in ("maxSlope", "stepHeight"):
            if has(k):
                check.fail(caller, f"a {ttype} body has no {k}")
    position = check.vec3(caller, "position", given["position"]) if has("position") else DEFAULTS["position"]
    rotation = check.quat(caller, "rotation", given["rotation"]) if has("rotation") else DEFAULTS["rotation"]
    if ttype == "static":
        for k in ("velocity", "angularVelocity"):
            if has(k):
                check.fail(caller, f"a static body has no {k}")
        velocity = angular = (0.0, 0.0, 0.0)
    else:
        velocity = check.vec3(caller, "velocity", given["velocity"]) if has("velocity") else DEFAULTS["velocity"]
        angular = check.vec3(caller, "angularVelocity", given["angularVelocity"]) if has("angularVelocity") \
            else DEFAULTS["angularVelocity"]
    return dict(type=ttype, shape=shape, size=size, radius=radius, height=height, density=density, mass=mass,
                friction=friction, restitution=restitution, damping=damping, angularDamping=angular_damping,
                gravityScale=gravity_scale, position=position, rotation=rotation, velocity=velocity,
                angularVelocity=angular)


def _vec(v, n, name):
    v = tuple(float(x) for x in v)
    if len(v) != n or not all(math.isfinite(x) for x in v):
        raise BearingError(f"addBody: {name} must be {n} finite numbers, got {v!r}")
    return v


class World:
    """A world of bodies, stepped with the solve stage on the GPU (or another bw_solver)."""

    def __init__(self, options: dict | None = None, solver=None):
        try:
            o = dict(check.options("World", options))
            # the reference's options (src/world.js:82, 314-395), and this path's own `reuse`
            check.known("World", {k: v for k, v in o.items() if k != "reuse"}, WORLD_OPTIONS[:4])
            g = check.vec3("World", "gravity", o["gravity"]) if "gravity" in o else (0.0, -9.81, 0.0)
            substeps = o.get("substeps", 8)
            if isinstance(substeps, bool) or not isinstance(substeps, int) or substeps < 1:
                check.fail("World", f"substeps must be a whole number, 1 or more, got {check.show(substeps)}")
            if "sleeping" in o and not isinstance(o["sleeping"], bool):
                check.fail("World", f"sleeping must be true or false, got {check.show(o['sleeping'])}")
            self._workers = _workers("World", o.get("workers", "auto"))
        except check.CheckError as e:
            raise BearingError(str(e)) from None
        if o.get("sleeping", False):
            raise BearingError("World: sleeping islands are not on this path; pass sleeping: false")
        self._lib = _ffi.host()
        # reuse: the kept-manifold cache of src/contact.js:388-595 (the reference always keeps one;
        # off by default here, where every pair whose boxes meet is collided afresh each step)
        opts = _ffi.Options((C.c_double * 3)(*g), substeps, 1 if o.get("reuse", False) else 0)
        self._w = self._lib.bw_create(C.byref(opts))
        self._lib.bw_set_workers(self._w, -1 if self._workers == "auto" else min(self._workers, 1 << 20))
        self._count = 0
        self._solver = None
        self._solver_keep = None
        self._narrowphase = None
        self._contact = None
        if solver is None:
            solver = GpuSolver()
        self.set_solver(solver)

    # -- the narrowphase ---------------------------------------------------------------------
    def set_narrowphase(self, device):
        """device: a GpuSolver, whose context then runs each step's narrowphase (bg_collide), or
        None for the host's own.  The step's rows are the same either way."""
        if device is None:
            fn, user = None, None
        else:
            fn, user = device.collide_fn, device.ctx
        if self._lib.bw_set_narrowphase(self._w, fn, user) != 0:
            raise BearingError("set_narrowphase failed")
        self._narrowphase = device

    def set_contact_step(self, device):
        """device: a GpuSolver, whose context then runs each step's whole contact side, from the
        narrowphase to store() (bg_contact_step); the rows stay on the device, so contacts() and
        begin_step() are not available.  Set it before the first step."""
        if not isinstance(device, GpuSolver):
            raise BearingError("set_contact_step takes a GpuSolver")
        if self._lib.bw_set_contact_step(self._w, C.c_void_p(device.contact_fn), C.c_void_p(device.ctx)) != 0:
            raise BearingError(self._error())
        self._contact = device

    # -- the solve stage ---------------------------------------------------------------------
    def set_solver(self, solver):
        """solver: a GpuSolver, or (function address, user pointer) of a bw_solver."""
        if isinstance(solver, GpuSolver):
            fn, user = solver.fn, solver.user
        else:
            fn, user = solver
        self._solver = solver
        rc = self._lib.bw_set_solver(self._w, C.c_void_p(fn), C.c_void_p(user))
        if rc != 0:
            raise BearingError(self._error())

    def _error(self) -> str:
        return self._lib.bw_last_error(self._w).decode()

    # -- bodies ------------------------------------------------------------------------------
    def addBody(self, spec: dict | None = None) -> int:
        """Adds a box, sphere or capsule (src/world.js:563-578); returns its slot.  Every option is
        checked before anything is written, in the reference's order and words (src/world.js
        resolve(), 2328-2462); a call that throws adds nothing."""
        if not self._w:
            raise BearingError("addBody: this world was destroyed")
        try:
            s = _resolve("addBody", spec)
        except check.CheckError as e:
            raise BearingError(str(e)) from None
        b = _ffi.BodySpec()
        b.type = TYPES[s["type"]]
        b.shape = SHAPES[s["shape"]]
        b.size = (C.c_double * 3)(*_vec(s["size"], 3, "size"))
        b.radius = float(s["radius"])
        b.height = float(s["height"])
        b.density = float(s["density"])
        b.mass = float(s["mass"])
        b.friction = float(s["friction"])
        b.restitution = float(s["restitution"])
        b.damping = float(s["damping"])
        b.angular_damping = float(s["angularDamping"])
        b.gravity_scale = float(s["gravityScale"])
        b.position = (C.c_double * 3)(*_vec(s["position"], 3, "position"))
        b.rotation = (C.c_double * 4)(*_vec(s["rotation"], 4, "rotation"))
        b.velocity = (C.c_double * 3)(*_vec(s["velocity"], 3, "velocity"))
        b.angular = (C.c_double * 3)(*_vec(s["angularVelocity"], 3, "angularVelocity"))
        slot = self._lib.bw_add_body(self._w, C.byref(b))
        if slot < 0:
            raise BearingError(self._error())
        self._count = slot + 1
        return slot

    # -- stepping ----------------------------------------------------------------------------
    def step(self, dt: float):
        """One step of dt seconds (src/world.js:880-1072)."""
        if not self._w:
            raise BearingError("step: this world was destroyed")
        if isinstance(dt, bool) or not isinstance(dt, (int, float)) or not (dt > 0) or dt == math.inf:
            raise BearingError(f"step: dt must be a positive number of seconds, got {check.show(dt)}")
        rc = self._lib.bw_step(self._w, float(dt))
        if rc != 0:
            extra = ""
            if self._contact is not None:
                extra = f" ({self._contact.error()})"
            elif isinstance(self._solver, GpuSolver):
                extra = f" ({self._solver.error()})"
            raise BearingError(f"step failed ({rc}): {self._error()}{extra}")

    def begin_step(self, dt: float):
        """The step up to the solve stage; the views then hold the solve stage's input."""
        rc = self._lib.bw_begin_step(self._w, float(dt))
        if rc != 0:
            raise BearingError(self._error())

    def end_step(self):
        rc = self._lib.bw_end_step(self._w)
        if rc != 0:
            raise BearingError(self._error())

    def views(self):
        """(bg_bodies, bg_rows, bg_step) over the world's own columns."""
        B, R, S = _ffi.Bodies(), _ffi.Rows(), _ffi.Step()
        self._lib.bw_bodies_view(self._w, C.byref(B))
        self._lib.bw_rows_view(self._w, C.byref(R))
        self._lib.bw_step_params(self._w, C.byref(S))
        return B, R, S

    # -- reading -----------------------------------------------------------------------------
    @property
    def transforms(self) -> np.ndarray:
        """World.transforms: 7 float32 per slot, position then rotation x y z w (a copy)."""
        ptr = self._lib.bw_transforms(self._w)
        return np.ctypeslib.as_array(ptr, shape=(7 * self._count,)).copy()

    @property
    def workers(self):
        """World.workers (src/world.js:501-524): the threads besides the caller's that the step's
        host side uses for its walk over the pairs ('auto': the machine's cores, up to 16).  The solve stage
        runs on the GPU whatever it is; as in the reference, results do not depend on it."""
        if not self._w:
            raise BearingError("workers: this world was destroyed")
        return self._workers

    @workers.setter
    def workers(self, value):
        if not self._w:
            raise BearingError("workers: this world was destroyed")
        try:
            self._workers = _workers("world.workers", value)
        except check.CheckError as e:
            raise BearingError(str(e)) from None
        self._lib.bw_set_workers(self._w, -1 if value == "auto" else min(value, 1 << 20))

    def stats(self) -> dict:
        st = _ffi.Stats()
        self._lib.bw_stats_get(self._w, C.byref(st))
        return {k: getattr(st, k) for k, _ in _ffi.Stats._fields_}

    def state(self) -> dict:
        """Every FP64 body column the solve stage writes, by slot (copies): position, rotation,
        velocity, angular, the tumble state (tumbled, ceiling), the step's start pose (start,
        start_q) and the world inverse inertia (inv_i)."""
        B, _, _ = self.views()
        n = self._count
        def arr(p, k):
            return np.ctypeslib.as_array(p, shape=(k * n,)).copy() if n else np.zeros(0)
        return {"position": arr(B.position, 3), "rotation": arr(B.rotation, 4),
                "velocity": arr(B.velocity, 3), "angular": arr(B.angular, 3),
                "tumbled": arr(B.tumbled, 3), "ceiling": arr(B.ceiling, 1), "start": arr(B.start, 3),
                "start_q": arr(B.start_q, 4), "inv_i": arr(B.inv_i, 6)}

    def contacts(self) -> dict:
        """The last step's manifolds as the solve stage left them (copies, in colour order): the
        impulses, drift, gaps, max impulses and relative velocities."""
        _, R, _ = self.views()
        n = R.count
        def arr(p, k):
            return np.ctypeslib.as_array(p, shape=(k * n,)).copy() if n else np.zeros(0)
        return {"normal_impulse": arr(R.normal_impulse, 4), "tangent_impulse1": arr(R.tangent_impulse1, 1),
                "tangent_impulse2": arr(R.tangent_impulse2, 1), "roll_impulse1": arr(R.roll_impulse1, 1),
                "roll_impulse2": arr(R.roll_impulse2, 1), "spin_impulse": arr(R.spin_impulse, 1),
                "drift1": arr(R.drift1, 1), "drift2": arr(R.drift2, 1), "gap": arr(R.gap, 1),
                "max_normal_impulse": arr(R.max_normal_impulse, 4),
                "relative_velocity": arr(R.relative_velocity, 4)}

    def destroy(self):
        if self._w:
            self._lib.bw_destroy(self._w)
            self._w = None
        if isinstance(self._solver, GpuSolver):
            self._solver.close()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class Batch:
    """Many independent worlds stepped together: each world's host side on CPU threads, then one
    launch solves every world's stage on the GPU, one CTA a world (bg_batch_solve_step)."""

    def __init__(self, worlds, device: int = 0, threads: int | None = None):
        import os as _os
        self.worlds = list(worlds)
        self._lib = _ffi.host()
        self._gpu = _ffi.gpu()
        arr = (C.c_void_p * len(self.worlds))(*[w._w for w in self.worlds])
        self._b = self._lib.bw_batch_create(arr, len(self.worlds))
        if not self._b:
            raise BearingError("Batch: no worlds")
        self.ctx = self._gpu.bg_create(device, 0)
        if not self.ctx:
            raise BearingError(f"bg_create({device}) failed: no usable CUDA device")
        try:
            affinity = len(_os.sched_getaffinity(0))   # the CPUs this process may run on
        except AttributeError:
            affinity = _os.cpu_count() or 1
        self.threads = threads or max(1, affinity)

    def begin_step(self, dt: float):
        rc = self._lib.bw_batch_begin_step(self._b, float(dt), self.threads)
        if rc != 0:
            raise BearingError(f"batch step failed ({rc})")

    def views(self):
        B, R, W, S = _ffi.Bodies(), _ffi.Rows(), _ffi.Worlds(), _ffi.Step()
        rc = self._lib.bw_batch_views(self._b, C.byref(B), C.byref(R), C.byref(W), C.byref(S))
        if rc != 0:
            raise BearingError("batch views: no step begun")
        return B, R, W, S

    def end_step(self):
        rc = self._lib.bw_batch_end_step(self._b, self.threads)
        if rc != 0:
            raise BearingError(f"batch end step failed ({rc})")

    def step(self, dt: float):
        """One step of every world: host sides, one batched GPU launch, host sides again."""
        self.begin_step(dt)
        B, R, W, S = self.views()
        rc = self._gpu.bg_batch_solve_step(self.ctx, C.byref(B), C.byref(R), C.byref(W), C.byref(S))
        if rc != 0:
            raise BearingError(f"batched solve failed ({rc}): {self._gpu.bg_last_error(self.ctx).decode()}")
        self.end_step()

    def destroy(self):
        if self._b:
            self._lib.bw_batch_destroy(self._b)
            self._b = None
        if self.ctx:
            self._gpu.bg_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
