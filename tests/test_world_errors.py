"""The World API's refusals, word for word as the reference's own error tests have them
(test/errors.test.js:76-84, 104-178, 329-330, 406-420), for what this path covers: the World's
options, addBody's for boxes, spheres and capsules, step's dt, a destroyed world, and a call that
throws changing nothing.  What the reference takes but this path does not cover (hulls and the
other shapes, characters, sensors, layers, locks, given inertia) is refused with a message that
says so."""
import math

import pytest

import oracle_io
from bearing_b200.world import BearingError, World

OPTIONS = ("type, shape, size, radius, height, vertices, indices, heights, columns, spacing, parts, density, mass, "
           "inertia, centerOfMass, friction, restitution, damping, angularDamping, gravityScale, layers, mask, "
           "sensor, lockRotation, maxSlope, stepHeight, position, rotation, velocity, angularVelocity")


def fresh():
    return World({}, solver=oracle_io.solver(0))


def message(call):
    with pytest.raises(BearingError) as e:
        call()
    return str(e.value)


WORLD_CASES = [
    (5, "World: options must be an object, got 5"),
    ({"gravty": [0, 0, 0]}, "World: unknown option 'gravty' (did you mean 'gravity'?)"),
    ({"wind": 1}, "World: unknown option 'wind' (the options are gravity, substeps, sleeping, workers)"),
    ({"gravity": [0, -9.81]}, "World: gravity must be 3 finite numbers, got 0,-9.81"),
    ({"substeps": 0}, "World: substeps must be a whole number, 1 or more, got 0"),
    ({"sleeping": 0}, "World: sleeping must be true or false, got 0"),
    ({"workers": -1}, "World: workers must be 'auto' or a whole number, 0 or more, got -1"),
]


@pytest.mark.parametrize("options,text", WORLD_CASES)
def test_world_options(options, text):
    assert message(lambda: World(options, solver=oracle_io.solver(0))) == text


ADD_BODY_CASES = [
    ("box", "addBody: options must be an object, got 'box'"),
    ({"postion": [0, 0, 0]}, "addBody: unknown option 'postion' (did you mean 'position'?)"),
    ({"Mass": 5}, "addBody: unknown option 'Mass' (did you mean 'mass'?)"),
    ({"banana": 1}, f"addBody: unknown option 'banana' (the options are {OPTIONS})"),
    ({"type": "fixed"}, "addBody: type must be 'dynamic', 'static', 'kinematic' or 'character', got 'fixed'"),
    ({"maxSlope": 0.5}, "addBody: a dynamic body has no maxSlope"),
    ({"shape": "cube"}, "addBody: shape must be 'box', 'sphere', 'capsule', 'hull', 'compound', 'mesh' or "
                        "'heightfield', got 'cube'"),
    ({"shape": "heightfield", "type": "character"},
     "addBody: type must be 'static' or 'kinematic' for a heightfield, got 'character'"),
    ({"shape": "hull", "type": "character"}, "addBody: type must be 'dynamic', 'static' or 'kinematic' for a hull, "
                                             "got 'character'"),
    ({"radius": 0.5}, "addBody: a box has no radius"),
    ({"shape": "sphere", "height": 2}, "addBody: a sphere has no height"),
    ({"size": [1, 0, 1]}, "addBody: size must be 3 positive numbers, got 1,0,1"),
    ({"shape": "sphere", "radius": -2}, "addBody: radius must be a positive number, got -2"),
    ({"shape": "capsule", "height": "2"}, "addBody: height must be a positive number, got '2'"),
    ({"shape": "capsule", "height": 0.8}, "addBody: height must be at least twice radius (1), got 0.8"),
    ({"mass": 1, "density": 1}, "addBody: give mass or density, not both"),
    ({"mass": 0}, "addBody: mass must be a positive number, got 0"),
    ({"density": math.inf}, "addBody: density must be a positive number, got Infinity"),
    ({"friction": -0.1}, "addBody: friction must be 0 or more, got -0.1"),
    ({"restitution": 1.2}, "addBody: restitution must be from 0 to 1, got 1.2"),
    ({"damping": math.nan}, "addBody: damping must be 0 or more, got NaN"),
    ({"angularDamping": math.inf}, "addBody: angularDamping must be 0 or more, got Infinity"),
    ({"gravityScale": "1"}, "addBody: gravityScale must be a finite number, got '1'"),
    ({"position": {"x": 1, "y": 2, "z": 3}}, "addBody: position must be 3 finite numbers, got an object"),
    ({"rotation": [0, 0, 0, 0]}, "addBody: rotation must be 4 finite numbers, not all zero, got 0,0,0,0"),
    ({"type": "static", "velocity": [0, 0, 0]}, "addBody: a static body has no velocity"),
    ({"velocity": [1, 2]}, "addBody: velocity must be 3 finite numbers, got 1,2"),
    ({"angularVelocity": None}, "addBody: angularVelocity must be 3 finite numbers, got null"),
]


@pytest.mark.parametrize("spec,text", ADD_BODY_CASES)
def test_add_body(spec, text):
    assert message(lambda: fresh().addBody(spec)) == text


@pytest.mark.parametrize("spec,what", [({"shape": "hull"}, "a hull"), ({"shape": "mesh", "type": "static"}, "a mesh"),
                                       ({"type": "character"}, "a character body"), ({"sensor": True}, "sensor"),
                                       ({"layers": 3}, "layers"), ({"lockRotation": [True, False, False]}, "lockRotation"),
                                       ({"inertia": [1, 1, 1]}, "inertia given")])
def test_what_this_path_does_not_cover_is_refused_saying_so(spec, what):
    assert message(lambda: fresh().addBody(spec)).startswith(f"addBody: {what} is not on this path")


def test_step_and_a_destroyed_world():
    w = fresh()
    assert message(lambda: w.step(0)) == "step: dt must be a positive number of seconds, got 0"
    w.destroy()
    assert message(lambda: w.step(1 / 60)) == "step: this world was destroyed"
    assert message(lambda: w.addBody({})) == "addBody: this world was destroyed"
    assert message(lambda: w.workers) == "workers: this world was destroyed"
    w = fresh()
    with pytest.raises(BearingError) as e:
        w.workers = "all"
    assert str(e.value) == "world.workers must be 'auto' or a whole number, 0 or more, got 'all'"


def test_a_call_that_throws_changes_nothing():
    w = fresh()
    w.addBody({"position": (1.0, 2.0, 3.0), "velocity": (4.0, 5.0, 6.0)})
    before = {k: v.tobytes() for k, v in w.state().items()}
    for bad in ({"position": (0.0, 0.0, 0.0), "radius": 1}, {"mass": 5, "velocity": [1, 2]},
                {"shape": "sphere", "radius": 1, "height": 3}):
        with pytest.raises(BearingError):
            w.addBody(bad)
    assert w._count == 1
    assert {k: v.tobytes() for k, v in w.state().items()} == before
