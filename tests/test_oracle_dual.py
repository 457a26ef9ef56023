"""The adjoint's checker, pinned on the CPU: the oracle's dual-number run of a world (narrowphase,
emit, basis, carry, solve stage and keep in dual numbers, oracle_dual_*).

* Its real part is the double run: a tower world stepped 40 times (through the ball's impact)
  has the same FP64 state, bit for bit, as the same world stepped by the oracle's double stage.
* Its derivatives are the derivatives: where no decision of the step changes for a small change
  of the parameters (a box sliding on the ground), they agree with central differences of the
  double run (h = 1e-6) to 1e-6 relative.
"""
import numpy as np

import oracle_io
from bearing_b200 import scenes
from bearing_b200.world import World

DT = 1 / 60


def test_the_dual_run_is_the_double_run():
    rng_seed = (5000, 2)
    a = World({}, solver=oracle_io.solver(0))
    _, info = scenes.tower(a, scenes.batch_rng(*rng_seed))
    b = World({}, solver=oracle_io.solver(0))
    scenes.tower(b, scenes.batch_rng(*rng_seed))
    dual = oracle_io.DualWorld(a, info["friction"], info["restitution"], info["ball"])
    for i in range(40):
        dual.step(DT)
        b.step(DT)
        sa, sb = a.state(), b.state()
        for k in ("position", "rotation", "velocity", "angular"):
            assert sa[k].tobytes() == sb[k].tobytes(), f"step {i + 1}: {k}"
    v, _ = dual.pose(info["ball"])
    assert v[2] > -3.0   # the ball has reached the tower
    dual.close()


def sliding(mu, e, vel):
    w = World({}, solver=oracle_io.solver(0))
    w.addBody({"type": "static", "size": (40.0, 1.0, 40.0), "position": (0.0, -0.5, 0.0), "friction": mu,
               "restitution": e})
    box = w.addBody({"size": (0.5, 0.5, 0.5), "position": (0.0, 0.25, 0.0), "velocity": tuple(vel), "friction": mu,
                     "restitution": e})
    return w, box


def test_dual_numbers_agree_with_central_differences():
    mu, e, vel, steps = 0.3, 0.2, np.array([2.0, 0.0, 1.0]), 20
    w, box = sliding(mu, e, vel)
    dual = oracle_io.DualWorld(w, mu, e, box)
    for _ in range(steps):
        dual.step(DT)
    v, tan = dual.pose(box)
    grad = 2 * v[:3] @ tan[:3]
    dual.close()
    h = 1e-6
    fd = np.zeros(5)
    for k in range(5):
        losses = []
        for sg in (1, -1):
            m2, e2, v2 = mu, e, vel.copy()
            if k == 0:
                m2 += sg * h
            elif k == 1:
                e2 += sg * h
            else:
                v2[k - 2] += sg * h
            w2, b2 = sliding(m2, e2, v2)
            for _ in range(steps):
                w2.step(DT)
            losses.append(float(np.sum(w2.state()["position"][3 * b2: 3 * b2 + 3] ** 2)))
        fd[k] = (losses[0] - losses[1]) / (2 * h)
    assert np.allclose(grad, fd, rtol=1e-6, atol=1e-9), (grad, fd)
    assert abs(grad[0]) > 0.1 and abs(grad[2]) > 0.1   # friction and the launch matter here
