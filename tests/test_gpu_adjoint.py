"""The adjoint of the solve stage on the GPU (bg_backward) and the backward pass through whole
steps (bearing_b200.adjoint), against the oracle.

* bg_backward recomputes the step before sweeping it: its results must be the oracle's, bit for
  bit (it replays from them, so any difference would be a different step).
* One step's adjoint against the oracle's dual-number derivative of the same step, by dot
  products: for random seeds y on the results and directions x on the input (moving bodies' state,
  every row input), y . (J x) from the oracle must equal (J^T y) . x from the GPU.
* The differentiable workload itself (towers struck by a ball, 120 steps, checkpoints every 20
  steps): each tower's gradient with respect to friction, restitution and the launch velocity
  against the oracle's dual-number run of the same world (1e-6 relative).
* Central differences, where the step takes no different decision for a small change of its
  parameters (a box sliding to rest on the ground): the gradient against (L(p + h) - L(p - h)) / 2h
  of the GPU's own forward steps, h = 1e-6.
"""
import ctypes as C

import numpy as np
import pytest

import oracle_io
from stage_io import BODY_COLUMNS, ROW_COLUMNS, StageCopy, first_difference
from bearing_b200 import _ffi, adjoint, scenes
from bearing_b200.world import GpuSolver, World

pytestmark = pytest.mark.gpu

DT = 1 / 60
BODY_IN = [("position", 3), ("rotation", 4), ("velocity", 3), ("angular", 3), ("tumbled", 3), ("ceiling", 1)]
ROW_SEEDED = [("normal_impulse", 4), ("tangent_impulse1", 1), ("tangent_impulse2", 1), ("roll_impulse1", 1),
              ("roll_impulse2", 1), ("spin_impulse", 1), ("drift1", 1), ("drift2", 1)]
ROW_CONST = [("normal", 3), ("t1", 3), ("t2", 3), ("friction", 1), ("restitution", 1), ("separation", 4),
             ("point", 12)]
_ctx = {}


def ctx():
    if "c" not in _ctx:
        _ctx["c"] = _ffi.gpu().bg_create(0, 0)
        assert _ctx["c"]
    return _ctx["c"]


def backward(copy, body_seed, row_seed):
    """bg_backward on one world's step; returns (the copy with the recomputed results, body
    adjoints, row adjoints)."""
    n, c = copy.capacity, copy.count
    bs = adjoint.Grads("body", n, {f: body_seed[f].copy() for f, _ in BODY_IN})
    rs = adjoint.Grads("row", c)
    for f, _ in ROW_SEEDED:
        rs[f][:] = row_seed[f]
    bg, rg = adjoint.Grads("body", n), adjoint.Grads("row", c)
    B, R, S = copy.views()
    rc = _ffi.gpu().bg_backward(ctx(), C.byref(B), C.byref(R), None, C.byref(S), C.byref(bs.s), C.byref(rs.s),
                                C.byref(bg.s), C.byref(rg.s))
    assert rc == 0, f"bg_backward: {rc} {_ffi.gpu().bg_last_error(ctx()).decode()}"
    return copy, bg, rg


def stage_input(build, steps):
    w = World({}, solver=oracle_io.solver(0))
    build(w)
    for _ in range(steps):
        w.step(DT)
    w.begin_step(DT)
    return StageCopy(w)


def tower(w):
    scenes.tower(w, scenes.batch_rng(5000, 3))


def small_pile(w):
    scenes.pile(w, count=300, seed=11, extent=8.0)


CASES = [(tower, 0), (tower, 24), (tower, 60), (scenes.pyramid, 20), (small_pile, 90)]


@pytest.mark.parametrize("build,steps", CASES, ids=["tower0", "tower24", "tower60", "pyramid20", "pile90"])
def test_backward_recomputes_the_step_bit_for_bit(build, steps):
    base = stage_input(build, steps)
    n, c = base.capacity, base.count
    zero_b = {f: np.zeros(k * max(n, 1)) for f, k in BODY_IN}
    zero_r = {f: np.zeros(k * max(c, 1)) for f, k in ROW_SEEDED}
    want = oracle_io.solve(base.copy())
    got, _, _ = backward(base.copy(), zero_b, zero_r)
    # the adjoint leaves start and start_q of bodies that are not awake unwritten, as bg_solve_step
    for f in ("start", "start_q", "inv_i"):
        got.body[f][:] = want.body[f]
    assert first_difference(want, got) is None, first_difference(want, got)


@pytest.mark.parametrize("build,steps", CASES, ids=["tower0", "tower24", "tower60", "pyramid20", "pile90"])
def test_backward_matches_the_oracles_derivative_by_dot_products(build, steps):
    base = stage_input(build, steps)
    n, c = base.capacity, base.count
    rng = np.random.default_rng(steps + 1)
    moving = (base.body["type"] == _ffi.BG_DYNAMIC) & (base.body["inv_mass"] != 0)
    y_b = {f: rng.standard_normal(k * n) * np.repeat(moving, k) for f, k in BODY_IN}
    y_r = {f: rng.standard_normal(k * c) for f, k in ROW_SEEDED}
    x_b = {f: rng.standard_normal(k * n) * np.repeat(moving, k) for f, k in BODY_IN}
    x_r = {f: rng.standard_normal(k * c) for f, k in ROW_SEEDED + ROW_CONST}
    # (J^T y) . x on the GPU
    _, bg, rg = backward(base.copy(), y_b, y_r)
    reverse = sum(float(bg[f][: k * n] @ x_b[f]) for f, k in BODY_IN)
    reverse += sum(float(rg[f][: k * c] @ x_r[f]) for f, k in ROW_SEEDED + ROW_CONST)
    # y . (J x) from the oracle's dual numbers
    j = base.copy()
    B, R, S = j.views()
    dB, dR = _ffi.Bodies(), _ffi.Rows()
    keep = {}
    pd = C.POINTER(C.c_double)
    for f, dt, per in BODY_COLUMNS:
        if dt == np.float64:
            keep["b" + f] = x_b[f].copy() if f in x_b else np.zeros(per * n)
            setattr(dB, f, keep["b" + f].ctypes.data_as(pd))
    for f, dt, per in ROW_COLUMNS:
        if dt == np.float64:
            keep["r" + f] = x_r[f].copy() if f in x_r else np.zeros(per * c)
            setattr(dR, f, keep["r" + f].ctypes.data_as(pd))
    oracle_io.lib().oracle_stage_jvp(C.byref(B), C.byref(R), C.byref(S), C.byref(dB), C.byref(dR))
    forward = sum(float(np.nan_to_num(keep["b" + f]) @ y_b[f]) for f, k in BODY_IN)
    forward += sum(float(keep["r" + f] @ y_r[f]) for f, k in ROW_SEEDED)
    assert abs(forward - reverse) <= 1e-8 * max(abs(forward), abs(reverse)), (forward, reverse)


def test_tower_gradients_match_the_dual_number_oracle():
    # Eight towers of the workload's 1,024 (worlds 0..7 of its seeds), 120 steps, checkpoints
    # every 20 steps: the backward pass against the oracle's dual-number run of each world.
    count = 8
    out = adjoint.tower_gradients(count, seed=5000, steps=120, checkpoint=20)
    for i in range(count):
        w = World({}, solver=oracle_io.solver(0))
        _, info = scenes.tower(w, scenes.batch_rng(5000, i))
        dual = oracle_io.DualWorld(w, info["friction"], info["restitution"], info["ball"])
        for _ in range(120):
            dual.step(DT)
        position = w.state()["position"]
        lo = 3 * int(sum(len(x["cubes"]) + 2 for x in out["infos"][:i]))
        assert np.array_equal(position, out["position"][lo: lo + position.size]), f"tower {i}: final state"
        loss, _ = scenes.tower_loss(position, info)
        g = np.zeros(5)
        for s, t in zip(info["cubes"], info["targets"]):
            v, tan = dual.pose(s)
            g += 2 * (v[:3] - t) @ tan[:3]
        dual.close()
        w.destroy()
        assert loss == out["losses"][i]
        err = np.max(np.abs(out["gradients"][i] - g)) / np.max(np.abs(g))
        assert err <= 1e-6, f"tower {i}: {out['gradients'][i]} vs dual {g} ({err:.2e})"


def sliding(mu, e, vel):
    w = World({}, solver=GpuSolver())
    w.addBody({"type": "static", "size": (40.0, 1.0, 40.0), "position": (0.0, -0.5, 0.0), "friction": mu,
               "restitution": e})
    box = w.addBody({"size": (0.5, 0.5, 0.5), "position": (0.0, 0.25, 0.0), "velocity": tuple(vel), "friction": mu,
                     "restitution": e})
    return w, box


def test_gradients_match_central_differences_where_no_decision_changes():
    # A box sliding on the ground, 20 steps: no contact starts, stops or changes its regime for a
    # change of 1e-6 in any parameter, so central differences converge to the gradient.
    mu, e, vel, steps = 0.3, 0.2, np.array([2.0, 0.0, 1.0]), 20
    w, box = sliding(mu, e, vel)
    w.set_solver((0, 0))
    bb = adjoint.BatchBackward([w], DT)
    try:
        bb.forward(steps, checkpoint=5)
        p = w.state()["position"]
        seed = np.zeros_like(p)
        seed[3 * box: 3 * box + 3] = 2 * p[3 * box: 3 * box + 3]
        bar, g_fr, g_re = bb.backward({"position": seed})
    finally:
        bb.close()
    grad = np.concatenate([[g_fr.sum(), g_re.sum()], bar["velocity"][3 * box: 3 * box + 3]])
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
            w2.destroy()
        fd[k] = (losses[0] - losses[1]) / (2 * h)
    assert np.allclose(grad, fd, rtol=1e-6, atol=1e-9), (grad, fd)
    w.destroy()
