"""The narrowphase (bearing_b200/host/collide_impl.hpp, the same source the device compiles for
bg_collide) held to the reference's own narrowphase tests, test/collide.test.js: its hand-worked
cases for every pair of shapes (61-198) and its properties over seeded random pairs (310-470):
agreement with a brute-force signed distance that shares no code with the narrowphase, points
midway between the surfaces, the normal turning round when a and b swap, a box point keeping its
id whichever face is the reference, continuity under a small move, and the same contact twice.

The shapes are made as the test makes them: its make(), and its random pairs from its linear
congruential generator at seed 2026 in its own order and double arithmetic, so every random pair
here is one the reference's tests check (the brute-force comparison on the first 120 of its 600
pairs of each kind, the others on all of theirs).  They are collided through bw_collide_pairs,
two slots a pair, with no gravity, so no shape has a weight for reducePoints to lean on."""
import ctypes as C
import math

import numpy as np

from bearing_b200 import _ffi

P = _ffi.BG_POINTS
EPS = 1e-9
MARGIN, TOLERANCE = 0.02, 0.005
REF = 1e-7
KIND = {"box": _ffi.BG_BOX, "sphere": _ffi.BG_SPHERE, "capsule": _ffi.BG_CAPSULE}


def turn(axis, radians):
    a = np.asarray(axis, float)
    a = a / np.linalg.norm(a)
    s = math.sin(radians / 2)
    return (a[0] * s, a[1] * s, a[2] * s, math.cos(radians / 2))


def make(shape="box", size=(1.0, 1.0, 1.0), radius=0.5, height=2.0, position=(0.0, 0.0, 0.0),
         rotation=(0.0, 0.0, 0.0, 1.0)):
    if shape == "box":
        dims = tuple(float(x) for x in size)
    elif shape == "sphere":
        dims = (float(radius), 0.0, 0.0)
    else:
        dims = (float(radius), float(height), 0.0)
    return {"kind": shape, "dims": dims, "position": tuple(float(x) for x in position),
            "rotation": tuple(float(x) for x in rotation)}


def collide_many(pairs, margin=0.2, tolerance=0.005):
    """Each (a, b) through bw_collide_pairs: (count, normal, points [(p, s, id)])."""
    n = len(pairs)
    nb = 2 * n
    pos = np.zeros(3 * nb); rot = np.zeros(4 * nb); dims = np.zeros(3 * nb)
    shape = np.zeros(nb, np.uint8); typ = np.zeros(nb, np.uint8); gs = np.ones(nb)
    for i, (a, b) in enumerate(pairs):
        for j, s in enumerate((a, b)):
            k = 2 * i + j
            pos[3 * k:3 * k + 3] = s["position"]; rot[4 * k:4 * k + 4] = s["rotation"]
            dims[3 * k:3 * k + 3] = s["dims"]; shape[k] = KIND[s["kind"]]
    B = _ffi.Bodies()
    B.capacity = nb
    pd = C.POINTER(C.c_double)
    B.position, B.rotation, B.dims = pos.ctypes.data_as(pd), rot.ctypes.data_as(pd), dims.ctypes.data_as(pd)
    B.gravity_scale = gs.ctypes.data_as(pd)
    B.shape = shape.ctypes.data_as(C.POINTER(C.c_uint8))
    B.type = typ.ctypes.data_as(C.POINTER(C.c_uint8))
    a = np.arange(0, nb, 2, dtype=np.int32); b = a + 1
    mg = np.full(n, float(margin)); tl = np.full(n, float(tolerance))
    L = _ffi.Pairs(n, a.ctypes.data_as(C.POINTER(C.c_int32)), b.ctypes.data_as(C.POINTER(C.c_int32)),
                   mg.ctypes.data_as(pd), tl.ctypes.data_as(pd))
    points = np.zeros(n, np.uint8); normal = np.zeros(3 * n); point = np.zeros(3 * P * n)
    sep = np.zeros(P * n); pid = np.zeros(P * n, np.uint32)
    out = _ffi.Manifolds(points.ctypes.data_as(C.POINTER(C.c_uint8)), normal.ctypes.data_as(pd),
                         point.ctypes.data_as(pd), sep.ctypes.data_as(pd), pid.ctypes.data_as(C.POINTER(C.c_uint32)))
    g = np.zeros(3)
    assert _ffi.host().bw_collide_pairs(C.byref(B), g.ctypes.data_as(pd), C.byref(L), C.byref(out), 4) == 0
    res = []
    for i in range(n):
        c = int(points[i])
        res.append((c, normal[3 * i:3 * i + 3].copy(),
                    [(point[3 * (P * i + k):3 * (P * i + k) + 3].copy(), float(sep[P * i + k]), int(pid[P * i + k]))
                     for k in range(c)]))
    return res


def run(a, b, margin=0.2, tolerance=0.005):
    return collide_many([(a, b)], margin, tolerance)[0]


def near(a, b, what, eps=EPS):
    for x, y in zip(np.atleast_1d(a), np.atleast_1d(b)):
        assert abs(x - y) <= eps, f"{what}: {x} vs {y}"


def same_points(got, expected, what):
    assert len(got) == len(expected), f"{what}: {len(got)} points, expected {len(expected)}"
    left = list(got)
    for p, s in expected:
        hit = [i for i, g in enumerate(left) if np.linalg.norm(g[0] - np.asarray(p)) < 1e-9]
        assert hit, f"{what}: no point at {p}; got {[tuple(np.round(g[0], 4)) for g in got]}"
        near(left[hit[0]][1], s, f"{what} separation at {p}")
        left.pop(hit[0])


# ---- hand-worked cases (test/collide.test.js:61-198) ----

def test_sphere_and_sphere():
    a = make("sphere", radius=1)
    c, n, pts = run(a, make("sphere", radius=0.5, position=(2, 0, 0)), 1)
    near(n, [1, 0, 0], "normal")
    same_points(pts, [((1.25, 0, 0), 0.5)], "within margin")
    assert run(a, make("sphere", radius=0.5, position=(3, 0, 0)), 0.5)[0] == 0
    same_points(run(a, make("sphere", radius=0.5, position=(1.2, 0, 0)))[2], [((0.85, 0, 0), -0.3)], "overlapping")
    c, n, pts = run(a, make("sphere", radius=0.5))
    near(n, [0, 1, 0], "concentric normal")
    same_points(pts, [((0, 0.25, 0), -1.5)], "concentric")


def test_sphere_and_box():
    box = make(size=(2, 2, 2))
    c, n, pts = run(make("sphere", position=(0, 1.6, 0)), box)
    near(n, [0, -1, 0], "face normal")
    same_points(pts, [((0, 1.05, 0), 0.1)], "face")
    c, n, pts = run(make("sphere", position=(1.3, 1.3, 0)), box)
    near(n, [-math.sqrt(0.5), -math.sqrt(0.5), 0], "edge normal")
    near(pts[0][1], 0.3 * math.sqrt(2) - 0.5, "edge separation")
    near(run(make("sphere", position=(1.2, 1.2, 1.2)), box)[2][0][1], 0.2 * math.sqrt(3) - 0.5, "corner separation")
    c, n, pts = run(make("sphere", position=(0, 0.9, 0)), box)
    near(n, [0, -1, 0], "inside normal")
    same_points(pts, [((0, 0.7, 0), -0.6)], "inside")
    c, n, pts = run(box, make("sphere", position=(0, 1.6, 0)))
    near(n, [0, 1, 0], "box first")
    same_points(pts, [((0, 1.05, 0), 0.1)], "box first")
    same_points(run(make("sphere", position=(0, 1.6, 0)), make(size=(2, 2, 2), rotation=turn((0, 1, 0), 0.7)))[2],
                [((0, 1.05, 0), 0.1)], "turned box")


def test_sphere_and_capsule():
    capsule = make("capsule", radius=0.5, height=2)
    c, n, pts = run(make("sphere", position=(1.2, 0, 0)), capsule)
    near(n, [-1, 0, 0], "beside normal")
    same_points(pts, [((0.6, 0, 0), 0.2)], "beside")
    c, n, pts = run(make("sphere", position=(0, 1.8, 0)), capsule, 0.5)
    near(n, [0, -1, 0], "past the end normal")
    same_points(pts, [((0, 1.15, 0), 0.3)], "past the end")
    c, n, pts = run(make("sphere", position=(0, 0, 0)), capsule)
    near(n, [0, 0, -1], "on the axis normal")
    near(pts[0][1], -1, "on the axis separation")


def test_capsule_and_capsule():
    a = make("capsule")
    c, n, pts = run(a, make("capsule", position=(1.1, 0, 0)))
    near(n, [1, 0, 0], "side by side normal")
    same_points(pts, [((0.55, -0.5, 0), 0.1), ((0.55, 0.5, 0), 0.1)], "side by side")
    same_points(run(a, make("capsule", position=(1.1, 0, 0), rotation=turn((1, 0, 0), math.pi / 2)))[2],
                [((0.55, 0, 0), 0.1)], "crossed")
    c, n, pts = run(a, make("capsule", position=(0, 2.1, 0)))
    near(n, [0, 1, 0], "end to end normal")
    same_points(pts, [((0, 1.05, 0), 0.1)], "end to end")
    same_points(run(a, make("capsule", position=(1.1, 0.6, 0)))[2], [((0.55, 0.1, 0), 0.1), ((0.55, 0.5, 0), 0.1)],
                "half alongside")


def test_capsule_and_box():
    box = make(size=(4, 1, 4))
    lying = turn((0, 0, 1), -math.pi / 2)
    c, n, pts = run(make("capsule", position=(0, 1.1, 0), rotation=lying), box)
    near(n, [0, -1, 0], "lying normal")
    same_points(pts, [((-0.5, 0.55, 0), 0.1), ((0.5, 0.55, 0), 0.1)], "lying")
    same_points(run(make("capsule", position=(0, 1.6, 0)), box)[2], [((0, 0.55, 0), 0.1)], "standing")
    c, n, pts = run(make("capsule", position=(2.3, 0.8, 0), rotation=turn((1, 0, 0), math.pi / 2)), box)
    near(n, [-math.sqrt(0.5), -math.sqrt(0.5), 0], "edge normal")
    assert c == 1
    near(pts[0][1], 0.3 * math.sqrt(2) - 0.5, "edge separation")
    c, n, pts = run(make("capsule", radius=0.3, height=6, position=(0, 0.3, 0), rotation=lying), box)
    near(n, [0, -1, 0], "through normal")
    same_points(pts, [((-2, 0.25, 0), -0.5), ((2, 0.25, 0), -0.5)], "through")


def test_box_and_box_stacked_small_on_large_turned_edges_corner():
    a = make(size=(2, 2, 2))
    c, n, pts = run(a, make(size=(2, 2, 2), position=(0, 2.1, 0)))
    near(n, [0, 1, 0], "stacked normal")
    same_points(pts, [((-1, 1.05, -1), 0.1), ((1, 1.05, -1), 0.1), ((1, 1.05, 1), 0.1), ((-1, 1.05, 1), 0.1)], "stacked")
    big, small = make(size=(4, 1, 4)), make(size=(1, 1, 1), position=(0, 1, 0))
    corners = [(-0.5, 0.5, -0.5), (0.5, 0.5, -0.5), (0.5, 0.5, 0.5), (-0.5, 0.5, 0.5)]
    c, n, pts = run(big, small)
    near(n, [0, 1, 0], "small on large")
    same_points(pts, [(p, 0) for p in corners], "small on large")
    c, n, pts = run(small, big)
    near(n, [0, -1, 0], "large under small")
    same_points(pts, [(p, 0) for p in corners], "large under small")
    c, n, pts = run(a, make(size=(2, 2, 2), position=(0, 2.05, 0), rotation=turn((0, 1, 0), math.pi / 4)))
    near(n, [0, 1, 0], "turned normal")
    assert c == 4
    for p, s, _ in pts:
        near(s, 0.05, "turned separation")
        assert abs(p[0]) <= 1 + EPS and abs(p[2]) <= 1 + EPS
    ridge = math.sqrt(2)
    c, n, pts = run(make(size=(2, 2, 2), rotation=turn((0, 0, 1), math.pi / 4)),
                    make(size=(2, 2, 2), position=(0, 2.8, 0), rotation=turn((1, 0, 0), math.pi / 4)))
    near(n, [0, 1, 0], "edges normal")
    same_points(pts, [((0, 1.4, 0), 2.8 - 2 * ridge)], "edges")
    up = np.ones(3) / math.sqrt(3)
    corner = turn((up[2], 0, -up[0]), math.acos(up[1]) + math.pi)
    c, n, pts = run(big, make(size=(1, 1, 1), position=(0, 0.5 + math.sqrt(3) / 2 + 0.01, 0), rotation=corner), 0.05)
    assert c == 1, "corner down: one point"
    near(pts[0][1], 0.01, "corner down separation", 1e-12)
    near(pts[0][0], [0, 0.505, 0], "corner down point", 1e-12)


def test_box_and_box_deep_same_place_apart():
    a = make(size=(2, 2, 2))
    c, n, pts = run(a, make(size=(2, 2, 2), position=(0, 0.5, 0)))
    near(n, [0, 1, 0], "deep normal")
    assert c == 4
    for _, s, _ in pts:
        near(s, -1.5, "deep separation")
    c, n, pts = run(a, make(size=(2, 2, 2)))
    near(n, [1, 0, 0], "same place normal")
    assert c == 4
    assert run(a, make(size=(2, 2, 2), position=(0, 2.3, 0)), 0.2)[0] == 0


def test_a_box_point_keeps_its_id_whichever_face_is_the_reference():
    a = make(size=(0.26, 0.08, 0.08))

    def at(t):
        return run(a, make(size=(0.14, 0.14, 0.44), position=(0.1, 0.108, 0.01), rotation=turn((1, 0, 0), t)), 0.01, 0.0004)
    r, s = at(0.001), at(0.003)
    near(r[1], [0, 1, 0], "the forearm's face", 0)
    assert s[1][2] > 0.002
    assert s[0] == 4
    assert sorted(p[2] for p in s[2]) == sorted(p[2] for p in r[2])
    for p in r[2]:
        q = next(q for q in s[2] if q[2] == p[2])
        near(q[0], p[0], f"point {p[2]}", 0.001)


# ---- seeded random pairs and the brute-force reference (test/collide.test.js:200-470) ----

class Lcg:
    """The test's generator, x -> (x * 1103515245 + 12345) mod 2^31, in double arithmetic as
    JavaScript does it (the product rounds once it passes 2^53), so the sequence is the test's."""

    def __init__(self, seed):
        self.x = float(seed)

    def __call__(self):
        self.x = (self.x * 1103515245.0 + 12345.0) % 2147483648.0
        return self.x / 2147483648.0


def random_shape(rnd, kind):
    q = np.array([rnd() - 0.5, rnd() - 0.5, rnd() - 0.5, rnd() - 0.5])
    q /= math.sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3])
    position = (rnd() * 2 - 1, rnd() * 2 - 1, rnd() * 2 - 1)
    if kind == "box":
        return make(size=(0.3 + rnd() * 1.5, 0.3 + rnd() * 1.5, 0.3 + rnd() * 1.5), position=position, rotation=q)
    if kind == "sphere":
        return make("sphere", radius=0.15 + rnd() * 0.6, position=position, rotation=q)
    radius = 0.15 + rnd() * 0.4
    return make("capsule", radius=radius, height=2 * radius + rnd() * 1.5, position=position, rotation=q)


KINDS = ["sphere", "capsule", "box"]
PAIRS = [(KINDS[i], KINDS[j]) for i in range(3) for j in range(i, 3)]


def axes_of(s):
    x, y, z, w = s["rotation"]
    return np.array([1 - 2 * (y * y + z * z), 2 * (x * y + z * w), 2 * (x * z - y * w),
                     2 * (x * y - z * w), 1 - 2 * (x * x + z * z), 2 * (y * z + x * w),
                     2 * (x * z + y * w), 2 * (y * z - x * w), 1 - 2 * (x * x + y * y)])


def half_of(s):
    d = s["dims"]
    if s["kind"] == "box":
        return np.array([d[0] / 2, d[1] / 2, d[2] / 2])
    if s["kind"] == "sphere":
        return np.array([d[0], 0, 0])
    return np.array([d[0], (d[1] - 2 * d[0]) / 2, 0])


def reach(s, n):
    """Support function along unit directions n (k x 3)."""
    c, x, h = np.asarray(s["position"]), axes_of(s), half_of(s)
    r = n @ c
    if s["kind"] == "sphere":
        return r + h[0]
    if s["kind"] == "capsule":
        return r + h[0] + h[1] * np.abs(n @ x[3:6])
    return r + sum(h[i] * np.abs(n @ x[3 * i:3 * i + 3]) for i in range(3))


def gap(a, b, n):
    return -reach(b, -n) - reach(a, n)


def kinks(s):
    x = axes_of(s)
    if s["kind"] == "sphere":
        return []
    if s["kind"] == "capsule":
        return [x[3:6]]
    return [x[0:3], x[3:6], x[6:9]]


def reference(a, b):
    """The largest gap along any direction (the test's brute force, vectorised)."""
    N = 2000
    golden = math.pi * (3 - math.sqrt(5))
    i = np.arange(N)
    y = 1 - (2 * i + 1) / N
    r = np.sqrt(1 - y * y)
    t = golden * i
    dirs = np.stack([np.cos(t) * r, y, np.sin(t) * r], 1)
    g = gap(a, b, dirs)
    k = int(np.argmax(g))
    best, bdir = float(g[k]), dirs[k]
    rnd = Lcg(99)
    step = 0.05
    while step > 1e-10:
        for _ in range(40):   # each step from the best so far, as the test's loop takes them
            cand = bdir + step * np.array([rnd() - 0.5, rnd() - 0.5, rnd() - 0.5])
            cand /= math.sqrt(cand @ cand)
            gv = float(gap(a, b, cand[None])[0])
            if gv > best:
                best, bdir = gv, cand
        step *= 0.5
    axes = kinks(a) + kinks(b)
    for kk in axes:
        u = np.cross(kk, [1, 0, 0]) if abs(kk[0]) < 0.9 else np.cross(kk, [0, 1, 0])
        u /= np.linalg.norm(u)
        v = np.cross(kk, u)

        def at(tt):
            tt = np.atleast_1d(tt)
            return np.outer(np.cos(tt), u) + np.outer(np.sin(tt), v)
        ts = np.arange(720) / 720 * 2 * math.pi
        gs = gap(a, b, at(ts))
        j = int(np.argmax(gs))
        bt, bg = ts[j], float(gs[j])
        best = max(best, bg)
        step = 0.01
        while step > 1e-13:
            moved = True
            while moved:
                moved = False
                gg = gap(a, b, at([bt - step, bt + step]))
                for tt, gv in zip((bt - step, bt + step), gg):
                    if gv > bg:
                        bg, bt, moved = float(gv), tt, True
                best = max(best, bg)
            step *= 0.5
    for p in range(len(axes)):
        for q in range(p + 1, len(axes)):
            c = np.cross(axes[p], axes[q])
            if np.linalg.norm(c) < 1e-9:
                continue
            n = c / np.linalg.norm(c)
            best = max(best, float(gap(a, b, n[None])[0]), float(gap(a, b, -n[None])[0]))
    return best


def sd(s, p):
    """Signed distance from p to the shape's surface (negative inside)."""
    x, h = axes_of(s), half_of(s)
    d = np.asarray(p) - np.asarray(s["position"])
    local = np.array([d @ x[0:3], d @ x[3:6], d @ x[6:9]])
    if s["kind"] == "sphere":
        return float(np.linalg.norm(local) - h[0])
    if s["kind"] == "capsule":
        y = max(-h[1], min(h[1], local[1]))
        return float(math.hypot(local[0], local[1] - y, local[2]) - h[0])
    q = np.abs(local) - h
    return float(np.linalg.norm(np.maximum(q, 0)) + min(q.max(), 0))


_SEQUENCE = None


def reference_pairs():
    """The random pairs of the test file's five random tests, in its order from seed 2026: 600 of
    each kind for the brute-force test, 400 for the midway test, 300 for the swap test, 300 (each
    with a direction of three draws) for the continuity test, 100 for the same-twice test."""
    global _SEQUENCE
    if _SEQUENCE is None:
        rnd = Lcg(2026)
        seq = {}
        for name, count in (("brute", 600), ("midway", 400), ("swap", 300), ("move", 300), ("same", 100)):
            seq[name] = {}
            for ka, kb in PAIRS:
                pairs = []
                for _ in range(count):
                    a, b = random_shape(rnd, ka), random_shape(rnd, kb)
                    if name == "move":
                        b = dict(b, moved=(rnd() - 0.5, rnd() - 0.5, rnd() - 0.5))
                    pairs.append((a, b))
                seq[name][(ka, kb)] = pairs
        _SEQUENCE = seq
    return _SEQUENCE


def test_random_pairs_agree_with_the_brute_force_reference():
    # the first 120 of the test's 600 pairs of each kind (the brute force is slow in Python)
    for (ka, kb), pairs in reference_pairs()["brute"].items():
        pairs = pairs[:120]
        got = collide_many(pairs, MARGIN, TOLERANCE)
        touching = apart = 0
        for k, ((a, b), (c, n, pts)) in enumerate(zip(pairs, got)):
            truth = reference(a, b)
            what = f"{ka}-{kb} #{k}"
            if c == 0:
                assert truth > MARGIN - REF, f"{what}: missed a contact at {truth}"
                apart += 1
                continue
            touching += 1
            near(np.linalg.norm(n), 1, f"{what}: unit normal", 1e-12)
            deepest = min(s for _, s, _ in pts)
            assert all(s <= MARGIN + 1e-12 for _, s, _ in pts), f"{what}: a point past the margin"
            assert float(gap(a, b, n[None])[0]) >= truth - TOLERANCE - REF, f"{what}: normal"
            assert deepest >= truth - TOLERANCE - REF, f"{what}: deepest {deepest} vs {truth}"
            axes = (ka == "box" and kb == "box") or (ka == "capsule" and kb == "box" and truth <= -half_of(a)[0])
            if not axes and not (ka == "box" and kb == "box"):
                near(deepest, truth, f"{what}: deepest vs reference", REF)
            elif truth <= 0:
                near(deepest, truth, f"{what}: deepest vs reference", TOLERANCE + REF)
            else:
                assert deepest <= truth + REF, f"{what}: reported apart further than they are"
        assert touching > 10 and apart > 10, f"{ka}-{kb}: {touching} touching, {apart} apart"


def test_every_point_sits_midway_between_the_surfaces():
    for (ka, kb), pairs in reference_pairs()["midway"].items():
        got = collide_many(pairs, MARGIN, TOLERANCE)
        slack = TOLERANCE if (ka == kb == "capsule") or (ka == kb == "box") else 0
        ball_of_a = ka == "capsule" and kb == "box"
        for k, ((a, b), (c, n, pts)) in enumerate(zip(pairs, got)):
            for p, s, _ in pts:
                on_a = sd(a, p - n * s / 2)
                on_b = sd(b, p + n * s / 2)
                assert on_a <= slack + 1e-9 and on_b <= slack + 1e-9, f"{ka}-{kb} #{k}: outside"
                if not ball_of_a:
                    assert on_a >= -slack - 1e-9, f"{ka}-{kb} #{k}: inside a"
                else:
                    assert on_a >= -half_of(a)[0] - 1e-9
                assert on_b >= -slack - 1e-9, f"{ka}-{kb} #{k}: inside b"


def test_swapping_a_and_b_turns_the_normal_round_and_keeps_the_contact():
    for (ka, kb), pairs in reference_pairs()["swap"].items():
        r_all = collide_many(pairs, MARGIN, TOLERANCE)
        s_all = collide_many([(b, a) for a, b in pairs], MARGIN, TOLERANCE)
        for k, (r, s) in enumerate(zip(r_all, s_all)):
            assert (s[0] > 0) == (r[0] > 0), f"{ka}-{kb} #{k}: touching one way only"
            if r[0] == 0:
                continue
            da, db = min(p[1] for p in r[2]), min(p[1] for p in s[2])
            if ka == kb == "box":
                near(da, db, f"{ka}-{kb} #{k}: deepest", TOLERANCE + 1e-12)
                continue
            near(s[1], -r[1], f"{ka}-{kb} #{k}: normal", 1e-12)
            if ka == kb:
                near(da, db, f"{ka}-{kb} #{k}: deepest", 1e-12)
            else:
                near(sorted(p[1] for p in s[2]), sorted(p[1] for p in r[2]), f"{ka}-{kb} #{k}: separations", 1e-12)


def test_moving_a_shape_by_d_changes_the_deepest_separation_by_at_most_d():
    d = 1e-3
    for (ka, kb), pairs in reference_pairs()["move"].items():
        moved = []
        for a, b in pairs:
            v = np.asarray(b["moved"])
            b2 = dict(b)
            b2["position"] = tuple(np.asarray(b["position"]) + d * v / math.sqrt(v @ v))
            moved.append((a, b2))
        r_all, s_all = collide_many(pairs, MARGIN, TOLERANCE), collide_many(moved, MARGIN, TOLERANCE)
        slack = TOLERANCE if ka == kb == "box" else 0
        for k, (r, s) in enumerate(zip(r_all, s_all)):
            if r[0] == 0 or s[0] == 0:
                continue
            before, after = min(p[1] for p in r[2]), min(p[1] for p in s[2])
            assert abs(after - before) <= d + slack + 1e-12, f"{ka}-{kb} #{k}: jumped {after - before}"


def test_the_same_pair_gives_the_same_contact_to_the_bit():
    for pairs in reference_pairs()["same"].values():
        r, s = collide_many(pairs, MARGIN, TOLERANCE), collide_many(pairs, MARGIN, TOLERANCE)
        for x, y in zip(r, s):
            assert x[0] == y[0] and x[1].tobytes() == y[1].tobytes()
            assert all(p[0].tobytes() == q[0].tobytes() and p[1] == q[1] and p[2] == q[2] for p, q in zip(x[2], y[2]))
