"""The colouring's test helpers: a plain restatement of src/graph.js:105-166 (the checker), and
made-up manifold lists with static, kinematic and frozen bodies, a hub in the overflow colour and
pairs in the resting run."""
import numpy as np


def reference_colour(type_, frozen, a, b):
    """src/graph.js:105-166 restated: the greedy colours in found order, then the row order (by
    colour, then b's slot, then found order) and the colour starts."""
    n = len(a)
    any_frozen = any(int(f) != 0 for f in frozen)
    used = {}
    colour = [0] * n
    for m in range(n):
        x, y = int(a[m]), int(b[m])
        dx, dy = type_[x] == 0, type_[y] == 0
        if any_frozen:
            fx, fy = frozen[x] != 0, frozen[y] != 0
            if (fx or type_[x] == 1) and (fy or type_[y] == 1):
                colour[m] = 33
                continue
            dx = dx and not fx
            dy = dy and not fy
        held = (used.get(x, 0) if dx else 0) | (used.get(y, 0) if dy else 0)
        if held == 0xFFFFFFFF:
            colour[m] = 32
            continue
        bit = ~held & (held + 1) & 0xFFFFFFFF
        colour[m] = bit.bit_length() - 1
        if dx:
            used[x] = used.get(x, 0) | bit
        if dy:
            used[y] = used.get(y, 0) | bit
    order = sorted(range(n), key=lambda m: (colour[m], int(b[m]), m))
    counts = np.bincount(np.asarray(colour, np.int64), minlength=34)
    starts = np.zeros(35, np.int32)
    starts[1:] = np.cumsum(counts)
    return np.asarray(colour, np.int32), np.asarray(order, np.int32), starts, int(starts[33])


def made_up_manifolds(seed, nb=300, count=1500, hub_degree=40):
    rng = np.random.default_rng(seed)
    type_ = rng.choice([0, 0, 0, 0, 1, 2], nb).astype(np.uint8)
    frozen = (rng.random(nb) < 0.1).astype(np.uint8) * (type_ == 0)
    a, b = [], []
    for _ in range(count):
        x, y = rng.choice(nb, 2, replace=False)
        a.append(min(x, y))
        b.append(max(x, y))
    hub = int(np.flatnonzero(type_ == 0)[0])
    frozen[hub] = 0
    for y in rng.choice(np.flatnonzero((type_ == 0) & (np.arange(nb) != hub)), hub_degree, replace=False):
        a.append(min(hub, int(y)))
        b.append(max(hub, int(y)))
    return type_, frozen, np.asarray(a, np.int32), np.asarray(b, np.int32)
