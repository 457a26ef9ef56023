"""What comes in through the World API is checked at the call that took it, and a bad value throws
naming that call, the option, what it must be and what it got, word for word as the reference's
src/core/check.js and src/world.js resolve() (2328-2462) word them:

    addBody: radius must be a positive number, got -2

Options the reference knows that this path does not cover (hulls, compounds, meshes, heightfields,
characters, sensors, layers, locks...) are refused with a message that says so."""
from __future__ import annotations

import math
from numbers import Real


class CheckError(ValueError):
    """A refused argument; the message is the reference's."""


def fail(caller: str, message: str):
    raise CheckError(f"{caller}: {message}" if caller else message)


def js_number(x) -> str:
    """A number as JavaScript's String() writes it (whole numbers without a point; NaN, Infinity)."""
    if isinstance(x, bool):
        return "true" if x else "false"
    x = float(x)
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "Infinity" if x > 0 else "-Infinity"
    if x == int(x) and abs(x) < 1e21:
        return str(int(x))
    text = repr(x)
    if "e" in text:   # 1e-07 -> 1e-7, 1e+21 stays
        mant, exp = text.split("e")
        sign = exp[0] if exp[0] in "+-" else "+"
        exp = exp.lstrip("+-").lstrip("0") or "0"
        text = f"{mant}e{sign}{exp}"
    return text


def show(value) -> str:
    """How a bad value reads in a message (src/core/check.js:28-38): arrays as 1,NaN,0, strings quoted."""
    if isinstance(value, str):
        return f"'{value}'"
    if value is None:
        return "null"
    if isinstance(value, bool):
        return "true" if value else "false"
    if isinstance(value, Real):
        return js_number(value)
    if callable(value):
        return "a function"
    if isinstance(value, (list, tuple)) or hasattr(value, "__array__"):
        items = list(value)
        return "an empty array" if not items else ",".join(show(x) for x in items)
    return "an object"


def _is_number(x) -> bool:
    return isinstance(x, Real) and not isinstance(x, bool) and math.isfinite(float(x))


def _array_of(value, n) -> bool:
    if isinstance(value, (str, bytes, dict)) or value is None:
        return False
    try:
        return len(value) == n
    except TypeError:
        return False


def finite(caller, name, value):
    if not _is_number(value):
        fail(caller, f"{name} must be a finite number, got {show(value)}")
    return float(value)


def positive(caller, name, value):
    if not _is_number(value) or value <= 0:
        fail(caller, f"{name} must be a positive number, got {show(value)}")
    return float(value)


def at_least_zero(caller, name, value):
    """src/world.js:2696-2701."""
    if not isinstance(value, Real) or isinstance(value, bool) or not (value >= 0) or value == math.inf:
        fail(caller, f"{name} must be 0 or more, got {show(value)}")
    return float(value)


def vec3(caller, name, value):
    if not _array_of(value, 3) or not all(_is_number(value[k]) for k in range(3)):
        fail(caller, f"{name} must be 3 finite numbers, got {show(value)}")
    return tuple(float(value[k]) for k in range(3))


def positive3(caller, name, value):
    if not _array_of(value, 3) or not all(_is_number(value[k]) and value[k] > 0 for k in range(3)):
        fail(caller, f"{name} must be 3 positive numbers, got {show(value)}")
    return tuple(float(value[k]) for k in range(3))


def quat(caller, name, value):
    """Four finite numbers, not all zero (the World normalises them on the way in)."""
    if _array_of(value, 4) and all(_is_number(value[k]) for k in range(4)) and any(value[k] != 0 for k in range(4)):
        return tuple(float(value[k]) for k in range(4))
    return fail(caller, f"{name} must be 4 finite numbers, not all zero, got {show(value)}")


def one_of(caller, name, value, choices):
    if value not in choices:
        listed = [f"'{c}'" for c in choices]
        phrase = listed[0] if len(listed) == 1 else f"{', '.join(listed[:-1])} or {listed[-1]}"
        fail(caller, f"{name} must be {phrase}, got {show(value)}")
    return value


def options(caller, value, name="options"):
    if value is None:
        return {}
    if not isinstance(value, dict):
        fail(caller, f"{name} must be an object, got {show(value)}")
    return value


def _distance(a: str, b: str) -> int:
    """Optimal string alignment distance: insertions, deletions, substitutions and swaps of two
    neighbours each count one (src/core/check.js distance)."""
    d = [[0] * (len(b) + 1) for _ in range(len(a) + 1)]
    for i in range(len(a) + 1):
        d[i][0] = i
    for j in range(len(b) + 1):
        d[0][j] = j
    for i in range(1, len(a) + 1):
        for j in range(1, len(b) + 1):
            cost = 0 if a[i - 1] == b[j - 1] else 1
            d[i][j] = min(d[i - 1][j] + 1, d[i][j - 1] + 1, d[i - 1][j - 1] + cost)
            if i > 1 and j > 1 and a[i - 1] == b[j - 2] and a[i - 2] == b[j - 1]:
                d[i][j] = min(d[i][j], d[i - 2][j - 2] + 1)
    return d[len(a)][len(b)]


def nearest(typed: str, names):
    """The known name closest to a typo (case ignored, the first listed on a tie), or None when
    none is within half the typed name's length."""
    best, best_d = None, math.inf
    for name in names:
        dd = _distance(typed.lower(), name.lower())
        if dd < best_d:
            best, best_d = name, dd
    return best if best_d < len(typed) / 2 else None


def known(caller, given: dict, names):
    for key in given:
        if key in names:
            continue
        near = nearest(str(key), names)
        fail(caller, f"unknown option '{key}' (did you mean '{near}'?)" if near
             else f"unknown option '{key}' (the options are {', '.join(names)})")
