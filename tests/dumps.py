"""Decoding and comparison of the canonical state dumps of fg_dump / fo_dump."""
import numpy as np


def decode(d):
    d = [int(x) for x in d]
    D, L, P = d[0], d[1], d[2]
    NL = 2 * L + 1
    i = 3
    parts = []
    for _ in range(P):
        active, bg = d[i], np.array([d[i + 1]], dtype=np.uint32).view(np.float32)[0]
        i += 2
        lists = []
        for _ in range(NL):
            n = d[i]
            lists.append(d[i + 1:i + 1 + n])
            i += 1 + n
        parts.append((active, float(bg), lists))
    plists = {}
    for which in ("iso", "delta", "status"):
        ls = []
        for _ in range(NL):
            n = d[i]
            ls.append(d[i + 1:i + 1 + n])
            i += 1 + n
        plists[which] = ls
    assert i == len(d), (i, len(d))
    return dict(D=D, L=L, parts=parts, plists=plists)


def first_difference(a, b):
    """Human-readable description of the first difference between two dumps, or None."""
    if np.array_equal(np.asarray(a), np.asarray(b)):
        return None
    A, B = decode(a), decode(b)
    if (A["D"], A["L"], len(A["parts"])) != (B["D"], B["L"], len(B["parts"])):
        return f"header differs: {A['D'], A['L'], len(A['parts'])} vs {B['D'], B['L'], len(B['parts'])}"
    for which in ("iso", "delta", "status"):
        for l, (x, y) in enumerate(zip(A["plists"][which], B["plists"][which])):
            if list(x) != list(y):
                return f"{which} partition list {l}: {list(x)[:20]} vs {list(y)[:20]}"
    for p, (x, y) in enumerate(zip(A["parts"], B["parts"])):
        if x[0] != y[0]:
            return f"partition {p} active {x[0]} vs {y[0]}"
        if x[1] != y[1]:
            return f"partition {p} background {x[1]} vs {y[1]}"
        for l, (u, v) in enumerate(zip(x[2], y[2])):
            if list(u) != list(v):
                su, sv = set(u), set(v)
                kind = "order" if su == sv else f"membership (+{sorted(su - sv)[:8]} -{sorted(sv - su)[:8]})"
                return f"partition {p} layer {l} {kind}: {list(u)[:16]} vs {list(v)[:16]}"
    return "dumps differ"
