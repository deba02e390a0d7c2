"""Replays golden-fixture step lists on any Surface-like object (oracle or device engine)."""


def run_steps(surface, steps):
    for st in steps:
        op = st[0]
        if op == "seed":
            surface.seed(st[1])
        elif op == "update":
            surface.update(c=st[1])
        elif op == "update_start":
            surface.update_start()
        elif op == "delta":
            surface.delta(st[1], st[2])
        elif op == "update_end":
            surface.update_end()
        elif op == "update_bounded":
            surface.update_bounded(st[1], st[2], c=st[3])
        else:
            raise ValueError(op)


def child_index(pos_child, ccount, coff):
    """Row-major index of a child position in the children grid (last axis fastest)."""
    idx = 0
    for a in range(len(pos_child)):
        v = pos_child[a] - coff[a]
        for b in range(a + 1, len(pos_child)):
            v *= ccount[b]
        idx += v
    return idx
