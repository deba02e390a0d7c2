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


def affected_positions(surface, layer_idx):
    """World positions of the affected() leaves in one layer, via the list accessors."""
    _, ccount, _ = surface.partitions()
    D = len(surface.size)
    out = []
    for p in surface.affected_partitions(layer_idx):
        # children index -> zero-based child coordinates (row-major, last axis fastest)
        c, r = [0] * D, p
        for a in range(D - 1, -1, -1):
            c[a] = r % ccount[a]
            r //= ccount[a]
        # grid offset -size/2 truncates toward zero (Surface.hpp:1716-1719)
        org = [c[a] * surface.part[a] + int(-surface.size[a] / 2) for a in range(D)]
        for leaf in surface.affected_list(p, layer_idx):
            q, r = [0] * D, leaf
            for a in range(D - 1, -1, -1):
                q[a] = r % surface.part[a]
                r //= surface.part[a]
            out.append([org[a] + q[a] for a in range(D)])
    return out


def child_index(pos_child, ccount, coff):
    """Row-major index of a child position in the children grid (last axis fastest)."""
    idx = 0
    for a in range(len(pos_child)):
        v = pos_child[a] - coff[a]
        for b in range(a + 1, len(pos_child)):
            v *= ccount[b]
        idx += v
    return idx
