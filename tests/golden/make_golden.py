"""Extract golden vectors from the Felt reference's own Catch tests into JSON fixtures.

The reference test sources are read as text; each case names the scenario it comes from
(file:line), restates the scenario's actions as a list of steps, and takes the expected values
(dense isogrid literals, layer sizes, vertices, simplices, curvatures) from the lines cited.
Run in an environment where the reference source tree is available:

    python tests/golden/make_golden.py /path/to/felt-reference

and commit the resulting tests/golden/reference_golden.json. The tests never read the reference
tree themselves.
"""
from __future__ import annotations

import json
import os
import re
import sys

NUM = r"-?\d+(?:\.\d+)?"


def lines_of(root, rel):
    with open(os.path.join(root, rel)) as f:
        return f.read().split("\n")


def data_block(lines, start):
    """Numbers of the `... = { ... };` literal whose opening line is `start` (1-based)."""
    i = start - 1
    while not re.search(r"(data\(\)|grid) = \{", lines[i]):
        i += 1
    text = ""
    depth = 0
    first = i
    while True:
        ln = re.sub(r"//.*", "", lines[i])
        for ch in ln:
            if ch == "{":
                depth += 1
            elif ch == "}":
                depth -= 1
        text += ln + "\n"
        if depth == 0 and i > first or (depth == 0 and "}" in ln):
            break
        i += 1
    body = text[text.index("{") + 1: text.rindex("}")]
    return [float(x) for x in re.findall(NUM, body)], i + 1


def layer_checks(lines, start, end):
    """CHECK(layer_size(surface, id) == n) lines within [start, end] -> {id: n}."""
    out = {}
    for ln in lines[start - 1: end]:
        m = re.search(r"layer_size\((?:surface|surface_loaded), (-?\d+)\) == (\d+)", ln)
        if m:
            out[int(m.group(1))] = int(m.group(2))
    return out


def part_layer_checks(lines, start, end):
    out = []
    for ln in lines[start - 1: end]:
        m = re.search(r"layer_size<\d,\d>\(surface, Vec\di\(([-\d, ]+)\), (-?\d+)\)\)\s*==\s*(\d+)",
                      ln)
        if m:
            out.append([[int(x) for x in m.group(1).split(",")], int(m.group(2)),
                        int(m.group(3))])
    return out


def surface_cases(root):
    f = "src/tests/test_Surface.cpp"
    L = lines_of(root, f)
    cases = []

    def grid_case(name, at, size, part, layers, steps, grid_line, checks_to, extra=None):
        vals, end = data_block(L, grid_line)
        case = dict(name=name, ref=f"{f}:{at}", size=size, part=part, layers=layers,
                    steps=steps, grid=vals, grid_ref=f"{f}:{grid_line}-{end}",
                    layer_sizes=layer_checks(L, grid_line, checks_to))
        if extra:
            case.update(extra)
        cases.append(case)

    seed = ["seed", [0, 0]]
    upd = lambda c: ["update", c]
    grid_case("seed_9x9", "58-103", [9, 9], [3, 3], 2, [seed], 79, 102)
    grid_case("radius1_9x9", "104-158", [9, 9], [3, 3], 2, [seed, upd(-1.0)], 108, 131)
    grid_case("radius2_9x9", "180-210", [9, 9], [3, 3], 2, [seed, upd(-1.0), upd(-1.0)], 192,
              209)
    grid_case("consumed_9x9", "212-251", [9, 9], [3, 3], 2, [seed] + [upd(-1.0)] * 11, 226, 249)
    grid_case("collapse_to_seed_9x9", "254-293", [9, 9], [3, 3], 2,
              [seed, upd(-1.0), upd(1.0)], 267, 294)
    grid_case("collapse_to_nothing_9x9", "295-346", [9, 9], [3, 3], 2,
              [seed, upd(-1.0), upd(1.0), upd(1.0)], 324, 346)
    grid_case("expand_0.6_9x9", "353-389", [9, 9], [3, 3], 2, [seed, upd(-0.6)], 364, 389)
    grid_case("contract_0.6_9x9", "391-424", [9, 9], [3, 3], 2, [seed, upd(-0.6), upd(0.6)], 402,
              424)
    grid_case("contract_0.6_again_9x9", "426-459", [9, 9], [3, 3], 2,
              [seed, upd(-0.6), upd(0.6), upd(0.6)], 437, 459)
    grid_case("central_partition_deactivated_21x21", "519-580", [21, 21], [2, 2], 2,
              [seed] + [upd(-1.0)] * 5, 540, 566,
              dict(partition_active={"0,1": True, "0,-1": True, "1,0": True, "-1,0": True,
                                     "0,0": False},
                   partition_active_ref=f"{f}:569-578"))
    # Local updates (update_start / delta / update_end).
    lseed = [seed]
    grid_case("local_contract_9x9", "598-633", [9, 9], [2, 2], 2,
              lseed + [["update_start"], ["delta", [0, 0], 1.0], ["update_end"]], 608, 632)
    grid_case("local_expand_9x9", "635-666", [9, 9], [2, 2], 2,
              lseed + [["update_start"], ["delta", [0, 0], -1.0], ["update_end"]], 643, 665)
    grid_case("bounded_update_9x9", "811-880", [9, 9], [2, 2], 2,
              lseed + [["update_bounded", [-1, -1], [1, 1], -0.6]], 816, 839)
    # affected() after a local update of two zero-layer points (test_Surface.cpp:668-759):
    # per layer the set of affected leaf positions (layer 0 not checked by the reference).
    aff = {}
    for ln in L[679:704]:
        m = re.search(r"check_layers_pos\[2 \+ (-?\d+)\]", ln)
        if m:
            cur = int(m.group(1))
            aff[cur] = []
        if "//" in ln.split("Vec2i")[0] if "Vec2i" in ln else False:
            continue
        for a, b in re.findall(r"Vec2i\((-?\d+), (-?\d+)\)", re.sub(r"//.*", "", ln)):
            aff[cur].append([int(a), int(b)])
    cases.append(dict(name="affected_after_local_update_9x9", ref=f"{f}:668-759", size=[9, 9],
                      part=[2, 2], layers=2, grid=None, layer_sizes={},
                      steps=lseed + [["update_start"], ["delta", [0, 0], -1.0], ["update_end"],
                                     ["update_start"], ["delta", [0, 1], 0.3],
                                     ["delta", [1, 0], 0.3], ["update_end"]],
                      affected={k: v for k, v in aff.items() if k != 0}))
    # Layer interactions.
    two = [["seed", [-4, 0]], ["seed", [4, 0]], upd(-1.0)]
    grid_case("two_seeds_16x9", "888-932", [16, 9], [3, 3], 2, two, 911, 931,
              dict(partition_layer_sizes=part_layer_checks(L, 903, 907)))
    towards = [["update_start"], ["delta", [-3, 0], -1.0], ["delta", [3, 0], -1.0],
               ["update_end"]]
    grid_case("two_seeds_towards_16x9", "934-973", [16, 9], [3, 3], 2, two + towards, 951, 972,
              dict(partition_layer_sizes=part_layer_checks(L, 943, 947)))
    back = [["update_start"], ["delta", [-3, 1], 1.0], ["delta", [-2, 0], 1.0],
            ["delta", [-3, -1], 1.0], ["delta", [3, 1], 1.0], ["delta", [2, 0], 1.0],
            ["delta", [3, -1], 1.0], ["update_end"]]
    grid_case("two_seeds_cycle_16x9", "975-1027", [16, 9], [3, 3], 2, two + (towards + back) * 10,
              1005, 1026, dict(partition_layer_sizes=part_layer_checks(L, 997, 1001)))
    # Surface<2,3>: two diagonal seeds, local updates (test_Surface.cpp:1083-1216).
    diag = [["seed", [-2, -2]], ["seed", [2, 2]]]
    for p in ([-2, -2], [-1, -2], [0, -2]):
        diag += [["update_start"], ["delta", p, -1.0], ["update_end"]]
    diag += [["update_start"], ["delta", [1, -2], -1.0], ["delta", [2, 2], 1.0], ["update_end"],
             ["update_start"], ["delta", [1, -1], -1.0], ["update_end"]]
    grid_case("diagonal_seeds_local_12x12_L3", "1083-1216", [12, 12], [2, 2], 3, diag, 1188,
              1216)
    # 3D layer sizes.
    s3 = [["seed", [0, 0, 0]], upd(-1.0)]
    cases.append(dict(name="radius1_11cubed_L3", ref=f"{f}:1031-1052", size=[11, 11, 11],
                      part=[3, 3, 3], layers=3, steps=s3, grid=None,
                      layer_sizes=layer_checks(L, 1043, 1052)))
    local3 = [["update_start"], ["delta", [0, 1, 0], -1.0], ["update_end"], ["update_start"],
              ["delta", [0, 2, 0], 1.0], ["delta", [1, 1, 0], 1.0], ["delta", [-1, 1, 0], 1.0],
              ["delta", [0, 1, 1], 1.0], ["delta", [0, 1, -1], 1.0], ["update_end"]]
    cases.append(dict(name="local_3d_11cubed_L3", ref=f"{f}:1054-1080", size=[11, 11, 11],
                      part=[3, 3, 3], layers=3, steps=s3 + local3, grid=None,
                      layer_sizes=layer_checks(L, 1070, 1079)))
    return cases


def poly_cases(root):
    f = "src/tests/test_Poly.cpp"
    L = lines_of(root, f)
    out = []

    def vec_checks(start, end, field):
        res = []
        for ln in L[start - 1: end]:
            m = re.search(r"vtxs\(\)\[(\d+)\]\.%s == ApproxVec\(Vec\df\{([^}]*)\}\)" % field, ln)
            if m:
                res.append([int(m.group(1))] + [float(x.replace("f", "")) for x in
                                                 m.group(2).split(",")])
        return res

    def spx_checks(start, end):
        res = []
        for ln in L[start - 1: end]:
            m = re.search(r"spxs\(\)\[(\d+)\]\.idxs == \(Vec\du\{([^}]*)\}\)", ln)
            if m:
                res.append([int(m.group(1))] + [int(x) for x in m.group(2).split(",")])
        return res

    def count(start, end, what):
        """First nonzero `poly.<what>().size() == n` check within [start, end]."""
        for ln in L[start - 1: end]:
            m = re.search(r"poly\.%s\(\)\.size\(\) == (\d+)" % what, ln)
            if m and int(m.group(1)) > 0:
                return int(m.group(1))
        return None

    out.append(dict(name="poly_single_3d", ref=f"{f}:14-104", size=[9, 9, 9], part=[3, 3, 3],
                    layers=3, steps=[["seed", [0, 0, 0]], ["update", -0.4]], partition=[0, 0, 0],
                    nvtx=count(62, 76, "vtxs"), nspx=count(62, 76, "spxs"),
                    pos=vec_checks(75, 84, "pos"), norm=vec_checks(85, 92, "norm"),
                    spx=spx_checks(94, 104)))
    # 2D single poly.
    two = dict(name="poly_single_2d", ref=f"{f}:134-211", size=[9, 9], part=[3, 3], layers=3,
               partition=[0, 0])
    # steps and counts parsed from the 2D scenario text
    text = "\n".join(L[133:241])
    m = re.search(r"return (-?[\d.]+)f;", text)
    two["steps"] = [["seed", [0, 0]], ["update", float(m.group(1))]]
    two["nvtx"] = count(134, 241, "vtxs")
    two["nspx"] = count(134, 241, "spxs")
    two["pos"] = vec_checks(134, 241, "pos")
    two["spx"] = spx_checks(134, 241)
    out.append(two)
    # Polys: central partition of a 15^3 / 5^3 surface.
    m1 = re.search(r"get\(Vec3i\(0,0,0\)\)\.vtxs\(\)\.size\(\) == (\d+)", L[341])
    m2 = re.search(r"get\(Vec3i\(0,0,0\)\)\.spxs\(\)\.size\(\) == (\d+)", L[342])
    out.append(dict(name="polys_central_15cubed", ref=f"{f}:326-344", size=[15, 15, 15],
                    part=[5, 5, 5], layers=3, steps=[["seed", [0, 0, 0]], ["update", -1.0]],
                    partition=[0, 0, 0], nvtx=int(m1.group(1)), nspx=int(m2.group(1))))
    return out


def curvature_cases(root):
    f = "src/tests/test_Grid.cpp"
    L = lines_of(root, f)
    out = []
    for start, dims, want_line in [(2198, 2, 2206), (2212, 2, 2222), (2319, 3, 2350),
                                   (2356, 3, 2372), (2378, 3, 2396)]:
        vals, end = data_block(L, start)
        m = re.search(r"curv\(Vec\di\([^)]*\)\) == (" + NUM + ")", "\n".join(L[end - 1:want_line]))
        out.append(dict(ref=f"{f}:{start}-{want_line}", dims=dims, size=[3] * dims,
                        offset=[-1] * dims, background=0.0, values=vals, pos=[0] * dims,
                        curv=float(m.group(1))))
    return out


def _nums(text):
    return [float(x) for x in re.findall(NUM, text)]


def numeric_queries(lines, start, end):
    """The Numeric API calls of [start, end] and what the test expects of them: `grid.<fn>(Vec..)`
    compared with a `Vec..f(...)` or an `Approx(...)`, inside a CHECK or through a named local
    (`const ... <name> = grid.<fn>(...)`, then `CHECK(<name> == ...)`)."""
    named, out = {}, []
    call = r"grid\.(\w+)\(Vec\d([if])\(([^)]*)\)\)"
    for ln in lines[start - 1: end]:
        m = re.search(r"const \w+ (\w+) = " + call, ln)
        if m:
            named[m.group(1)] = (m.group(2), m.group(3) == "f", _nums(m.group(4)))
            continue
        m = re.search(r"CHECK\(" + call + r" == Vec\df\(([^)]*)\)\)", ln)
        if m:
            out.append(dict(fn=m.group(1), real=m.group(2) == "f", pos=_nums(m.group(3)),
                            want=_nums(m.group(4)), approx=False))
            continue
        m = re.search(r"CHECK\((\w+) == (?:Vec\df\(([^)]*)\)|Approx\((" + NUM + r")f?\))\)", ln)
        if m and m.group(1) in named:
            fn, real, pos = named[m.group(1)]
            exact = m.group(2) is not None
            out.append(dict(fn=fn, real=real, pos=pos,
                            want=_nums(m.group(2)) if exact else [float(m.group(3))],
                            approx=not exact))
    return out


def numeric_cases(root):
    """Known answers of the Numeric API on 3x3 and 3x3x3 grids (test_Grid.cpp:1993-2290): interp
    and get at real positions, gradF, gradB, gradC, grad and gradE at nodes. The grid spacing is
    1 on this path, so the dx = 2 variants after line 2290 are left out."""
    f = "src/tests/test_Grid.cpp"
    L = lines_of(root, f)

    def sets(a, b, dims):
        vals = [0.0] * 3 ** dims
        for ln in L[a - 1: b]:
            m = re.search(r"grid\.set\(Vec\di\(([^)]*)\), (" + NUM + r")f?\)", ln)
            if m:
                p = [int(x) + 1 for x in _nums(m.group(1))]
                idx = 0
                for x in p:
                    idx = idx * 3 + x
                vals[idx] = float(m.group(2))
        return vals

    out = []
    for a, b, dims, block in [(2016, 2045, 2, False), (2049, 2075, 2, False),
                              (2079, 2110, 2, False), (2138, 2151, 2, True),
                              (2153, 2166, 2, True), (2168, 2180, 2, True),
                              (2182, 2194, 2, True), (2234, 2290, 3, True)]:
        vals = data_block(L, a)[0] if block else sets(a, b, dims)
        out.append(dict(ref=f"{f}:{a}-{b}", dims=dims, size=[3] * dims, offset=[-1] * dims,
                        background=0.0, values=vals, queries=numeric_queries(L, a, b)))
    return out


def catch_leaves(lines, start, end):
    """The leaf sections (THEN) of the Catch scenario in [start, end]. Catch runs a leaf with the
    statements of every enclosing section; each leaf comes back as those statements in order
    (`actions`) and its own (`checks`). Statements on a section's header line are not read (the
    reference's tests put none there)."""
    frames = [dict(kind="ROOT", open=0, stmts=[])]
    depth, pending, out = 0, None, []
    for ln in lines[start - 1: end]:
        code = re.sub(r"//.*", "", ln)
        bare = re.sub(r'"[^"]*"', '""', code)
        m = re.search(r"\b(SCENARIO|GIVEN|WHEN|AND_WHEN|THEN)\s*\(", bare)
        if m:
            pending = dict(kind=m.group(1), open=None, stmts=[])
        elif pending is None and bare.strip() not in ("", "{", "}"):
            frames[-1]["stmts"].append(code.strip())
        for ch in bare:
            if ch == "{":
                depth += 1
                if pending is not None:
                    pending["open"] = depth
                    frames.append(pending)
                    pending = None
            elif ch == "}":
                if len(frames) > 1 and frames[-1]["open"] == depth:
                    f = frames.pop()
                    if f["kind"] == "THEN":
                        out.append(dict(actions=[s for fr in frames for s in fr["stmts"]],
                                        checks=f["stmts"]))
                depth -= 1
    return out


def lookup_cases(root):
    """Lookup::SingleListSingleIdx and Lookup::MultiListSingleIdx (test_Grid.cpp:151-500): the
    leaf lists' order under track, untrack (swap with the last entry) and reset, and each
    position's index in its list. One case per leaf section: the positions, the actions of its
    enclosing sections, and its checks."""
    f = "src/tests/test_Grid.cpp"
    L = lines_of(root, f)
    out = []
    for a, b in [(151, 328), (330, 500)]:
        text = "\n".join(L[a - 1: b])
        pos = {m.group(1): [int(x) for x in _nums(m.group(2))]
               for m in re.finditer(r"const Vec3i (pos\d+)\(([^)]*)\);", text)}
        m = re.search(r"Grid grid\(Vec3i\(([^)]*)\), Vec3i\(([^)]*)\)\)", text)
        size, off = [int(x) for x in _nums(m.group(1))], [int(x) for x in _nums(m.group(2))]
        for k, leaf in enumerate(catch_leaves(L, a, b)):
            steps = []
            for s in leaf["actions"]:
                m = re.match(r"grid\.track\((pos\d+)_idx(?:, (\d+))?\);", s)
                if m:
                    steps.append(["track", m.group(1), int(m.group(2) or 0)])
                    continue
                m = re.match(r"grid\.untrack\((?:grid\.index\((pos\d+)\)|(pos\d+)_idx)(?:, (\d+))?\);", s)
                if m:
                    steps.append(["untrack", m.group(1) or m.group(2), int(m.group(3) or 0)])
                    continue
                if re.match(r"grid\.reset\(\);", s):
                    steps.append(["reset"])
            checks = []
            for s in leaf["checks"]:
                m = re.match(r"CHECK\(grid\.list\((\d*)\)\.size\(\) == (\d+)\);", s)
                if m:
                    checks.append(["size", int(m.group(1) or 0), int(m.group(2))])
                    continue
                m = re.match(r"CHECK\(grid\.list\((\d*)\)\[(\d+)\] == (pos\d+)_idx\);", s)
                if m:
                    checks.append(["entry", int(m.group(1) or 0), int(m.group(2)), m.group(3)])
                    continue
                m = re.match(r"CHECK\(grid\.get\((pos\d+)\) == (\d+|null_idx)\);", s)
                if m:
                    v = -1 if m.group(2) == "null_idx" else int(m.group(2))
                    checks.append(["get", m.group(1), v])
                    continue
                m = re.match(r"CHECK\(grid\.is_tracked\((pos\d+)_idx\) == (true|false)\);", s)
                if m:
                    checks.append(["tracked", m.group(1), m.group(2) == "true"])
            if checks:
                out.append(dict(ref=f"{f}:{a}-{b}#{k}", size=size, offset=off, positions=pos,
                                steps=steps, checks=checks))
    return out


def multi_lookup_cases(root):
    """Lookup::Multi (test_Grid.cpp:502-731), the lookup with one index per list: list order
    under track (a second track in the same list does nothing), untrack (swap with the last
    entry) and reset, and each position's index in each list. One case per leaf section."""
    f = "src/tests/test_Grid.cpp"
    L = lines_of(root, f)
    a, b = 525, 731
    text = "\n".join(L[a - 1: b])
    pos = {m.group(1): [int(x) for x in _nums(m.group(2))]
           for m in re.finditer(r"const Vec3i (pos\d+)\(([^)]*)\);", text)}
    m = re.search(r"Grid grid\(Vec3i\(([^)]*)\), Vec3i\(([^)]*)\)\)", text)
    size, off = [int(x) for x in _nums(m.group(1))], [int(x) for x in _nums(m.group(2))]
    out = []
    for k, leaf in enumerate(catch_leaves(L, a, b)):
        steps = []
        for s in leaf["actions"]:
            m = re.match(r"grid\.(track|untrack)\((pos\d+)_idx, (\d+)\);", s)
            if m:
                steps.append([m.group(1), m.group(2), int(m.group(3))])
            elif re.match(r"grid\.reset\(\);", s):
                steps.append(["reset"])
        checks = []
        for s in leaf["checks"]:
            m = re.match(r"(?:CHECK|REQUIRE)\(grid\.list\((\d+)\)\.size\(\) == (\d+)\);", s)
            if m:
                checks.append(["size", int(m.group(1)), int(m.group(2))])
                continue
            m = re.match(r"(?:CHECK|REQUIRE)\(grid\.list\((\d+)\)\[(\d+)\] == (pos\d+)_idx\);", s)
            if m:
                checks.append(["entry", int(m.group(1)), int(m.group(2)), m.group(3)])
                continue
            m = re.match(r"(?:CHECK|REQUIRE)\(grid\.get\((pos\d+)\)\((\d+)\) == (\d+|Felt::null_idx)\);", s)
            if m:
                v = -1 if "null" in m.group(3) else int(m.group(3))
                checks.append(["get", m.group(1), int(m.group(2)), v])
        if checks:
            out.append(dict(ref=f"{f}:{a}-{b}#{k}", size=size, offset=off, positions=pos,
                            steps=steps, checks=checks))
    return out


def partitioned_lookup_case(root):
    """Partitioned::Lookup (test_Grid.cpp:1175-1243, the block before the masked reset): leaf
    positions tracked into lists of a 9^3 grid in 3^3 partitions, and the children lists, the
    children lookup, each partition's leaf lists and the leaves' indices that result."""
    f = "src/tests/test_Grid.cpp"
    L = lines_of(root, f)
    a, b = 1175, 1243
    text = "\n".join(L[a - 1: b])
    m = re.search(r"Grid grid\(Vec3i\(([^)]*)\), Vec3i\(([^)]*)\), Vec3i\(([^)]*)\)\)", text)
    size, off, part = ([int(x) for x in _nums(m.group(i))] for i in (1, 2, 3))
    vecs = {m.group(1): [int(x) for x in _nums(m.group(2))]
            for m in re.finditer(r"const Vec3i (\w+)\(([^)]*)\);", text)}
    leaves = [lf for lf in catch_leaves(L, a, b) if any("track(" in s for s in lf["actions"])]
    assert len(leaves) == 1
    steps = []
    for s in leaves[0]["actions"]:
        m = re.match(r"grid\.track\((pos\d+), (\d+)\);", s)
        if m:
            steps.append([m.group(1), int(m.group(2))])
            continue
        m = re.match(r"grid\.track\(\w+_idx, grid\.children\(\)\.get\(\w+\)\.index\((pos\d+)\), (\d+)\);", s)
        if m:
            steps.append([m.group(1), int(m.group(2))])
    checks = []
    for s in leaves[0]["checks"]:
        m = re.match(r"CHECK\(grid\.children\(\)\.lookup\(\)\.list\((\d+)\)\.size\(\) == (\d+)\);", s)
        if m:
            checks.append(["children_size", int(m.group(1)), int(m.group(2))])
            continue
        m = re.match(r"CHECK\(grid\.children\(\)\.lookup\(\)\.list\((\d+)\)\[(\d+)\] == (\w+)_idx\);", s)
        if m:
            checks.append(["children_entry", int(m.group(1)), int(m.group(2)), m.group(3)])
            continue
        m = re.match(r"CHECK\(grid\.children\(\)\.lookup\(\)\.get\((\w+)\)\((\d+)\) == (\d+)\);", s)
        if m:
            checks.append(["children_get", m.group(1), int(m.group(2)), int(m.group(3))])
            continue
        m = re.match(r"CHECK\(grid\.children\(\)\.get\((\w+)\)\.list\((\d+)\)\.size\(\) == (\d+)\);", s)
        if m:
            checks.append(["leaves_size", m.group(1), int(m.group(2)), int(m.group(3))])
            continue
        m = re.match(r"CHECK\(grid\.children\(\)\.get\((\w+)\)\.get\((pos\d+)\) == (\d+)\);", s)
        if m:
            checks.append(["leaf_get", m.group(1), m.group(2), int(m.group(3))])
    return dict(ref=f"{f}:{a}-{b}", size=size, offset=off, part=part, vectors=vecs, steps=steps,
                checks=checks)


def neighs_case(root):
    f = "src/tests/test_Grid.cpp"
    L = lines_of(root, f)
    text = "\n".join(L[2398:2416])
    vs = re.findall(r"Vec3i\((-?\d+), (-?\d+), (-?\d+)\)", text)
    pts = [[int(a), int(b), int(c)] for a, b, c in vs]
    return dict(ref=f"{f}:2398-2416", centre=pts[0], order=pts[1:])


VEC = r"Vec([23])[fi]\(([^()]*)\)"


def vec_of(text):
    """Numbers of the first VecNf/VecNi(...) literal in a line."""
    m = re.search(VEC, text)
    return [float(x.strip().rstrip("f")) for x in m.group(2).split(",")]


def ray_cases(root):
    """Raycasting (test_Surface.cpp, SCENARIO "Surface - raycasting"): per case the surface set
    up by its GIVEN (size, partition, layers, seed, updates), the ray (origin, direction,
    whether the test normalises it) and the expectation: a hit position with its Approx epsilon,
    a miss, or any hit. Rotation sweeps record the axis; the rays follow from it."""
    rel = "src/tests/test_Surface.cpp"
    ln = lines_of(root, rel)
    at = lambda i: ln[i - 1]

    def setup(decl_line):
        m = re.search(r"Surface<(\d), (\d)> surface\((Vec\di\([^)]*\)), (Vec\di\([^)]*\))\)",
                      at(decl_line))
        D, L = int(m.group(1)), int(m.group(2))
        size = [int(x) for x in vec_of(m.group(3))]
        part = [int(x) for x in vec_of(m.group(4))]
        return D, L, size, part

    def updates(first, last):
        out = []
        for i in range(first, last + 1):
            m = re.search(r"return (-?\d+(?:\.\d+)?)f;", at(i))
            if m:
                out.append(["update", float(m.group(1))])
        return out

    cases = []
    # GIVEN at 1284: seed at 1286, three updates 1287-1295
    D, L, size, part = setup(1284)
    base = [["seed", [int(x) for x in vec_of(at(1286))]]] + updates(1287, 1295)
    for ray_ln, chk_ln, extra in [(1301, 1305, []), (1311, 1315, []), (1321, 1325, []),
                                  (1331, 1335, []), (1347, 1351, updates(1341, 1343)),
                                  (1358, 1362, []), (1368, 1372, [])]:
        r = at(ray_ln)
        vecs = re.findall(VEC, r)
        origin = [float(x.strip().rstrip("f")) for x in vecs[0][1].split(",")]
        direction = [float(x.strip().rstrip("f")) for x in vecs[1][1].split(",")]
        c = at(chk_ln)
        if "!= surface.ray_miss" in c:
            expect, hit = "hit", None
        elif "== surface.ray_miss" in c:
            expect, hit = "miss", None
        else:
            expect, hit = "at", vec_of(c)
        cases.append(dict(ref=f"{rel}:{ray_ln}-{chk_ln}", dims=D, layers=L, size=size, part=part,
                          steps=base + extra, origin=origin, dir=direction,
                          normalize="normalized()" in r, expect=expect, hit=hit,
                          epsilon=float(re.search(r"epsilon\(([\d.]+)\)", c).group(1))
                          if "epsilon(" in c else None))
    # 2D GIVEN at 1420: seed 1423, updates 1424-1432, ray 1438, check 1442
    D2, L2, size2, part2 = setup(1420)
    steps2 = [["seed", [int(x) for x in vec_of(at(1423))]]] + updates(1424, 1432)
    r, c = at(1438), at(1442)
    vecs = re.findall(VEC, r)
    cases.append(dict(ref=f"{rel}:1438-1442", dims=D2, layers=L2, size=size2, part=part2,
                      steps=steps2,
                      origin=[float(x.strip().rstrip("f")) for x in vecs[0][1].split(",")],
                      dir=[float(x.strip().rstrip("f")) for x in vecs[1][1].split(",")],
                      normalize=False, expect="at", hit=vec_of(c),
                      epsilon=float(re.search(r"epsilon\(([\d.]+)\)", c).group(1))))
    # rotation sweeps (1373-1413 on the GIVEN at 1284; 1495-1533 on the GIVEN at 1479): rays
    # from R*(0, 0, -10) along R*(0, 0, 1), R = AngleAxis(k * 0.1 * pi, axis), k = 0..19
    for given, lo, hi in [(1284, 1373, 1413), (1479, 1495, 1533)]:
        Dg, Lg, sz, pt = setup(given)
        st = [["seed", [0, 0, 0]]] + updates(given + 3, given + 11)
        for i in range(lo, hi + 1):
            t = at(i)
            if "check(Vec3f" not in t:
                continue
            axis = [0.0, 1.0, 0.0] if "UnitY" in t else vec_of(t)
            cases.append(dict(ref=f"{rel}:{i}", dims=Dg, layers=Lg, size=sz, part=pt, steps=st,
                              sweep_axis=axis, normalize_axis="normalized()" in t,
                              expect="hit"))
    return cases


def serial_cases(root):
    """Surface::save / Surface::load (test_Surface.cpp:464-500): the 9x9 surface after one
    update of -0.6 is saved and loaded; the loaded surface's snapshot equals the original's, and
    after an update of 0.6 it holds the grid literal that follows."""
    f = "src/tests/test_Surface.cpp"
    L = lines_of(root, f)
    start = next(i for i, ln in enumerate(L, 1) if "surface is serialised to disk then loaded" in ln)
    upd_at = next(i for i in range(start, start + 40) if "surface_loaded.update" in L[i - 1])
    grid_at = next(i for i in range(upd_at, upd_at + 20) if "isogrid_check.data() =" in L[i - 1])
    vals, end = data_block(L, grid_at)
    return [dict(name="save_load_then_contract_9x9", ref=f"{f}:{start}-{end}", size=[9, 9],
                 part=[3, 3], layers=2, before=[["seed", [0, 0]], ["update", -0.6]],
                 after=[["update", 0.6]], grid=vals, grid_ref=f"{f}:{grid_at}-{end}")]


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FELT_REFERENCE")
    if not root:
        sys.exit("usage: make_golden.py <reference source root> (or set FELT_REFERENCE)")
    out = dict(surface=surface_cases(root), poly=poly_cases(root),
               curvature=curvature_cases(root), numeric=numeric_cases(root), lookup=lookup_cases(root),
               multi_lookup=multi_lookup_cases(root),
               partitioned_lookup=partitioned_lookup_case(root),
               neighs=neighs_case(root), ray=ray_cases(root), serial=serial_cases(root))
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_golden.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst, {k: (len(v) if isinstance(v, list) else 1) for k, v in out.items()})


if __name__ == "__main__":
    main()
