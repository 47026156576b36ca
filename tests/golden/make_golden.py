"""Extract the reference's known-answer test vectors for the sweep path into JSON.

Run in a checkout that holds the reference sources (glotzerlab/hoomd-rs v1.4.0):

    python tests/golden/make_golden.py <path of the reference checkout>

The reference is Rust and cannot be built here, so its unit tests are read as
text: every literal that a test on the hot path asserts (SFC64 outputs, checkerboard
index maps, wrap/ghost images, convex overlap cases, sphere overlaps, LJ special
points, hard-pair delta energies) is parsed out of the test source and written with
the ``file:line`` it came from. The output, ``reference_known_answers.json``, is
committed; the tests only read the JSON.
"""
from __future__ import annotations

import json
import math
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _read(root, rel):
    with open(os.path.join(root, rel)) as f:
        return f.read()


def _line_of(text, pos):
    return text.count("\n", 0, pos) + 1


def _num(s: str) -> float:
    s = s.strip()
    m = re.fullmatch(r"([-+]?[0-9.]+)(?:_f64)?\.next_down\(\)", s)
    if m:
        return math.nextafter(float(m.group(1)), -math.inf)
    s = s.replace("_", "")
    s = s.replace("f64", "")
    if not re.fullmatch(r"[-+0-9.e/* ()]+", s):
        raise ValueError(f"unexpected numeric expression {s!r}")
    return float(eval(s, {"__builtins__": {}}, {}))  # digits and + - * / only


def _fn_blocks(text):
    """Yield (name, start, end) for each `fn name(` block (brace matched)."""
    for m in re.finditer(r"\bfn\s+(\w+)\s*(?:<[^>]*>)?\s*\(", text):
        i = text.find("{", m.end())
        depth = 0
        j = i
        while j < len(text):
            if text[j] == "{":
                depth += 1
            elif text[j] == "}":
                depth -= 1
                if depth == 0:
                    break
            j += 1
        yield m.group(1), m.start(), j


def sfc64(root):
    rel = "hoomd-rand/src/sfc.rs"
    t = _read(root, rel)
    m = re.search(r"SFC64_REFERENCE_OUTPUT: \[u64; (\d+)\] = \[(.*?)\];", t, re.S)
    vals = [int(x.replace("_", "")) for x in re.findall(r"[\d_]+", m.group(2))]
    assert len(vals) == int(m.group(1))
    d = re.search(r"fn test_sfc64_deep\(\).*?2_u64\.pow\((\d+)\) - 1.*?assert_eq!\(rng\.next_u64\(\), ([\d_]+)\)",
                  t, re.S)
    return {
        "seed_from_u64_0": {"values": [str(v) for v in vals], "src": f"{rel}:{_line_of(t, m.start())}"},
        "deep": {"index": 2 ** int(d.group(1)) - 1, "value": str(int(d.group(2).replace("_", ""))),
                 "src": f"{rel}:{_line_of(t, d.start())}"},
    }


def checkerboard(root):
    rel = "hoomd-mc/src/hypercuboid.rs"
    t = _read(root, rel)
    out = {"point_to_space_index": [], "compute_dimensions": [], "space_indices_by_color": []}
    for name, s, e in _fn_blocks(t):
        body = t[s:e]
        if name.startswith("test_point_to_space_index"):
            m = re.search(r"with_fixed_origin\(\s*([\d.]+)\.try_into\(\)\?,\s*\[([\d.]+)\.try_into\(\)\?,\s*"
                          r"([\d.]+)\.try_into\(\)\?\],\s*\[(true|false); 2\]", body)
            rng, lx, ly, per = float(m.group(1)), float(m.group(2)), float(m.group(3)), m.group(4) == "true"
            for c in re.finditer(r"point_to_space_index\(&Cartesian::from\(\[([^\]]+)\]\)\) == (None|Some\((\d+)\))",
                                 body):
                pt = [_num(x) for x in c.group(1).split(",")]
                out["point_to_space_index"].append({
                    "range": rng, "edge_lengths": [lx, ly], "periodic": per, "point": pt,
                    "expected": None if c.group(2) == "None" else int(c.group(3)),
                    "src": f"{rel}:{_line_of(t, s + c.start())}"})
        elif name.startswith("test_compute_dimensions"):
            for c in re.finditer(
                    r"compute_dimensions\(\s*\[([\d.]+)\.try_into\(\)\?,\s*([\d.]+)\.try_into\(\)\?\],\s*"
                    r"([\d.]+)\.try_into\(\)\?,\s*(\[true; 2\]|\[false; 2\]|\[true, false\]),?\s*\);\s*"
                    r"check!\(space_width == \[([^\]]+)\]\);\s*check!\(shape == \[([^\]]+)\]\);", body):
                per = {"[true; 2]": [True, True], "[false; 2]": [False, False], "[true, false]": [True, False]}[c.group(4)]
                out["compute_dimensions"].append({
                    "edge_lengths": [float(c.group(1)), float(c.group(2))], "range": float(c.group(3)),
                    "periodic": per, "space_width": [_num(x) for x in c.group(5).split(",")],
                    "shape": [int(x) for x in c.group(6).split(",")],
                    "src": f"{rel}:{_line_of(t, s + c.start())}"})
        elif name.startswith("test_construct_space_indices_by_color"):
            m = re.search(r"construct_space_indices_by_color\(\[([\d, ]+)\]\)", body)
            shape = [int(x) for x in m.group(1).split(",")]
            entries = [(int(a), int(b), int(eval(v, {"__builtins__": {}}, {})))
                       for a, b, v in re.findall(r"space_indices_by_color\[(\d+)\]\[(\d+)\] == ([\d +]+)\)", body)]
            out["space_indices_by_color"].append({"shape": shape, "entries": entries,
                                                  "src": f"{rel}:{_line_of(t, s)}"})
    return out


def wrap_and_ghosts(root):
    rel = "hoomd-microstate/src/boundary/periodic/cuboid.rs"
    t = _read(root, rel)
    wraps, ghosts = [], []
    for name, s, e in _fn_blocks(t):
        body = t[s:e]
        if name not in ("wrap", "ghosts"):
            continue
        em = re.search(r"Hypercuboid \{\s*edge_lengths: \[(.*?)\]\s*,?\s*\}", body, re.S)
        if not em:
            continue
        L = [float(x) for x in re.findall(r"(?:pos\()?([\d.]+)(?:\)|\.try_into)", em.group(1))]
        pm = re.search(r"Periodic::new\(([\d.]+), cuboid\)", body)
        rng = float(pm.group(1))
        if name == "wrap":
            for c in re.finditer(r"let point = Point::new\(\[([^\]]+)\]\.into\(\)\);\s*"
                                 r"assert_eq!\(periodic\.wrap\(point\), Ok\((point|Point::new\(\[([^\]]+)\]\.into\(\)\))\)\);",
                                 body):
                p = [_num(x) for x in c.group(1).split(",")]
                exp = p if c.group(2) == "point" else [_num(x) for x in c.group(3).split(",")]
                wraps.append({"edge_lengths": L, "point": p, "expected": exp, "src": f"{rel}:{_line_of(t, s + c.start())}"})
        else:
            for c in re.finditer(r"generate_ghosts\(&Point::new\(\[([^\]]+)\]\.into\(\)\)\);\s*"
                                 r"(assert!\(ghosts\.is_empty\(\)\)|assert_ghost_positions\(&ghosts, &\[(.*?)\]\);)",
                                 body, re.S):
                p = [_num(x) for x in c.group(1).split(",")]
                exp = [] if c.group(2).startswith("assert!") else [
                    [_num(x) for x in g.split(",")] for g in re.findall(r"\[([^\[\]]+)\]", c.group(3))]
                ghosts.append({"edge_lengths": L, "range": rng, "point": p, "expected": exp,
                               "src": f"{rel}:{_line_of(t, s + c.start())}"})
    return wraps, ghosts


_ROTATIONS = {
    # rotations set up at the top of each reference test, as (axis, angle) factors:
    # the versor is the product of the factors in order (q2.combine(&q1) -> [q2, q1]).
    "overlap_octahedron_no_rot": ([], []),
    "overlap_cube_no_rot": ([], []),
    "overlap_cube_rot1": ([], [([0.0, 0.0, 1.0], "PI/4")]),
    "overlap_cube_rot3": ([], [([0.0, 0.0, 1.0], "PI/4"), ([1.0, 0.0, 0.0], "PI/4")]),
}


def convex(root):
    rel = "hoomd-geometry/src/shape/convex_polytope.rs"
    t = _read(root, rel)
    shapes = {}
    for name in ("square", "triangle", "octahedron", "cube"):
        m = re.search(r"fn " + name + r"\(\) -> Convex<\w+> \{.*?with_vertices\(\[(.*?)\]\)", t, re.S)
        verts = [[_num(x.replace("FRAC_1_SQRT_2", repr(1 / math.sqrt(2)))) for x in v.split(",")]
                 for v in re.findall(r"\[([^\[\]]+)\]\.into\(\)", m.group(1))]
        shapes[name] = verts
    cases2d, cases3d = [], []
    for name, s, e in _fn_blocks(t):
        body = t[s:e]
        if name in ("square_no_rot", "square_rot"):
            ang = 0.0 if name == "square_no_rot" else math.pi / 4
            for c in re.finditer(r"assert!\((!?)square\.intersects_at\(&square, &\[([^\]]+)\]\.into\(\), &a\)\);", body):
                cases2d.append({"a": "square", "b": "square", "v_ij": [_num(x) for x in c.group(2).split(",")],
                                "theta_ij": ang, "expected": c.group(1) != "!", "symmetric": False,
                                "src": f"{rel}:{_line_of(t, s + c.start())}"})
        elif name == "square_triangle":
            for c in re.finditer(r"assert_symmetric_overlap\(\s*\[([^\]]+)\]\.into\(\),\s*&square,\s*&triangle,\s*"
                                 r"r_square,\s*r_triangle,\s*(true|false),?\s*\)", body):
                cases2d.append({"a": "square", "b": "triangle", "r_ab": [_num(x) for x in c.group(1).split(",")],
                                "theta_a": -math.pi / 4, "theta_b": math.pi, "expected": c.group(2) == "true",
                                "symmetric": True, "src": f"{rel}:{_line_of(t, s + c.start())}"})
        elif name in _ROTATIONS:
            shape = "octahedron" if "octahedron" in name else "cube"
            qa, qb = _ROTATIONS[name]
            for c in re.finditer(r"assert_symmetric_overlap\(\s*\[([^\]]+)\]\.into\(\),\s*&(\w+),\s*&(\w+),\s*"
                                 r"(\w+),\s*(\w+),\s*(true|false),?\s*\)", body):
                cases3d.append({"shape": shape, "r_ab": [_num(x) for x in c.group(1).split(",")],
                                "q_a": [[ax, math.pi / 4] for ax, _ in qa], "q_b": [[ax, math.pi / 4] for ax, _ in qb],
                                "expected": c.group(6) == "true", "src": f"{rel}:{_line_of(t, s + c.start())}"})
    return shapes, cases2d, cases3d


def surface_mesh_2d(root):
    """Separating-axis cases of ConvexSurfaceMesh2d (hoomd-blue's polygon cases, restated there)."""
    rel = "hoomd-geometry/src/shape/convex_surface_mesh_2d.rs"
    t = _read(root, rel)
    shapes = {}
    for name in ("square", "triangle"):
        m = re.search(r"fn " + name + r"\(\) -> ConvexSurfaceMesh2d \{.*?from_point_set\(\[(.*?)\]\)", t, re.S)
        shapes[name] = [[_num(x) for x in v.split(",")] for v in re.findall(r"\[([^\[\]]+)\]\.into\(\)", m.group(1))]
    cases = []
    for name, s, e in _fn_blocks(t):
        body = t[s:e]
        if name in ("square_no_rot", "square_rot"):
            ang = 0.0 if name == "square_no_rot" else math.pi / 4
            for c in re.finditer(r"assert!\((!?)square\.intersects_at\(&square, &\[([^\]]+)\]\.into\(\), &a\)\);", body):
                cases.append({"a": "square", "b": "square", "v_ij": [_num(x) for x in c.group(2).split(",")],
                              "theta_ij": ang, "expected": c.group(1) != "!", "symmetric": False,
                              "src": f"{rel}:{_line_of(t, s + c.start())}"})
        elif name == "square_triangle":
            for c in re.finditer(r"assert_symmetric_overlap\(\s*\[([^\]]+)\]\.into\(\),\s*&square,\s*&triangle,\s*"
                                 r"r_square,\s*r_triangle,\s*(true|false),?\s*\)", body):
                cases.append({"a": "square", "b": "triangle", "r_ab": [_num(x) for x in c.group(1).split(",")],
                              "theta_a": -math.pi / 4, "theta_b": math.pi, "expected": c.group(2) == "true",
                              "symmetric": True, "src": f"{rel}:{_line_of(t, s + c.start())}"})
    return {"shapes": shapes, "cases": cases}


def spheres(root):
    rel = "hoomd-geometry/src/shape/sphere.rs"
    t = _read(root, rel)
    out = []
    for name, s, e in _fn_blocks(t):
        if name != "intersects_at":
            continue
        body = t[s:e]
        r = re.findall(r"Sphere::with_radius\(([\d.]+)\.try_into\(\)\?\)", body)
        if len(r) < 2:
            continue
        for c in re.finditer(r"check!\((!?)sphere0\.intersects_at\(&sphere1, &Cartesian::from\(\[([^\]]+)\]\), &identity\)\)",
                             body):
            out.append({"radius0": float(r[0]), "radius1": float(r[1]),
                        "v_ij": [_num(x) for x in c.group(2).split(",")], "expected": c.group(1) != "!",
                        "src": f"{rel}:{_line_of(t, s + c.start())}"})
    return out


def lj(root):
    rel = "hoomd-interaction/src/univariate/lennard_jones.rs"
    t = _read(root, rel)
    m = re.search(r"fn special_points_12_6\(\s*#\[values\(([^)]*)\)\] epsilon: f64,\s*#\[values\(([^)]*)\)\] sigma: f64",
                  t, re.S)
    eps = [float(x) for x in m.group(1).split(",")]
    sig = [float(x) for x in m.group(2).split(",")]
    return {"epsilon": eps, "sigma": sig, "checks": [
        {"r_over_sigma": "1", "energy_over_epsilon": 0.0, "kind": "abs"},
        {"r_over_sigma": "2^(1/6)", "energy_over_epsilon": -1.0, "kind": "rel"},
        {"r_over_sigma": "2", "energy_over_epsilon": -63.0 / 1024.0, "kind": "rel"}],
        "src": f"{rel}:{_line_of(t, m.start())}"}


def pairwise_doc(root):
    rel = "hoomd-interaction/src/pairwise_cutoff.rs"
    t = _read(root, rel)
    dm = re.search(r"Body::point\(Cartesian::from\(\[0\.0, 0\.0\]\)\),\s*///\s*Body::point\(Cartesian::from\(\[2\.0, 0\.0\]\)\),"
                   r".*?delta_energy_one\(\s*///\s*&microstate,\s*///\s*1,\s*///\s*&Body::point\(\[([^\]]+)\]\.into\(\)\),"
                   r".*?assert_eq!\(delta_energy, f64::INFINITY\);.*?&Body::point\(\[([^\]]+)\]\.into\(\)\),"
                   r".*?assert_eq!\(delta_energy, 0\.0\);", t, re.S)
    lm = re.search(r"Body::point\(Cartesian::from\(\[0\.0, 0\.0\]\)\),\s*///\s*Body::point\(Cartesian::from\(\[1\.0, 0\.0\]\)\),"
                   r"\s*///\s*Body::point\(Cartesian::from\(\[0\.0, 5\.0\]\)\),\s*///\s*Body::point\(Cartesian::from\(\[-1\.0, 5\.0\]\)\),"
                   r".*?epsilon: ([\d.]+),.*?r_cut: ([\d.]+),.*?assert_eq!\(total_energy, (-?[\d.]+)\);", t, re.S)
    return {
        "hard_circle_delta": {"bodies": [[0.0, 0.0], [2.0, 0.0]], "diameter": 1.0, "moved": 1,
                              "trials": [[_num(x) for x in dm.group(1).split(",")], [_num(x) for x in dm.group(2).split(",")]],
                              "expected": ["inf", 0.0], "src": f"{rel}:{_line_of(t, dm.start())}"},
        "lj_total": {"bodies": [[0.0, 0.0], [1.0, 0.0], [0.0, 5.0], [-1.0, 5.0]], "epsilon": float(lm.group(1)),
                     "sigma": "2^(-1/6)", "r_cut": float(lm.group(2)), "expected": float(lm.group(3)),
                     "src": f"{rel}:{_line_of(t, lm.start())}"},
    }


def main(root):
    wraps, ghosts = wrap_and_ghosts(root)
    shapes, c2, c3 = convex(root)
    data = {
        "reference": "glotzerlab/hoomd-rs v1.4.0",
        "sfc64": sfc64(root),
        "checkerboard": checkerboard(root),
        "wrap": wraps,
        "ghosts": ghosts,
        "convex_shapes": shapes,
        "convex_2d": c2,
        "convex_3d": c3,
        "surface_mesh_2d": surface_mesh_2d(root),
        "spheres": spheres(root),
        "lennard_jones": lj(root),
        "pairwise_doc": pairwise_doc(root),
    }
    out = os.path.join(HERE, "reference_known_answers.json")
    with open(out, "w") as f:
        json.dump(data, f, indent=1)
    counts = {k: (len(v) if isinstance(v, list) else "") for k, v in data.items()}
    print(out, counts, {k: len(v) for k, v in data["checkerboard"].items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
