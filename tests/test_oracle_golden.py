"""Pin the CPU oracle to the reference's own known-answer tests.

Every case below comes from tests/golden/reference_known_answers.json, which
tests/golden/make_golden.py parsed out of the reference's unit tests (each case
carries the reference file:line). These run without a GPU.
"""
import math

import numpy as np
import pytest

import oracle


def test_sfc64_against_numpy_stream(golden):
    # hoomd-rand/src/sfc.rs:158-205: 17 outputs of SFC64::seed_from_u64(0)
    want = [int(v) for v in golden["sfc64"]["seed_from_u64_0"]["values"]]
    got = oracle.sfc64_seed_from_u64(0, len(want))
    assert [int(x) for x in got] == want


def test_sfc64_deep(golden):
    # hoomd-rand/src/sfc.rs:208-214: the 2^17-th output
    d = golden["sfc64"]["deep"]
    got = oracle.sfc64_seed_from_u64(0, 1, skip=d["index"])
    assert int(got[0]) == int(d["value"])


@pytest.mark.parametrize("case", range(32))
def test_point_to_space_index(golden, case):
    c = golden["checkerboard"]["point_to_space_index"][case]
    L = c["edge_lengths"]
    w, s = oracle.checkerboard_dimensions(L, c["range"], c["periodic"])
    origin = [-x / 2.0 for x in L]
    assert oracle.point_to_space_index(origin, w, s, c["periodic"], c["point"]) == c["expected"], c["src"]


def test_compute_dimensions(golden):
    cases = golden["checkerboard"]["compute_dimensions"]
    assert len(cases) == 5
    for c in cases:
        per = c["periodic"]
        if per[0] != per[1]:
            # mixed periodicity: check each axis on its own
            for a in range(2):
                w, s = oracle.checkerboard_dimensions([c["edge_lengths"][a]] * 2, c["range"], per[a])
                assert w[0] == c["space_width"][a] and s[0] == c["shape"][a], c["src"]
            continue
        w, s = oracle.checkerboard_dimensions(c["edge_lengths"], c["range"], per[0])
        assert list(w) == c["space_width"], c["src"]
        assert [int(x) for x in s] == c["shape"], c["src"]


def test_space_indices_by_color(golden):
    for c in golden["checkerboard"]["space_indices_by_color"]:
        if len(c["shape"]) > 3:
            continue  # the sweep path is 2-D and 3-D
        cols = oracle.space_indices_by_color(c["shape"])
        assert cols.shape[0] == 2 ** len(c["shape"])
        for color, k, v in c["entries"]:
            assert int(cols[color][k]) == v, c["src"]


def test_wrap(golden):
    for c in golden["wrap"]:
        got = oracle.wrap(c["point"], c["edge_lengths"])
        assert list(got) == c["expected"], c["src"]


def test_ghosts(golden):
    for c in golden["ghosts"]:
        got = oracle.generate_ghosts(c["point"], c["edge_lengths"], c["range"])
        want = np.array(c["expected"], dtype=float).reshape(-1, len(c["edge_lengths"]))
        assert got.shape == want.shape, c["src"]
        got = np.array(sorted(map(tuple, got)))
        want = np.array(sorted(map(tuple, want)))
        if got.size:
            np.testing.assert_allclose(got, want, rtol=1e-12, err_msg=c["src"])


def _versor(factors):
    q = np.array([1.0, 0.0, 0.0, 0.0])
    for axis, angle in factors:
        q = oracle.versor_combine(q, oracle.versor_from_axis_angle(axis, angle))
    return q


def _conj(q):
    return np.array([q[0], -q[1], -q[2], -q[3]])


def test_convex_polyhedron_overlaps(golden):
    # convex_polytope.rs:683-879 through assert_symmetric_overlap (:531-562)
    shapes = golden["convex_shapes"]
    assert len(golden["convex_3d"]) == 62
    for c in golden["convex_3d"]:
        v = np.array(shapes[c["shape"]])
        qa = _versor(c["q_a"])
        qb = _versor(c["q_b"])
        for r_ab, oa, ob in ((np.array(c["r_ab"]), qa, qb), (-np.array(c["r_ab"]), qb, qa)):
            ia = _conj(oa)
            v_ij = oracle.versor_rotate(ia, r_ab)
            o_ij = oracle.versor_combine(ob, ia)
            assert oracle.convex_intersects_at_3d(v, v, v_ij, o_ij) == c["expected"], c["src"]


def test_convex_polygon_overlaps(golden):
    shapes = golden["convex_shapes"]
    assert len(golden["convex_2d"]) == 34
    for c in golden["convex_2d"]:
        a = np.array(shapes[c["a"]])
        b = np.array(shapes[c["b"]])
        if not c["symmetric"]:
            assert oracle.convex_intersects_at_2d(a, b, c["v_ij"], c["theta_ij"]) == c["expected"], c["src"]
            continue
        for r_ab, sa, sb, ta, tb in ((np.array(c["r_ab"]), a, b, c["theta_a"], c["theta_b"]),
                                     (-np.array(c["r_ab"]), b, a, c["theta_b"], c["theta_a"])):
            inv = -ta
            s, co = oracle.cr_sincos(inv)
            v_ij = [r_ab[0] * co - r_ab[1] * s, r_ab[0] * s + r_ab[1] * co]
            assert oracle.convex_intersects_at_2d(sa, sb, v_ij, tb + inv) == c["expected"], c["src"]


def test_surface_mesh_separating_axes(golden):
    # ConvexSurfaceMesh2d::intersects_at (convex_surface_mesh_2d.rs:578-640) on the
    # reference's own cases (square_no_rot, square_rot, square_triangle).
    g = golden["surface_mesh_2d"]
    assert len(g["cases"]) == 34
    shapes = {k: np.array(v) for k, v in g["shapes"].items()}
    for c in g["cases"]:
        a, b = shapes[c["a"]], shapes[c["b"]]
        if not c["symmetric"]:
            assert oracle.surface_mesh_intersects_at_2d(a, b, c["v_ij"], c["theta_ij"]) == c["expected"], c["src"]
            continue
        for r_ab, sa, sb, ta, tb in ((np.array(c["r_ab"]), a, b, c["theta_a"], c["theta_b"]),
                                     (-np.array(c["r_ab"]), b, a, c["theta_b"], c["theta_a"])):
            inv = -ta
            s, co = oracle.cr_sincos(inv)
            v_ij = [r_ab[0] * co - r_ab[1] * s, r_ab[0] * s + r_ab[1] * co]
            assert oracle.surface_mesh_intersects_at_2d(sa, sb, v_ij, tb + inv) == c["expected"], c["src"]


def _exact_sincos(x):
    """sin x, cos x of the binary64 x to ~75 digits (Machin pi, Taylor series), then rounded."""
    from decimal import Decimal, localcontext
    with localcontext() as ctx:
        ctx.prec = 90

        def arctan_inv(n):
            n = Decimal(n)
            s, t, k, sign = Decimal(0), 1 / n, 1, 1
            while True:
                term = t / k
                if term < Decimal(10) ** -88:
                    return s
                s += sign * term
                t /= n * n
                k += 2
                sign = -sign

        half_pi = (16 * arctan_inv(5) - 4 * arctan_inv(239)) / 2
        X = Decimal(x)
        k = (X / half_pi).to_integral_value()
        r = X - k * half_pi
        sn, cs = Decimal(0), Decimal(0)
        term, n = r, 1
        while abs(term) > Decimal(10) ** -85:
            sn += term
            term = -term * r * r / ((n + 1) * (n + 2))
            n += 2
        term, n = Decimal(1), 0
        while abs(term) > Decimal(10) ** -85:
            cs += term
            term = -term * r * r / ((n + 1) * (n + 2))
            n += 2
        sn, cs = [(sn, cs), (cs, -sn), (-sn, -cs), (-cs, sn)][int(k) % 4]
        return float(sn), float(cs)


def test_cr_sincos_is_correctly_rounded():
    # The 2-D rotation path (Angle -> RotationMatrix, angle.rs:120-150) uses these values on
    # the device and in the oracle: check them against a 90-digit evaluation.
    rng = np.random.default_rng(17)
    xs = list(rng.uniform(-7.0, 7.0, 300)) + list(rng.uniform(-1e5, 1e5, 100))
    xs += [math.pi / 4, -math.pi / 4, math.pi / 2, math.pi, 3 * math.pi / 2, 1e-9, -3e-8, 2.0 ** -26, 1e6,
           355.0, 103993.0, float(2 ** 20 - 1)]
    for x in xs:
        assert oracle.cr_sincos(float(x)) == _exact_sincos(float(x)), x
    with pytest.raises(ValueError):
        oracle.cr_sincos(2.0 ** 20)


def test_cr_sincos_against_platform_libm():
    # The reference calls the platform libm; this platform's sin/cos are not always
    # correctly rounded. The two agree on almost every argument and never by more than 1 ulp.
    rng = np.random.default_rng(18)
    xs = rng.uniform(-4.0, 4.0, 20000)
    diff = 0
    for x in xs:
        s, c = oracle.cr_sincos(float(x))
        for got, ref in ((s, math.sin(x)), (c, math.cos(x))):
            if got != ref:
                diff += 1
                assert abs(got - ref) <= np.spacing(abs(ref))
    assert diff < 0.01 * 2 * len(xs)


def test_sphere_overlaps_through_hard_sphere_pair(golden):
    # sphere.rs:592-: |v|^2 <= (r0 + r1)^2. The sweep path uses HardSphere (strict <) on
    # sites; these cases are away from the boundary, so both agree.
    for c in golden["spheres"]:
        d = c["radius0"] + c["radius1"]
        sysm = oracle.System(3, [100.0] * 3, [[0.0, 0.0, 0.0], c["v_ij"]], diameter=d)
        assert (sysm.overlap_count() == 1) == c["expected"], c["src"]


def test_lennard_jones_special_points(golden):
    g = golden["lennard_jones"]
    for eps in g["epsilon"]:
        for sig in g["sigma"]:
            assert abs(oracle.lj_energy(eps, sig, sig)) < 1e-12
            assert math.isclose(oracle.lj_energy(eps, sig, 2.0 ** (1.0 / 6.0) * sig), -eps, rel_tol=1e-12)
            assert math.isclose(oracle.lj_energy(eps, sig, 2.0 * sig), -63.0 / 1024.0 * eps, rel_tol=1e-12)


def test_hard_circle_delta_energy_doc(golden):
    g = golden["pairwise_doc"]["hard_circle_delta"]
    s = oracle.System(2, [100.0, 100.0], g["bodies"], diameter=g["diameter"])
    assert s.delta_energy_one(g["moved"], g["trials"][0]) == math.inf
    assert s.delta_energy_one(g["moved"], g["trials"][1]) == 0.0


def test_lj_total_energy_doc(golden):
    g = golden["pairwise_doc"]["lj_total"]
    sigma = 1.0 / 2.0 ** (1.0 / 6.0)
    # Unshifted Isotropic<LennardJones>: a shift at the zero crossing r = sigma is exactly 0.
    s = oracle.System(2, [100.0, 100.0], g["bodies"], interaction=oracle.LENNARD_JONES, lj_epsilon=g["epsilon"],
                      lj_sigma=sigma, lj_r_cut=g["r_cut"], lj_r_shift=sigma)
    assert s.total_energy() == g["expected"]


def test_ziggurat_tables_shape():
    x, f = oracle.ziggurat_tables()
    assert x[1] == 3.6541528853610088 and x[256] == 0.0
    assert np.all(np.diff(x[1:]) < 0)
    assert abs(x[0] - 3.910757959537090) < 1e-12
    assert f[256] == 1.0


def test_cbrt_accuracy():
    rng = np.random.default_rng(5)
    for u in np.concatenate([rng.random(2000), [1e-300, 2.0 ** -53, 0.5, 0.125, 1.0 - 2.0 ** -53]]):
        got = oracle.cbrt(float(u))
        assert abs(got - np.cbrt(u)) <= 2.0 * np.spacing(np.cbrt(u))
