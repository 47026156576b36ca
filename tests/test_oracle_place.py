"""The oracle's restatement of state preparation: the OverlapPenalty pair energy against the
reference's known answers (hoomd-interaction/src/univariate/overlap_penalty.rs tests), and
QuickInsert / QuickCompress (hoomd-mc/src/quick_insert.rs, quick_compress.rs) against the
behaviour their own tests and the benchmark placement (benchmarks/src/place.rs) rely on."""
import math

import numpy as np
import pytest

import oracle


def pair_energy(x, k, dmax, eps, d=1.0):
    """Energy of two overlap-penalty spheres (diameter d) at distance r = d + x along x."""
    r = d + x
    o = oracle.System(3, [10.0, 10.0, 10.0], [[0.0, 0.0, 0.0], [r, 0.0, 0.0]], interaction=oracle.OVERLAP_PENALTY,
                      diameter=d, penalty=(k, dmax, eps))
    return o.total_energy()


def test_overlap_penalty_shoulder():
    # overlap_penalty.rs tests::shoulder: k = 0, eps = 15, d_max = 1
    assert pair_energy(1.0, 0.0, 1.0, 15.0) == 0.0
    assert pair_energy(0.0, 0.0, 1.0, 15.0) == 0.0
    assert pair_energy(-2.0 ** -53, 0.0, 1.0, 15.0) == 15.0  # 0.0_f64.next_down() after r = 1 - 2^-53
    assert pair_energy(-0.5, 0.0, 1.0, 15.0) == 15.0


def test_overlap_penalty_core():
    # tests::core: k = 0, eps = 0, d_max = 0.5
    assert pair_energy(0.5, 0.0, 0.5, 0.0) == 0.0
    assert pair_energy(-0.5, 0.0, 0.5, 0.0) == 0.0
    assert pair_energy(-0.5 - 2.0 ** -53, 0.0, 0.5, 0.0) == math.inf  # (-0.5).next_down()
    assert pair_energy(-0.75, 0.0, 0.5, 0.0) == math.inf


def test_overlap_penalty_harmonic():
    # tests::harmonic: k = 6, eps = 0, d_max = 10; energy(-0.125) = 0.5 k 0.125^2
    assert pair_energy(-0.125, 6.0, 10.0, 0.0, d=2.0) == 0.5 * 6.0 * 0.125 ** 2
    assert pair_energy(0.5, 6.0, 10.0, 0.0) == 0.0


def test_quick_insert_hard_spheres():
    # quick_insert.rs tests::hard_spheres, in a periodic 6 x 6 box: one body at the origin,
    # QuickInsert(target 10) applied until complete, then a serial sweep; 11 bodies, energy 0
    o = oracle.System(2, [6.0, 6.0], [[0.0, 0.0]], diameter=1.0)
    qi = {"target": 10, "allowed_overlaps": max(10 // 8, 1), "inserted": 0, "complete": 0}
    for _ in range(100):
        o.quick_insert(qi)
        if qi["complete"]:
            break
    o.serial_sweep(oracle.TRANSLATE, 0.1, 1.0)
    assert qi["inserted"] == 10 and qi["complete"] == 1
    assert o.n_bodies == 11
    assert o.total_energy() == 0.0


def test_quick_insert_counts_and_substep():
    o = oracle.System(3, [8.0, 8.0, 8.0], np.zeros((0, 3)), interaction=oracle.OVERLAP_PENALTY, diameter=1.0)
    qi = {"target": 200, "allowed_overlaps": 25, "inserted": 0, "complete": 0}
    a, r = o.quick_insert(qi)
    _, _, step, sub = o.state()
    assert (step, sub) == (0, 1)
    assert a == qi["inserted"] == o.n_bodies > 0
    # stops at 25 overlapping insertions or when all 200 are in
    assert a == 200 or a < 200
    assert o.total_energy() >= 0.0


def _place(o, n, rho, dim, target_steps=20000):
    """place_single_site_point_bodies (benchmarks/src/place.rs:31-110): QuickInsert then
    QuickCompress every 20 steps, a serial translation sweep (0.1) every step."""
    qi = {"target": n, "allowed_overlaps": max(n // 8, 1), "inserted": 0, "complete": 0}
    qc = {"target_volume": n / rho, "maximum_energy_per_site": 1000.0, "maximum_delta": 0.05, "state": 0,
          "is_final": 0, "boundary": [0.0, 0.0, 0.0]}
    for _ in range(target_steps):
        _, _, step, _ = o.state()
        if step % 20 == 0:
            if qi["complete"]:
                o.quick_compress(qc)
            else:
                o.quick_insert(qi)
        o.serial_sweep(oracle.TRANSLATE, 0.1, 1.0)
        o.increment_step()
        if qc["state"] == 3:
            break
    return qi, qc


def test_place_point_bodies_2d():
    n, rho = 64, 0.6
    L0 = math.sqrt(n / (0.7 * rho))
    o = oracle.System(2, [L0, L0], np.zeros((0, 2)), interaction=oracle.OVERLAP_PENALTY, diameter=1.0)
    qi, qc = _place(o, n, rho, 2)
    assert qi["complete"] and qc["state"] == 3
    assert o.n_bodies == n
    assert np.prod(o.box()) == pytest.approx(n / rho, rel=1e-12)
    assert o.total_energy() == 0.0


def test_set_box_maps_bodies():
    rng = np.random.default_rng(3)
    L = np.array([7.0, 9.0, 11.0])
    pos = (rng.random((50, 3)) - 0.5) * L
    o = oracle.System(3, L, pos, diameter=1.0)
    o.set_box(L * 0.9)
    got = o.state()[0]
    want = np.clip(pos * (0.9 * L / L), -0.9 * L / 2, np.nextafter(0.9 * L / 2, -np.inf))
    assert np.allclose(got, want, rtol=0, atol=1e-12)
    assert np.all(np.abs(got) <= 0.9 * L / 2)


def test_grand_canonical_hard_spheres_fugacity():
    # grand_canonical.rs tests::hard_spheres_fugacity, periodic 6 x 6: QuickInsert 10 bodies,
    # then 100 applies at fugacity 0 remove every body; 100 at fugacity 1 insert some
    o = oracle.System(2, [6.0, 6.0], [[0.0, 0.0]], diameter=1.0)
    qi = {"target": 10, "allowed_overlaps": 1, "inserted": 0, "complete": 0}
    for _ in range(100):
        o.quick_insert(qi)
        if qi["complete"]:
            break
    o.serial_sweep(oracle.TRANSLATE, 0.1, 1.0)
    assert qi["complete"] and o.n_bodies == 11 and o.total_energy() == 0.0
    ia, ir, ra, rr = o.grand_canonical(1.0, 0.0, 100)
    assert o.n_bodies == 0 and ra == 11 and ia == 0
    o.grand_canonical(1.0, 1.0, 100)
    assert o.n_bodies > 0
    assert o.total_energy() == 0.0


def test_removal_reuses_smallest_tag():
    # the tagged container: swap_remove by index, freed tags reused smallest first; GSD rows
    # follow tags
    o = oracle.System(2, [20.0, 20.0], [[float(i) * 2.0 - 9.0, 0.0] for i in range(6)], diameter=1.0)
    # drive removals at fugacity 0 until two bodies are gone, then insert at high fugacity
    while o.n_bodies > 4:
        o.grand_canonical(1.0, 0.0, 1)
    pos_index = o.state()[0]
    frame, _ = o.gsd_frame()
    assert sorted(map(tuple, frame[:, :2].astype(np.float64))) == sorted(map(tuple, pos_index.astype(np.float32)
                                                                          .astype(np.float64)))


# ---- the orientable placement: ApproximateShapeOverlap ------------------------------------------
HEXAGON = np.array([[0.5 * math.cos(2.0 * math.pi * x / 6), 0.5 * math.sin(2.0 * math.pi * x / 6)] for x in range(6)])
CUBE = np.array([[x, y, z] for x in (-0.5, 0.5) for y in (-0.5, 0.5) for z in (-0.5, 0.5)])


def test_approximate_separation_cuboid_known_answer():
    # hoomd-geometry/src/lib.rs:290-303: two 2 x 2 x 2 cuboids 1.8 apart separate after >= 0.2
    cube2 = 2.0 * CUBE
    d = oracle.approximate_separation(cube2, [1.8, 0.0, 0.0], [1.0, 0.0, 0.0, 0.0], 0.01)
    assert d >= 0.2
    # apart already: 0; at the same place: moved along the default unit (the last axis) to 2R
    assert oracle.approximate_separation(cube2, [2.5, 0.0, 0.0], [1.0, 0.0, 0.0, 0.0], 0.01) == 0.0
    d0 = oracle.approximate_separation(cube2, [0.0, 0.0, 0.0], [1.0, 0.0, 0.0, 0.0], 0.01)
    assert 2.0 <= d0 < 2.0 + 0.011


def test_approximate_shape_overlap_hexagon_known_answers():
    # approximate_shape_overlap.rs:75-121: regular hexagons (circumradius 0.5), OverlapPenalty
    # default, resolution 0.01, r_cut 1: >= 100 at 0.6, finite and >= 0 at 0.9, 0 at 1.0
    def energy(x):
        o = oracle.System(2, [10.0, 10.0], [[0.0, 0.0], [x, 0.0]], [0.0, 0.0],
                          interaction=oracle.CONVEX_POLYGON_PENALTY, vertices=HEXAGON, r_cut=1.0)
        return o.total_energy()
    assert energy(0.6) >= 100.0
    assert 0.0 <= energy(0.9) < math.inf
    assert energy(1.0) == 0.0
    # the penalty at the separation: 0.5 k d^2 + eps, infinite beyond d_max = 0.2
    d = oracle.approximate_separation(HEXAGON, [0.9, 0.0], [0.0], 0.01)
    assert energy(0.9) == 0.5 * 10000.0 * (d * d) + 100.0
    assert energy(0.55) == math.inf


def test_orientable_insertion_draws_orientations():
    # UniformIn for oriented bodies (uniform_in.rs:158-176): unit versors; angles in [0, 2 pi)
    o = oracle.System(3, [8.0] * 3, np.zeros((0, 3)), np.zeros((0, 4)), interaction=oracle.CONVEX_POLYHEDRON_PENALTY,
                      vertices=CUBE)
    qi = {"target": 40, "allowed_overlaps": 5, "inserted": 0, "complete": 0}
    o.quick_insert(qi)
    _, ori, _, _ = o.state()
    assert ori.shape[0] == qi["inserted"] > 0
    assert np.allclose(np.linalg.norm(ori, axis=1), 1.0, atol=1e-15)
    o2 = oracle.System(2, [8.0] * 2, np.zeros((0, 2)), np.zeros(0), interaction=oracle.CONVEX_POLYGON_PENALTY,
                       vertices=HEXAGON)
    qi2 = {"target": 40, "allowed_overlaps": 5, "inserted": 0, "complete": 0}
    o2.quick_insert(qi2)
    th = o2.state()[1]
    assert len(th) == qi2["inserted"] > 0 and np.all((th >= 0.0) & (th < 2.0 * math.pi))


def place_orientable(o, n, rho, max_steps=20000):
    """place_single_site_orientable_bodies (benchmarks/src/place.rs:120-219) on an oracle system
    created empty at half the density: QuickInsert then QuickCompress every 10 steps, a translation
    (0.03) and a rotation (0.1) ParallelSweep every step at kT = 1."""
    qi = {"target": n, "allowed_overlaps": max(n // 8, 1), "inserted": 0, "complete": 0}
    qc = {"target_volume": n / rho, "maximum_energy_per_site": 1000.0, "maximum_delta": 0.05, "state": 0,
          "is_final": 0, "boundary": [0.0, 0.0, 0.0]}
    for _ in range(max_steps):
        if qc["state"] == 3:
            break
        _, _, step, _ = o.state()
        if step % 10 == 0:
            if qi["complete"]:
                o.quick_compress(qc)
            else:
                o.quick_insert(qi)
        o.parallel_sweep(oracle.TRANSLATE, 0.03, 1.0, o.boundary_range)
        o.parallel_sweep(oracle.ROTATE, 0.1, 1.0, o.boundary_range)
        o.increment_step()
    return qi, qc


def test_place_orientable_hexagons_reaches_target():
    n, rho = 24, 0.9  # area fraction 0.9 x 0.6495 (the hexagon's area, 3 sqrt(3) / 8) = 0.58
    L0 = math.sqrt(n / (0.5 * rho))
    o = oracle.System(2, [L0, L0], np.zeros((0, 2)), np.zeros(0), interaction=oracle.CONVEX_POLYGON_PENALTY,
                      vertices=HEXAGON)
    qi, qc = place_orientable(o, n, rho)
    assert qi["complete"] and qc["state"] == 3 and o.n_bodies == n
    assert np.prod(o.box()) == pytest.approx(n / rho, rel=1e-12)
    assert o.total_energy() == 0.0
    pos, th, _, _ = o.state()
    hard = oracle.System(2, o.box(), pos, th, interaction=oracle.HARD_CONVEX_POLYGON, vertices=HEXAGON)
    assert hard.overlap_count() == 0
