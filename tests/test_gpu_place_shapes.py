"""Preparing states of oriented convex shapes on the GPU against the oracle: the insertion
hamiltonian PairwiseCutoff(Anisotropic(ApproximateShapeOverlap(Convex(shape), OverlapPenalty,
resolution))) (hoomd-interaction/src/pairwise/approximate_shape_overlap.rs), its ParallelSweep
(translation and rotation), QuickInsert with uniform random orientations and QuickCompress, and
the benchmark placement loop built from them (benchmarks/src/place.rs:120-219). Positions,
orientations, counters and boxes must equal the oracle's bit for bit (the ParallelSweep sums
the pair energies in another order than the oracle; a decision could differ only where the
order bound says so, and those are counted)."""
import math

import numpy as np
import pytest

import oracle
from hoomd_rs_b200 import (FP32_RECHECK, FP64, ROTATE, TRANSLATE, Anisotropic, ApproximateShapeOverlap, Context,
                           ConvexPolygon, ConvexPolyhedron, ConvexSurfaceMesh2d, HardShape, HmcError, Microstate,
                           OverlapPenalty, PairwiseCutoff, Periodic, QuickCompress, QuickInsert,
                           place_single_site_orientable_bodies)

pytestmark = pytest.mark.gpu

CUBE = np.array([[x, y, z] for x in (-0.5, 0.5) for y in (-0.5, 0.5) for z in (-0.5, 0.5)])


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


def hexagon():
    return ConvexPolygon.regular(6)


def hamiltonians(shape, resolution=0.01, penalty=None):
    hard = PairwiseCutoff(HardShape(shape))
    r_cut = hard.maximum_interaction_range
    soft = PairwiseCutoff(Anisotropic(ApproximateShapeOverlap.new(shape, penalty or OverlapPenalty(), resolution),
                                      r_cut))
    return hard, soft


def oracle_kind(shape):
    return oracle.CONVEX_POLYHEDRON_PENALTY if isinstance(shape, ConvexPolyhedron) else oracle.CONVEX_POLYGON_PENALTY


def test_pair_energy_known_answers(ctx):
    # approximate_shape_overlap.rs:75-121: hexagons >= 100 at 0.6, finite at 0.9, 0 at 1.0 (r_cut 1)
    hard, soft = hamiltonians(hexagon())
    for x in (0.55, 0.6, 0.9, 0.97, 1.0):
        g = Microstate(ctx, Periodic(1.0, [10.0, 10.0]), [[0.0, 0.0], [x, 0.0]], hard, orientations=[0.0, 0.3])
        g.set_hamiltonian(soft)
        o = oracle.System(2, [10.0, 10.0], [[0.0, 0.0], [x, 0.0]], [0.0, 0.3], interaction=oracle.CONVEX_POLYGON_PENALTY,
                          vertices=hexagon().vertices, r_cut=1.0)
        assert g.total_energy() == o.total_energy(), x
    g = Microstate(ctx, Periodic(1.0, [10.0, 10.0]), [[0.0, 0.0], [0.6, 0.0]], hard)
    g.set_hamiltonian(soft)
    assert g.total_energy() >= 100.0
    g.set_hamiltonian(hard)
    assert g.total_energy() == math.inf  # HardShape again


def test_cube_pair_energies_equal_the_oracle(ctx):
    hard, soft = hamiltonians(ConvexPolyhedron.with_vertices(CUBE))
    rng = np.random.default_rng(3)
    for _ in range(40):
        d = rng.normal(size=3)
        d *= rng.uniform(0.6, 1.8) / np.linalg.norm(d)
        q = rng.normal(size=(2, 4))
        q /= np.linalg.norm(q, axis=1, keepdims=True)
        pos = [[0.0, 0.0, 0.0], list(d)]
        g = Microstate(ctx, Periodic(math.sqrt(3.0), [12.0] * 3), pos, hard, orientations=q)
        g.set_hamiltonian(soft)
        o = oracle.System(3, [12.0] * 3, pos, q, interaction=oracle.CONVEX_POLYHEDRON_PENALTY, vertices=CUBE)
        assert g.total_energy() == o.total_energy()


def pair_systems(ctx, shape, n, rho, dim, seed):
    hard, soft = hamiltonians(shape)
    L0 = (n / (0.5 * rho)) ** (1.0 / dim)
    r = hard.maximum_interaction_range
    g = Microstate(ctx, Periodic(r, [L0] * dim), np.zeros((0, dim)), hard, seed=seed, capacity=n,
                   body_interaction_range=r)
    g.set_hamiltonian(soft)
    o = oracle.System(dim, [L0] * dim, np.zeros((0, dim)), np.zeros((0, 4)) if dim == 3 else np.zeros(0), seed=seed,
                      interaction=oracle_kind(shape), vertices=shape.vertices)
    return g, o, hard, soft


def same_state(g, o):
    po, oo, step, sub = o.state()
    assert g.n == o.n_bodies
    assert np.array_equal(g.positions(), po)
    ori = g.orientations()
    assert np.array_equal(ori, oo.reshape(ori.shape))
    assert g._counter() == (step, sub)
    assert np.array_equal(g.box(), o.box())


@pytest.mark.parametrize("kind", ["hexagons", "cubes"])
def test_placement_loop_bit_identical(ctx, kind):
    # place.rs:120-219 step by step on both sides
    shape, n, rho, dim = {"hexagons": (hexagon(), 24, 0.9, 2),
                          "cubes": (ConvexPolyhedron.with_vertices(CUBE), 48, 0.45, 3)}[kind]
    g, o, hard, soft = pair_systems(ctx, shape, n, rho, dim, 0x5EED0041)
    qi, qc = QuickInsert.new(n), QuickCompress.with_target_volume(n / rho)
    oqi = {"target": n, "allowed_overlaps": max(n // 8, 1), "inserted": 0, "complete": 0}
    oqc = {"target_volume": n / rho, "maximum_energy_per_site": 1000.0, "maximum_delta": 0.05, "state": 0,
           "is_final": 0, "boundary": [0.0, 0.0, 0.0]}
    ambiguous, steps = 0, 0
    for step in range(20000):
        if qc.is_complete():
            break
        if step % 10 == 0:
            if qi.is_complete():
                qc.apply(g)
                o.quick_compress(oqc)
                assert qc.state == oqc["state"]
            else:
                qi.apply(g)
                o.quick_insert(oqi)
                assert qi.inserted == oqi["inserted"]
        for mv, omv, m in ((TRANSLATE, oracle.TRANSLATE, 0.03), (ROTATE, oracle.ROTATE, 0.1)):
            c = g.sweep(mv, m, 1.0, FP64)
            a, r = o.parallel_sweep(omv, m, 1.0, o.boundary_range)
            ambiguous += c.order_ambiguous
            if ambiguous == 0:
                assert (c.accepted, c.rejected) == (a, r), step
        g.increment_step()
        o.increment_step()
        steps = step
        if step % 50 == 0 and ambiguous == 0:
            same_state(g, o)
    assert ambiguous == 0
    assert qc.is_complete() and oqc["state"] == 3, steps
    same_state(g, o)
    assert g.total_energy() == 0.0 == o.total_energy()
    g.set_hamiltonian(hard)
    assert g.overlap_count() == 0


def test_fp32_mode_runs_fp64(ctx):
    # the insertion hamiltonian has no FP32 path: both precision modes give the same trajectory
    shape = ConvexPolyhedron.with_vertices(CUBE)
    hard, soft = hamiltonians(shape)
    rng = np.random.default_rng(9)
    L = 7.0
    pos = (rng.random((150, 3)) - 0.5) * L
    q = rng.normal(size=(150, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    out = []
    for prec in (FP64, FP32_RECHECK):
        g = Microstate(ctx, Periodic(math.sqrt(3.0), [L] * 3), pos, hard, orientations=q, seed=4)
        g.set_hamiltonian(soft)
        counts = [(c.accepted, c.rejected) for c in
                  (g.sweep(mv, m, 1.0, prec, increment_step=True) for mv, m in [(TRANSLATE, 0.05), (ROTATE, 0.1)] * 3)]
        out.append((counts, g.positions(), g.orientations()))
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][2], out[1][2])


def test_place_cubes_on_the_device(ctx):
    # 2048 cubes to packing fraction 0.50 under the insertion hamiltonian; no hard overlap after
    shape = ConvexPolyhedron.with_vertices(CUBE)
    hard, soft = hamiltonians(shape)
    n, rho = 2048, 0.50
    g = place_single_site_orientable_bodies(ctx, n, rho, hard.maximum_interaction_range, soft, hard, 3, seed=11)
    assert g.n == n
    assert g.volume() == pytest.approx(n / rho, rel=1e-12)
    assert g.overlap_count() == 0
    q = g.orientations()
    assert np.allclose(np.linalg.norm(q, axis=1), 1.0, atol=1e-12)


def test_entry_points_and_errors(ctx):
    hard, soft = hamiltonians(ConvexPolyhedron.with_vertices(CUBE))
    g = Microstate(ctx, Periodic(math.sqrt(3.0), [6.0] * 3), [[0.0, 0.0, 0.0]], hard)
    g.set_hamiltonian(soft)
    with pytest.raises(HmcError):  # the serial sweep runs under HardShape only
        g.serial_sweep(0.1)
    # r_cut beyond the shape's range, a resolution finer than the device loop's bound
    too_far = PairwiseCutoff(Anisotropic(soft.pair.interaction, 2.0))
    with pytest.raises(HmcError):
        g.set_hamiltonian(too_far)
    fine = PairwiseCutoff(Anisotropic(ApproximateShapeOverlap.new(soft.pair.interaction.shape, OverlapPenalty(),
                                                                  1e-9), math.sqrt(3.0)))
    with pytest.raises(HmcError):
        g.set_hamiltonian(fine)
    # the shape of the insertion hamiltonian must be the system's own
    other = ConvexPolyhedron.with_vertices(1.1 * CUBE)
    with pytest.raises(HmcError):
        g.set_hamiltonian(PairwiseCutoff(Anisotropic(ApproximateShapeOverlap.new(other, OverlapPenalty(), 0.01),
                                                     math.sqrt(3.0))))


def hexagon_mesh():
    return ConvexSurfaceMesh2d.from_point_set(ConvexPolygon.regular(6).vertices)


def test_mesh_pair_energies_equal_the_oracle(ctx):
    # ConvexSurfaceMesh2d: the separating-axis test without bounding circles in intersects_at
    mesh = hexagon_mesh()
    hard, soft = hamiltonians(mesh)
    r_cut = hard.maximum_interaction_range
    rng = np.random.default_rng(5)
    for _ in range(60):
        d = rng.normal(size=2)
        d *= rng.uniform(0.3, 1.05) / np.linalg.norm(d)
        th = rng.uniform(0.0, 2.0 * math.pi, 2)
        pos = [[0.0, 0.0], list(d)]
        g = Microstate(ctx, Periodic(r_cut, [8.0, 8.0]), pos, hard, orientations=th)
        g.set_hamiltonian(soft)
        o = oracle.System(2, [8.0, 8.0], pos, th, interaction=oracle.SURFACE_MESH_2D_PENALTY, vertices=mesh.vertices,
                          r_cut=r_cut)
        assert g.total_energy() == o.total_energy()
        g.close()


def test_mesh_placement_loop_bit_identical(ctx):
    mesh = hexagon_mesh()
    n, rho = 24, 0.9
    hard, soft = hamiltonians(mesh)
    L0 = (n / (0.5 * rho)) ** 0.5
    r = hard.maximum_interaction_range
    g = Microstate(ctx, Periodic(r, [L0, L0]), np.zeros((0, 2)), hard, seed=0x5EED0042, capacity=n)
    g.set_hamiltonian(soft)
    o = oracle.System(2, [L0, L0], np.zeros((0, 2)), np.zeros(0), seed=0x5EED0042,
                      interaction=oracle.SURFACE_MESH_2D_PENALTY, vertices=mesh.vertices)
    qi, qc = QuickInsert.new(n), QuickCompress.with_target_volume(n / rho)
    oqi = {"target": n, "allowed_overlaps": max(n // 8, 1), "inserted": 0, "complete": 0}
    oqc = {"target_volume": n / rho, "maximum_energy_per_site": 1000.0, "maximum_delta": 0.05, "state": 0,
           "is_final": 0, "boundary": [0.0, 0.0, 0.0]}
    for step in range(20000):
        if qc.is_complete():
            break
        if step % 10 == 0:
            if qi.is_complete():
                qc.apply(g)
                o.quick_compress(oqc)
            else:
                qi.apply(g)
                o.quick_insert(oqi)
        for mv, omv, m in ((TRANSLATE, oracle.TRANSLATE, 0.03), (ROTATE, oracle.ROTATE, 0.1)):
            c = g.sweep(mv, m, 1.0, FP64)
            a, rj = o.parallel_sweep(omv, m, 1.0, o.boundary_range)
            assert c.order_ambiguous == 0
            assert (c.accepted, c.rejected) == (a, rj), step
        g.increment_step()
        o.increment_step()
    assert qc.is_complete() and oqc["state"] == 3
    same_state(g, o)
    g.set_hamiltonian(hard)
    assert g.overlap_count() == 0


def test_place_hexagons_benchmark_density(ctx):
    # benchmarks/src/mc/regular_polygon.rs:187-244: ConvexSurfaceMesh2d hexagons placed at packing
    # fraction 0.68 under the approximate shape overlap (1024 here); no hard overlap after
    mesh = hexagon_mesh()
    hard, soft = hamiltonians(mesh)
    area = 1.5 * math.sqrt(3.0) * 0.25  # regular hexagon of circumradius 0.5
    n = 1024
    g = place_single_site_orientable_bodies(ctx, n, 0.68 / area, hard.maximum_interaction_range, soft, hard, 2,
                                            seed=12)
    assert g.n == n and g.overlap_count() == 0
