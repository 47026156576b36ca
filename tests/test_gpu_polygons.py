"""GPU parity of the hard convex polygon sweep: Convex<ConvexPolygon> (XenoCollide in 2-D) and
ConvexSurfaceMesh2d (separating axes), with Translate<Cartesian<2>> and Rotate<Angle> moves.

The device evaluates the pair test in FP64 with the reference's expression order and
correctly rounded sin/cos, the same arithmetic as the oracle, so decisions and whole
trajectories (positions and angles) must equal the oracle's bit for bit in both precision
modes (the FP32 pass only prefilters candidates on the circumcircle distance).
"""
import math

import numpy as np
import pytest

import oracle
from hoomd_rs_b200 import (FP32_RECHECK, FP64, ROTATE, TRANSLATE, Context, ConvexPolygon, ConvexSurfaceMesh2d,
                           HardShape, HmcError, Microstate, PairwiseCutoff, Periodic, lattice)

pytestmark = pytest.mark.gpu

SQUARE = np.array([[-0.5, -0.5], [0.5, -0.5], [0.5, 0.5], [-0.5, 0.5]])
PENTAGON = np.array([[math.cos(2 * math.pi * k / 5 + 0.3), math.sin(2 * math.pi * k / 5 + 0.3)] for k in range(5)]) * 0.6
KINDS = {
    "polygon": (lambda v: ConvexPolygon.with_vertices(v), oracle.HARD_CONVEX_POLYGON),
    "surface_mesh": (lambda v: ConvexSurfaceMesh2d.from_point_set(v), oracle.HARD_CONVEX_SURFACE_MESH_2D),
}


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


def systems(ctx, kind, verts, n, spacing, seed, angles=None, positions=None, L=None):
    make_shape, okind = KINDS[kind]
    shape = make_shape(verts)
    R = shape.bounding_radius
    if positions is None:
        m = int(math.ceil(math.sqrt(n)))
        L = m * spacing * 2 * R
        positions = lattice.cubic_lattice(n, L, 2, seed, jitter=0.0)
    if angles is None:
        angles = np.random.default_rng(seed).uniform(-math.pi, math.pi, len(positions))
    g = Microstate(ctx, Periodic(2 * R, [L, L]), positions, PairwiseCutoff(HardShape(shape)), seed=seed,
                   orientations=angles)
    o = oracle.System(2, [L, L], positions, angles, seed=seed, interaction=okind, vertices=shape.vertices)
    return g, o, L, R


def test_device_sincos_is_the_oracle_sincos(ctx):
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.uniform(-10, 10, 20000), rng.uniform(-1e5, 1e5, 2000), [0.0, -0.0, 1e-300, 2.0 ** -27,
                                                                                    math.pi / 4, 1048575.5]])
    s, c = ctx.sincos(x)
    want = np.array([oracle.cr_sincos(float(v)) for v in x])
    assert np.array_equal(s, want[:, 0]) and np.array_equal(c, want[:, 1])
    with pytest.raises(HmcError):
        ctx.sincos([2.0 ** 20])


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
@pytest.mark.parametrize("kind,verts", [("polygon", PENTAGON), ("surface_mesh", SQUARE), ("polygon", SQUARE)])
def test_polygon_trajectory_bit_identical(ctx, kind, verts, precision):
    g, o, L, R = systems(ctx, kind, verts, 900, 1.02, seed=0x5EED0006)
    okind = oracle.ROTATE
    for sweep in range(8):
        move, maximum = (TRANSLATE, 0.12) if sweep % 2 == 0 else (ROTATE, 0.25)
        c = g.sweep(move, maximum, 1.0, precision, n_sweeps=1, increment_step=True)
        a, r = o.parallel_sweep(oracle.TRANSLATE if move == TRANSLATE else okind, maximum, 1.0, 2 * R)
        o.increment_step()
        assert (c.accepted, c.rejected) == (a, r), sweep
        assert 0 < a < a + r
    po, ao, _, _ = o.state()
    assert np.array_equal(g.positions(), po)
    assert np.array_equal(g.orientations(), ao.reshape(-1))
    assert g.overlap_count() == 0 == o.overlap_count()


@pytest.mark.parametrize("kind", ["polygon", "surface_mesh"])
def test_reference_polygon_cases_through_the_sweep_pair_test(ctx, golden, kind):
    # convex_polytope.rs:489-600 / convex_surface_mesh_2d.rs:1197-1330, square-square cases: body 0
    # at the origin with angle 0, a trial of body 1 at v_ij with angle theta_ij. The device and
    # the oracle must agree, and agree with the reference's expectation.
    cases = golden["convex_2d"] if kind == "polygon" else golden["surface_mesh_2d"]["cases"]
    L = 40.0
    for c in [c for c in cases if c["a"] == c["b"] == "square" and not c["symmetric"]]:
        pos = np.array([[0.0, 0.0], [7.0, 7.0]])
        g, o, _, _ = systems(ctx, kind, SQUARE, 2, 0, 1, angles=np.zeros(2), positions=pos, L=L)
        trial = np.array(c["v_ij"])
        dec, _ = g.eval_moves([1], [trial], None, 1.0, FP64, orientations=[c["theta_ij"]])
        dec32, _ = g.eval_moves([1], [trial], None, 1.0, FP32_RECHECK, orientations=[c["theta_ij"]])
        want, _ = o.eval_moves([1], [trial], [c["theta_ij"]], [0.5], 1.0)
        assert bool(dec[0]) == bool(dec32[0]) == bool(want[0]) == (not c["expected"]), c["src"]
        g.close()


@pytest.mark.parametrize("kind,verts", [("polygon", PENTAGON), ("surface_mesh", SQUARE)])
def test_random_near_contact_polygon_moves(ctx, kind, verts):
    g, o, L, R = systems(ctx, kind, verts, 1024, 1.03, seed=9)
    for sweep in range(4):
        move, maximum = (TRANSLATE, 0.15) if sweep % 2 == 0 else (ROTATE, 0.4)
        g.sweep(move, maximum, 1.0, FP64, n_sweeps=1, increment_step=True)
        o.parallel_sweep(oracle.TRANSLATE if move == TRANSLATE else oracle.ROTATE, maximum, 1.0, 2 * R)
        o.increment_step()
    pos, ang = g.positions(), g.orientations()
    rng = np.random.default_rng(4)
    m = 30_000
    bodies = rng.integers(0, 1024, m)
    js = (bodies + rng.integers(1, 1024, m)) % 1024
    v = rng.normal(size=(m, 2))
    v /= np.linalg.norm(v, axis=1)[:, None]
    near = pos[js] + v * rng.uniform(0.9 * R, 2.0 * R, m)[:, None]
    own = pos[bodies] + rng.normal(size=(m, 2)) * 0.1
    half = rng.random(m) < 0.5
    trial = np.where(half[:, None], near, own)
    lam = trial / L
    lam = lam - np.round(lam)
    trial = np.where(lam == 0.5, -0.5, lam) * L
    th = np.where(half, rng.uniform(-math.pi, math.pi, m), ang[bodies] + rng.normal(size=m) * 0.2)
    want, _ = o.eval_moves(bodies, trial, th, np.full(m, 0.5), 1.0)
    d64, _ = g.eval_moves(bodies, trial, None, 1.0, FP64, orientations=th)
    d32, _ = g.eval_moves(bodies, trial, None, 1.0, FP32_RECHECK, orientations=th)
    assert np.array_equal(d64, want), np.flatnonzero(d64 != want)[:10]
    assert np.array_equal(d32, want)
    assert 0.05 < want.mean() < 0.95


@pytest.mark.parametrize("kind", ["polygon", "surface_mesh"])
def test_planted_polygon_overlap_and_tune(ctx, kind):
    pos = np.array([[0.0, 0.0], [0.9, 0.3], [5.0, 5.0]])
    g, o, L, R = systems(ctx, kind, SQUARE, 3, 0, 1, angles=np.array([0.0, 0.2, 1.0]), positions=pos, L=14.0)
    assert g.overlap_count() == o.overlap_count() == 1
    g2, o2, _, _ = systems(ctx, kind, SQUARE, 900, 1.02, seed=21)
    for move, om in ((TRANSLATE, oracle.TRANSLATE), (ROTATE, oracle.ROTATE)):
        assert g2.tune(move, 0.1, 1.0, FP32_RECHECK, 0.3, 2000, 6) == o2.tune_stream(om, 0.1, 1.0, 0.3, 2000, 6)


def test_polygon_input_validation(ctx):
    h = PairwiseCutoff(HardShape(ConvexSurfaceMesh2d(SQUARE[::-1].copy())))  # clockwise: rejected
    with pytest.raises(HmcError):
        Microstate(ctx, Periodic(1.5, [10.0, 10.0]), np.zeros((1, 2)), h)
    h = PairwiseCutoff(HardShape(ConvexPolygon.with_vertices(SQUARE)))
    with pytest.raises(HmcError):
        Microstate(ctx, Periodic(1.5, [10.0, 10.0]), np.zeros((1, 2)), h, orientations=[1e6])


ROD2 = np.array([[-1.5, -0.15], [1.5, -0.15], [1.5, 0.15], [-1.5, 0.15]])


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
@pytest.mark.parametrize("kind", ["polygon", "surface_mesh"])
def test_rod_trajectory_with_long_pair_lists(ctx, kind, precision):
    # Thin rectangles on a tight lattice: ~28 neighbours of a trial lie inside its circumcircle,
    # so the four trials of a warp usually list more pairs for the full test than the warp's
    # list holds, and the pass drains it before the stencil walk ends. The trajectory must equal
    # the oracle's.
    make_shape, okind = KINDS[kind]
    shape = make_shape(ROD2)
    nx, ny = 8, 40
    a = np.array([3.1, 0.33])
    L = a * np.array([nx, ny])
    idx = np.indices([nx, ny]).reshape(2, -1).T.astype(np.float64)
    pos = -L / 2 + (idx + 0.5) * a
    R = shape.bounding_radius
    ang = np.zeros(len(pos))
    g = Microstate(ctx, Periodic(2 * R, list(L)), pos, PairwiseCutoff(HardShape(shape)), seed=0x5EED0014,
                   orientations=ang)
    o = oracle.System(2, list(L), pos, ang, seed=0x5EED0014, interaction=okind, vertices=shape.vertices)
    for sweep in range(6):
        move, maximum = (TRANSLATE, 0.05) if sweep % 2 == 0 else (ROTATE, 0.03)
        c = g.sweep(move, maximum, 1.0, precision, n_sweeps=1, increment_step=True)
        acc, rej = o.parallel_sweep(oracle.TRANSLATE if move == TRANSLATE else oracle.ROTATE, maximum, 1.0, 2 * R)
        o.increment_step()
        assert (c.accepted, c.rejected) == (acc, rej), sweep
        assert 0 < acc < acc + rej
    po, ao, _, _ = o.state()
    assert np.array_equal(g.positions(), po)
    assert np.array_equal(g.orientations(), ao.reshape(-1))
    assert g.overlap_count() == 0 == o.overlap_count()
