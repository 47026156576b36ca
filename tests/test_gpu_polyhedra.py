"""GPU parity of the hard convex polyhedron sweep (cubes) with translation and rotation moves.

The device runs XenoCollide in FP64 with the reference's expression order, so decisions and
whole trajectories (positions and versors) must equal the oracle's bit for bit, in both
precision modes (the FP32 pass only prefilters candidates on the circumsphere distance).
"""
import math

import numpy as np
import pytest

import oracle
from hoomd_rs_b200 import (FP32_RECHECK, FP64, ROTATE, TRANSLATE, Context, ConvexPolyhedron, HardShape, Microstate,
                           PairwiseCutoff, Periodic, lattice)

pytestmark = pytest.mark.gpu

CUBE = np.array([[x, y, z] for x in (-0.5, 0.5) for y in (-0.5, 0.5) for z in (-0.5, 0.5)])


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


def cube_systems(ctx, n, phi, seed, orientations=None, positions=None, L=None):
    if positions is None:
        L = (n / phi) ** (1.0 / 3.0)
        positions = lattice.cubic_lattice(n, L, 3, seed, jitter=0.01)
    h = PairwiseCutoff(HardShape(ConvexPolyhedron.with_vertices(CUBE)))
    rng = math.sqrt(3.0)
    g = Microstate(ctx, Periodic(rng, [L] * 3), positions, h, seed=seed, orientations=orientations)
    o = oracle.System(3, [L] * 3, positions, orientations, seed=seed, interaction=oracle.HARD_CONVEX_POLYHEDRON,
                      vertices=CUBE)
    return g, o, L


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
def test_cube_trajectory_bit_identical(ctx, precision):
    g, o, L = cube_systems(ctx, 1728, 0.50, seed=0x5EED0003)
    for sweep in range(8):
        move, maximum = (TRANSLATE, 0.08) if sweep % 2 == 0 else (ROTATE, 0.1)
        c = g.sweep(move, maximum, 1.0, precision, n_sweeps=1, increment_step=True)
        a, r = o.parallel_sweep(oracle.TRANSLATE if move == TRANSLATE else oracle.ROTATE, maximum, 1.0, math.sqrt(3.0))
        o.increment_step()
        assert (c.accepted, c.rejected) == (a, r), sweep
    po, qo, _, _ = o.state()
    assert np.array_equal(g.positions(), po)
    assert np.array_equal(g.orientations(), qo)
    assert g.overlap_count() == 0 == o.overlap_count()
    q = g.orientations()
    assert np.abs(np.linalg.norm(q, axis=1) - 1).max() < 1e-12  # versors compose without renormalising


def _versor(factors):
    q = np.array([1.0, 0.0, 0.0, 0.0])
    for axis, angle in factors:
        q = oracle.versor_combine(q, oracle.versor_from_axis_angle(axis, angle))
    return q


def test_reference_cube_cases_through_the_sweep_pair_test(ctx, golden):
    # convex_polytope.rs:784-879 with q_a = identity, placed as body 0 at the origin and a
    # trial of body 1 at r_ab: accepted exactly when the reference says no overlap.
    cases = [c for c in golden["convex_3d"] if c["shape"] == "cube"]
    L = 12.0
    for c in cases:
        qb = _versor(c["q_b"])
        pos = np.array([[0.0, 0.0, 0.0], [4.0, 4.0, 4.0]])
        g, o, _ = cube_systems(ctx, 2, 0, 1, positions=pos, L=L)
        r = np.array(c["r_ab"])
        lam = r / L
        lam = lam - np.round(lam)
        trial = np.where(lam == 0.5, -0.5, lam) * L
        dec, _ = g.eval_moves([1], [trial], None, 1.0, FP64, orientations=[qb])
        dec32, _ = g.eval_moves([1], [trial], None, 1.0, FP32_RECHECK, orientations=[qb])
        want, _ = o.eval_moves([1], [trial], [qb], [0.5], 1.0)
        assert bool(dec[0]) == bool(dec32[0]) == bool(want[0]) == (not c["expected"]), c["src"]
        g.close()


def test_random_near_contact_cube_moves(ctx):
    g, o, L = cube_systems(ctx, 1000, 0.45, seed=9)
    for sweep in range(4):
        move, maximum = (TRANSLATE, 0.1) if sweep % 2 == 0 else (ROTATE, 0.2)
        g.sweep(move, maximum, 1.0, FP64, n_sweeps=1, increment_step=True)
        o.parallel_sweep(oracle.TRANSLATE if move == TRANSLATE else oracle.ROTATE, maximum, 1.0, math.sqrt(3.0))
        o.increment_step()
    pos = g.positions()
    ori = g.orientations()
    rng = np.random.default_rng(3)
    m = 20_000
    bodies = rng.integers(0, 1000, m)
    # half: the body placed next to another at a random orientation (mostly overlapping);
    # half: a small displacement and rotation of its own pose (often free, often touching)
    js = (bodies + rng.integers(1, 1000, m)) % 1000
    v = rng.normal(size=(m, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    near = pos[js] + v * rng.uniform(0.95, 1.75, m)[:, None]
    own = pos[bodies] + rng.normal(size=(m, 3)) * 0.15
    half = rng.random(m) < 0.5
    trial = np.where(half[:, None], near, own)
    lam = trial / L
    lam = lam - np.round(lam)
    trial = np.where(lam == 0.5, -0.5, lam) * L
    qr = rng.normal(size=(m, 4))
    qr /= np.linalg.norm(qr, axis=1)[:, None]
    dq = np.concatenate([np.ones((m, 1)), rng.normal(size=(m, 3)) * 0.1], axis=1)
    dq /= np.linalg.norm(dq, axis=1)[:, None]
    qown = np.array([oracle.versor_combine(dq[i], ori[bodies[i]]) for i in range(m)])
    q = np.where(half[:, None], qr, qown)
    want, _ = o.eval_moves(bodies, trial, q, np.full(m, 0.5), 1.0)
    d64, _ = g.eval_moves(bodies, trial, None, 1.0, FP64, orientations=q)
    d32, _ = g.eval_moves(bodies, trial, None, 1.0, FP32_RECHECK, orientations=q)
    assert np.array_equal(d64, want), np.flatnonzero(d64 != want)[:10]
    assert np.array_equal(d32, want)
    assert 0.05 < want.mean() < 0.95


def test_planted_cube_overlap(ctx):
    pos = np.array([[0.0, 0.0, 0.0], [0.9, 0.2, 0.0], [5.0, 5.0, 5.0]])
    g, o, _ = cube_systems(ctx, 3, 0, 1, positions=pos, L=14.0)
    assert g.overlap_count() == o.overlap_count() == 1


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
def test_cube_overlapping_passes_equal_serialised_passes(ctx, monkeypatch, precision):
    # colour passes launched while the previous one finishes give the serialised trajectory
    n, phi = 1 << 15, 0.55
    L = (n / phi) ** (1.0 / 3.0)
    pos = lattice.cubic_lattice(n, L, 3, 0x5EED0003, jitter=0.0)
    h = PairwiseCutoff(HardShape(ConvexPolyhedron.with_vertices(CUBE)))
    monkeypatch.setenv("HMC_B200_PDL", "1")
    a = Microstate(ctx, Periodic(math.sqrt(3.0), [L] * 3), pos, h, seed=0x5EED0003)
    monkeypatch.setenv("HMC_B200_PDL", "0")
    b = Microstate(ctx, Periodic(math.sqrt(3.0), [L] * 3), pos, h, seed=0x5EED0003)
    for move, maximum in [(TRANSLATE, 0.08), (ROTATE, 0.1), (TRANSLATE, 0.08)]:
        ca = a.sweep(move, maximum, 1.0, precision, n_sweeps=1, increment_step=True)
        cb = b.sweep(move, maximum, 1.0, precision, n_sweeps=1, increment_step=True)
        assert (ca.accepted, ca.rejected) == (cb.accepted, cb.rejected)
    assert np.array_equal(a.positions(), b.positions())
    assert np.array_equal(a.orientations(), b.orientations())


ROD = np.array([[x, y, z] for x in (-1.5, 1.5) for y in (-0.15, 0.15) for z in (-0.15, 0.15)])


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
def test_rod_trajectory_with_long_pair_lists(ctx, precision):
    # Thin rods on a tight lattice: a trial has hundreds of neighbours inside its circumsphere,
    # so the four trials of a warp list far more pairs for the full test than the warp's list
    # holds and the pass drains it many times per trial; the two-space y and z axes make every
    # stencil row cover its whole axis. The trajectory must equal the oracle's.
    nx, ny = 8, 18
    a = np.array([3.1, 0.35, 0.35])
    L = a * np.array([nx, ny, ny])
    idx = np.indices([nx, ny, ny]).reshape(3, -1).T.astype(np.float64)
    pos = -L / 2 + (idx + 0.5) * a
    R = float(np.linalg.norm(ROD[0]))
    h = PairwiseCutoff(HardShape(ConvexPolyhedron.with_vertices(ROD)))
    g = Microstate(ctx, Periodic(2 * R, list(L)), pos, h, seed=0x5EED0013)
    o = oracle.System(3, list(L), pos, None, seed=0x5EED0013, interaction=oracle.HARD_CONVEX_POLYHEDRON, vertices=ROD)
    for sweep in range(4):
        move, maximum = (TRANSLATE, 0.04) if sweep % 2 == 0 else (ROTATE, 0.03)
        c = g.sweep(move, maximum, 1.0, precision, n_sweeps=1, increment_step=True)
        acc, rej = o.parallel_sweep(oracle.TRANSLATE if move == TRANSLATE else oracle.ROTATE, maximum, 1.0, 2 * R)
        o.increment_step()
        assert (c.accepted, c.rejected) == (acc, rej), sweep
        assert 0 < acc < acc + rej
    po, qo, _, _ = o.state()
    assert np.array_equal(g.positions(), po)
    assert np.array_equal(g.orientations(), qo)
    assert g.overlap_count() == 0 == o.overlap_count()
