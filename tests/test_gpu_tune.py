"""GPU move-size tuner (Tune::tune_with_options, hoomd-mc/src/lib.rs:430-449, tune_local.rs:21-89).

By default the device runs tune_local_trial as the reference does: every sample of every round
from the one stream Counter(step, substep, seed).make_rng(), in order (one warp), so the tuned
move size equals the oracle's restatement of that loop bit for bit. The opt-in per-sample-stream
tuner (each sample its own counter index, rounds evaluated in parallel) equals the oracle's
per-sample tuner: (a + 1.5)/(t + 1.5) is computed from the same integer counts either way.
"""
import math

import numpy as np
import pytest

import oracle
from hoomd_rs_b200 import (FP32_RECHECK, FP64, ROTATE, TRANSLATE, Context, ConvexPolygon, ConvexPolyhedron,
                           HardShape, HardSphere, Isothermal, Isotropic, LennardJones, Microstate, PairwiseCutoff,
                           ParallelSweep, Periodic, Shifted, Translate, TuneOptions, lattice)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


def both(g, o, move, om, maximum, kt, precision, target, samples, steps, per_sample):
    got = g.tune(move, maximum, kt, precision, target, samples, steps, per_sample_streams=per_sample)
    fn = o.tune if per_sample else o.tune_stream
    return got, fn(om, maximum, kt, target, samples, steps)


@pytest.mark.parametrize("per_sample", [False, True])
@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
@pytest.mark.parametrize("dim,phi", [(3, 0.5), (2, 0.7)])
def test_tune_hard_spheres_matches_oracle(ctx, dim, phi, precision, per_sample):
    pos, L = lattice.hard_sphere_box(3000, phi, dim, 0x5EED0002)
    g = Microstate(ctx, Periodic(1.0, [L] * dim), pos, PairwiseCutoff(HardSphere(1.0)), seed=77, step=3)
    o = oracle.System(dim, [L] * dim, pos, diameter=1.0, seed=77, step=3)
    got, want = both(g, o, TRANSLATE, oracle.TRANSLATE, 0.13, 1.0, precision, 0.3, 4000, 8, per_sample)
    assert got == want
    # the state is untouched
    assert np.array_equal(g.positions(), o.state()[0])


def test_tune_default_is_the_single_stream(ctx):
    # the reference's defaults (8000 samples, 32 rounds) on 3-D spheres, FCC at 0.50, from the
    # fixed size 0.13 of benchmarks/src/mc/hard_sphere.rs: the stream tuner equals the oracle's
    # single-stream loop and differs from the per-sample variant
    pos, L = lattice.hard_sphere_box(4 * 12 ** 3, 0.5, 3, 0x5EED0002, lattice="fcc")
    g = Microstate(ctx, Periodic(1.0, [L] * 3), pos, PairwiseCutoff(HardSphere(1.0)), seed=0x5EED0002)
    o = oracle.System(3, [L] * 3, pos, diameter=1.0, seed=0x5EED0002)
    got = g.tune(TRANSLATE, 0.13, 1.0, FP32_RECHECK, 0.3, 8000, 32)
    assert got == o.tune_stream(oracle.TRANSLATE, 0.13, 1.0, 0.3, 8000, 32)
    assert got != g.tune(TRANSLATE, 0.13, 1.0, FP32_RECHECK, 0.3, 8000, 32, per_sample_streams=True)


@pytest.mark.parametrize("per_sample", [False, True])
def test_tune_lennard_jones_matches_oracle(ctx, per_sample):
    pos, L = lattice.lennard_jones_box(2048, 0.8, 3, 9)
    h = PairwiseCutoff(Isotropic(Shifted(LennardJones(1.0, 1.0), 2.5), 2.5))
    g = Microstate(ctx, Periodic(2.5, [L] * 3), pos, h, seed=9, step=2)
    o = oracle.System(3, [L] * 3, pos, seed=9, step=2, interaction=oracle.LENNARD_JONES, lj_r_cut=2.5, lj_r_shift=2.5)
    got, want = both(g, o, TRANSLATE, oracle.TRANSLATE, 0.1, 1.2, FP64, 0.4, 2000, 6, per_sample)
    assert got == want


@pytest.mark.parametrize("per_sample", [False, True])
def test_tune_cube_translation_and_rotation_match_oracle(ctx, per_sample):
    cube = np.array([[x, y, z] for x in (-0.5, 0.5) for y in (-0.5, 0.5) for z in (-0.5, 0.5)])
    n, phi = 1000, 0.5
    L = (n / phi) ** (1 / 3)
    pos = lattice.cubic_lattice(n, L, 3, 4)
    g = Microstate(ctx, Periodic(math.sqrt(3), [L] * 3), pos, PairwiseCutoff(HardShape(ConvexPolyhedron(cube))),
                   seed=4)
    o = oracle.System(3, [L] * 3, pos, None, seed=4, interaction=oracle.HARD_CONVEX_POLYHEDRON, vertices=cube)
    for move, om in ((TRANSLATE, oracle.TRANSLATE), (ROTATE, oracle.ROTATE)):
        got, want = both(g, o, move, om, 0.1, 1.0, FP32_RECHECK, 0.3, 2000, 6, per_sample)
        assert got == want, move
    # Rotate<Versor>::adjust clamps the maximum at pi/2 (rotate/versor.rs:128-135): a dilute
    # state accepts nearly every rotation and the tuner grows the size up to the clamp
    dilute = lattice.cubic_lattice(64, 40.0, 3, 4)
    gd = Microstate(ctx, Periodic(math.sqrt(3), [40.0] * 3), dilute,
                    PairwiseCutoff(HardShape(ConvexPolyhedron(cube))), seed=4)
    od = oracle.System(3, [40.0] * 3, dilute, None, seed=4, interaction=oracle.HARD_CONVEX_POLYHEDRON, vertices=cube)
    got = gd.tune(ROTATE, 0.5, 1.0, FP64, 0.3, 500, 8)
    assert got == od.tune_stream(oracle.ROTATE, 0.5, 1.0, 0.3, 500, 8) == math.pi / 2


def test_tune_polygon_rotation_matches_oracle(ctx):
    square = np.array([[-0.5, -0.5], [0.5, -0.5], [0.5, 0.5], [-0.5, 0.5]])
    n, phi = 900, 0.55
    L = math.sqrt(n / phi)
    pos = lattice.cubic_lattice(n, L, 2, 8)
    g = Microstate(ctx, Periodic(math.sqrt(2), [L, L]), pos,
                   PairwiseCutoff(HardShape(ConvexPolygon.with_vertices(square))), seed=8, orientations=np.zeros(n))
    o = oracle.System(2, [L, L], pos, np.zeros(n), seed=8, interaction=oracle.HARD_CONVEX_POLYGON, vertices=square)
    for move, om in ((TRANSLATE, oracle.TRANSLATE), (ROTATE, oracle.ROTATE)):
        got, want = both(g, o, move, om, 0.2, 1.0, FP64, 0.3, 2000, 6, False)
        assert got == want, move


def test_tune_reaches_target_and_sweep_api(ctx):
    pos, L = lattice.hard_sphere_box(20000, 0.5, 3, 0x5EED0002)
    h = PairwiseCutoff(HardSphere(1.0))
    micro = Microstate(ctx, Periodic(1.0, [L] * 3), pos, h, seed=5)
    sweep = ParallelSweep(1.0, Translate.with_maximum_distance(0.13))
    sweep.tune_with_options(micro, h, Isothermal(1.0), TuneOptions(target_acceptance=0.3, samples=8000, steps=32))
    tuned = sweep.local_trial.maximum_distance
    # one more tuning round at the tuned size: its scale factor (r + 1.5) / (t + 1.5) gives the
    # single-body acceptance r the tuner measures (tune_local.rs samples bodies one at a time)
    r = micro.tune(TRANSLATE, tuned, 1.0, FP64, 0.3, 20000, 1) / tuned * 1.8 - 1.5
    assert abs(r - 0.3) < 0.02
    # the checkerboard sweep also rejects moves that leave their space, so its ratio is lower
    c = sweep.apply(micro, h, Isothermal(1.0))
    assert 0.2 < c.acceptance_ratio() < 0.3
