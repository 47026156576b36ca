"""GPU move-size tuner (Tune::tune_with_options, hoomd-mc/src/lib.rs:430-449, tune_local.rs:21-89).

With per-sample counter streams shared by device and oracle, every sampled decision is the
same on both, so the tuned move size is identical: (a + 1.5)/(t + 1.5) is computed from
the same integer counts.
"""
import math

import numpy as np
import pytest

import oracle
from hoomd_rs_b200 import (FP32_RECHECK, FP64, ROTATE, TRANSLATE, Context, ConvexPolyhedron, HardShape, HardSphere,
                           Isothermal, Microstate, PairwiseCutoff, ParallelSweep, Periodic, Translate, TuneOptions,
                           lattice)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
@pytest.mark.parametrize("dim,phi", [(3, 0.5), (2, 0.7)])
def test_tune_hard_spheres_matches_oracle(ctx, dim, phi, precision):
    pos, L = lattice.hard_sphere_box(3000, phi, dim, 0x5EED0002)
    g = Microstate(ctx, Periodic(1.0, [L] * dim), pos, PairwiseCutoff(HardSphere(1.0)), seed=77, step=3)
    o = oracle.System(dim, [L] * dim, pos, diameter=1.0, seed=77, step=3)
    got = g.tune(TRANSLATE, 0.13, 1.0, precision, 0.3, 4000, 8)
    want = o.tune(oracle.TRANSLATE, 0.13, 1.0, 0.3, 4000, 8)
    assert got == want
    # the state is untouched
    assert np.array_equal(g.positions(), o.state()[0])


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


def test_tune_cube_rotation_matches_oracle(ctx):
    cube = np.array([[x, y, z] for x in (-0.5, 0.5) for y in (-0.5, 0.5) for z in (-0.5, 0.5)])
    n, phi = 1000, 0.5
    L = (n / phi) ** (1 / 3)
    pos = lattice.cubic_lattice(n, L, 3, 4)
    g = Microstate(ctx, Periodic(math.sqrt(3), [L] * 3), pos, PairwiseCutoff(HardShape(ConvexPolyhedron(cube))),
                   seed=4)
    o = oracle.System(3, [L] * 3, pos, None, seed=4, interaction=oracle.HARD_CONVEX_POLYHEDRON, vertices=cube)
    for move, om in ((TRANSLATE, oracle.TRANSLATE), (ROTATE, oracle.ROTATE)):
        assert g.tune(move, 0.1, 1.0, FP32_RECHECK, 0.3, 2000, 6) == o.tune(om, 0.1, 1.0, 0.3, 2000, 6)
