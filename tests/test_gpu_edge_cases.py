"""Edge cases of the sweep: systems with no body and with one body, bodies at exactly the contact
distance, and batches whose replicas are empty or smaller than one body per colour. Each is
compared with the oracle's ParallelSweep (parallel_sweep.rs:390-421) or with a single system."""
import numpy as np
import pytest

import oracle
from hoomd_rs_b200 import (FP32_RECHECK, FP64, TRANSLATE, Batch, Context, HardSphere, Isotropic, LennardJones,
                           Microstate, PairwiseCutoff, Periodic, Shifted)

pytestmark = pytest.mark.gpu

PRECISIONS = [FP64, FP32_RECHECK]


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("dim", [2, 3])
def test_empty_system_sweeps(ctx, dim, precision):
    # no body: a sweep makes no trial (count.total() >= N holds at once) and moves the Counter
    g = Microstate(ctx, Periodic(1.0, [10.0] * dim), np.zeros((0, dim)), PairwiseCutoff(HardSphere(1.0)), seed=3)
    for n_sweeps, inc in ((1, True), (3, True), (2, False)):
        c = g.sweep(TRANSLATE, 0.2, 1.0, precision, n_sweeps=n_sweeps, increment_step=inc)
        assert (c.accepted, c.rejected, c.pair_checks) == (0, 0, 0)
    assert g.step() == 4 and g.substep() == 0
    assert g.overlap_count() == 0
    assert g.positions().shape == (0, dim)
    g.close()


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("dim", [2, 3])
def test_one_body_matches_oracle(ctx, dim, precision):
    # one body: one trial per sweep, accepted unless the move leaves the body's space
    pos = np.full((1, dim), 0.3)
    g = Microstate(ctx, Periodic(1.0, [6.0] * dim), pos, PairwiseCutoff(HardSphere(1.0)), seed=11)
    o = oracle.System(dim, [6.0] * dim, pos, seed=11)
    for d in (0.1, 0.9, 2.5, 0.4):
        c = g.sweep(TRANSLATE, d, 1.0, precision, n_sweeps=1, increment_step=True)
        a, r = o.parallel_sweep(oracle.TRANSLATE, d, 1.0, 1.0)
        o.increment_step()
        assert (c.accepted, c.rejected) == (a, r) and a + r == 1
    assert np.array_equal(g.positions(), o.state()[0])


@pytest.mark.parametrize("precision", PRECISIONS)
def test_pairs_at_contact_distance_match_oracle(ctx, precision):
    # a row of spheres exactly one diameter apart (|r|^2 == sigma^2 is not an overlap,
    # hard_sphere.rs): the FP32 bound sends every such pair to FP64, and the trajectory equals
    # the oracle's
    n = 12
    L = float(n)
    pos = np.zeros((n, 3))
    pos[:, 0] = -L / 2.0 + 0.5 + np.arange(n)
    g = Microstate(ctx, Periodic(1.0, [L] * 3), pos, PairwiseCutoff(HardSphere(1.0)), seed=21)
    o = oracle.System(3, [L] * 3, pos, seed=21)
    assert g.overlap_count() == 0 and o.overlap_count() == 0
    for _ in range(4):
        c = g.sweep(TRANSLATE, 0.05, 1.0, precision, n_sweeps=1, increment_step=True)
        a, r = o.parallel_sweep(oracle.TRANSLATE, 0.05, 1.0, 1.0)
        o.increment_step()
        assert (c.accepted, c.rejected) == (a, r)
    assert np.array_equal(g.positions(), o.state()[0])


@pytest.mark.parametrize("precision", PRECISIONS)
def test_batch_with_empty_and_tiny_replicas(ctx, precision):
    # replicas of 0, 1 and 3 bodies beside a regular one: each equals its single system
    rng = np.random.default_rng(5)
    specs = [(np.zeros((0, 3)), 8.0), (np.array([[0.1, 0.2, 0.3]]), 4.0),
             (np.array([[-1.0, 0.0, 0.0], [0.5, 0.5, 0.5], [1.6, -1.2, 0.4]]), 5.0),
             (rng.uniform(-4.0, 4.0, (1, 3)), 8.0)]
    reps = [{"boundary": Periodic(1.0, [L] * 3), "positions": p, "seed": 40 + k} for k, (p, L) in enumerate(specs)]
    b = Batch(ctx, reps)
    singles = [Microstate(ctx, r["boundary"], r["positions"], PairwiseCutoff(HardSphere(1.0)), seed=r["seed"])
               for r in reps]
    for _ in range(3):
        counts, _ = b.sweep(0.4, precision, increment_step=True)
        for k, m in enumerate(singles):
            c = m.sweep(TRANSLATE, 0.4, 1.0, precision, n_sweeps=1, increment_step=True)
            assert (counts[k].accepted, counts[k].rejected) == (c.accepted, c.rejected), k
    for k, m in enumerate(singles):
        assert np.array_equal(b.positions(k), m.positions()), k
    assert counts[0].accepted + counts[0].rejected == 0


@pytest.mark.parametrize("precision", PRECISIONS)
def test_lj_two_bodies_at_the_cut_off_match_oracle(ctx, precision):
    # two Lennard-Jones sites around r_cut: pairs move in and out of the cut-off, where the FP32
    # bound defers to FP64, and the decisions equal the oracle's
    pos = np.array([[0.0, 0.0, 0.0], [2.5, 0.0, 0.0]])
    h = PairwiseCutoff(Isotropic(Shifted(LennardJones(1.0, 1.0), 2.5), 2.5))
    g = Microstate(ctx, Periodic(2.5, [8.0] * 3), pos, h, seed=31)
    o = oracle.System(3, [8.0] * 3, pos, seed=31, interaction=oracle.LENNARD_JONES, lj_epsilon=1.0, lj_sigma=1.0,
                      lj_r_cut=2.5, lj_r_shift=2.5)
    for _ in range(20):
        c = g.sweep(TRANSLATE, 0.3, 1.0, precision, n_sweeps=1, increment_step=True)
        a, r = o.parallel_sweep(oracle.TRANSLATE, 0.3, 1.0, 2.5)
        o.increment_step()
        assert c.order_ambiguous == 0
        assert (c.accepted, c.rejected) == (a, r)
    assert np.array_equal(g.positions(), o.state()[0])
