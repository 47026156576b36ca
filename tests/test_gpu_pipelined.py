"""Pipelined sweeps: hmc_sweep with n_sweeps > 1 and increment_step enqueues the sweeps back to
back and waits once per 64 sweeps instead of once per sweep. A sweep that needs more colour sets
than were enqueued stops the rest (their passes see kErrAborted), is completed, and the sweeps
after it are enqueued again. The trajectory, the Count and the Counter must equal those of the
same sweeps made one call at a time."""
import math

import numpy as np
import pytest

from hoomd_rs_b200 import (FP32_RECHECK, FP64, ROTATE, TRANSLATE, Context, ConvexPolygon, ConvexPolyhedron,
                           HardShape, HardSphere, Isotropic, LennardJones, Microstate, PairwiseCutoff, Periodic,
                           Shifted, lattice)

pytestmark = pytest.mark.gpu

CUBE = np.array([[x, y, z] for x in (-0.5, 0.5) for y in (-0.5, 0.5) for z in (-0.5, 0.5)])
SQUARE = np.array([[-0.5, -0.5], [0.5, -0.5], [0.5, 0.5], [-0.5, 0.5]])


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


def make(ctx, kind):
    if kind == "spheres":
        pos, L = lattice.hard_sphere_box(32768, 0.5, 3, 0x5EED0090)
        return lambda: Microstate(ctx, Periodic(1.0, [L] * 3), pos, PairwiseCutoff(HardSphere(1.0)), seed=7), 0.2
    if kind == "disks":
        pos, L = lattice.hard_sphere_box(4096, 0.7, 2, 0x5EED0091)
        return lambda: Microstate(ctx, Periodic(1.0, [L] * 2), pos, PairwiseCutoff(HardSphere(1.0)), seed=8), 0.1
    if kind == "lj":  # 14 colour sets per sweep: the first pipelined sweep needs more than enqueued
        pos, L = lattice.lennard_jones_box(8192, 0.8, 3, 0x5EED0092)
        h = PairwiseCutoff(Isotropic(Shifted(LennardJones(1.0, 1.0), 2.5), 2.5))
        return lambda: Microstate(ctx, Periodic(2.5, [L] * 3), pos, h, seed=9), 0.1
    if kind == "cubes":
        L = (4096 / 0.55) ** (1.0 / 3.0)
        pos = lattice.cubic_lattice(4096, L, 3, 0x5EED0093, jitter=0.01)
        h = PairwiseCutoff(HardShape(ConvexPolyhedron.with_vertices(CUBE)))
        return lambda: Microstate(ctx, Periodic(math.sqrt(3.0), [L] * 3), pos, h, seed=10), 0.08
    L = math.sqrt(4096 / 0.6)
    pos = lattice.cubic_lattice(4096, L, 2, 0x5EED0094, jitter=0.0)
    h = PairwiseCutoff(HardShape(ConvexPolygon.with_vertices(SQUARE)))
    return lambda: Microstate(ctx, Periodic(math.sqrt(2.0), [L, L]), pos, h, seed=11,
                              orientations=np.zeros(4096)), 0.1


def fields(c):
    return (c.accepted, c.rejected, c.rechecks, c.pair_checks, c.order_ambiguous)


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
@pytest.mark.parametrize("kind", ["spheres", "disks", "lj", "cubes", "squares"])
def test_pipelined_sweeps_equal_one_call_per_sweep(ctx, kind, precision):
    factory, d = make(ctx, kind)
    a, b = factory(), factory()
    moves = [(TRANSLATE, d)] if kind in ("spheres", "disks", "lj") else [(TRANSLATE, d), (ROTATE, 0.1)]
    for move, maximum in moves:
        n = 70 if kind in ("disks", "squares") else 5  # 70: two chunks of the pipeline
        ca = a.sweep(move, maximum, 1.0, precision, n_sweeps=n, increment_step=True)
        want = [0, 0, 0, 0, 0]
        max_err = 0.0
        for _ in range(n):
            cb = b.sweep(move, maximum, 1.0, precision, n_sweeps=1, increment_step=True)
            want = [x + y for x, y in zip(want, fields(cb))]
            max_err = max(max_err, cb.max_fp32_error)
        assert list(fields(ca)) == want, move
        assert ca.max_fp32_error == max_err
        assert (a.step(), a.substep()) == (b.step(), b.substep())
    assert np.array_equal(a.positions(), b.positions())
    if kind in ("cubes", "squares"):
        assert np.array_equal(a.orientations(), b.orientations())


def test_pipelined_sweeps_after_unincremented_ones(ctx):
    # a call that does not increment the step leaves substep > 0; the next pipelined call starts
    # from it, as the one-at-a-time sweeps do
    factory, d = make(ctx, "spheres")
    a, b = factory(), factory()
    for g in (a, b):
        g.sweep(TRANSLATE, d, 1.0, FP32_RECHECK, n_sweeps=2, increment_step=False)
    assert a.substep() > 0
    ca = a.sweep(TRANSLATE, d, 1.0, FP32_RECHECK, n_sweeps=3, increment_step=True)
    tot = [0, 0]
    for _ in range(3):
        cb = b.sweep(TRANSLATE, d, 1.0, FP32_RECHECK, n_sweeps=1, increment_step=True)
        tot = [tot[0] + cb.accepted, tot[1] + cb.rejected]
    assert [ca.accepted, ca.rejected] == tot
    assert np.array_equal(a.positions(), b.positions())
    assert (a.step(), a.substep()) == (b.step(), b.substep())
