"""The serial Sweep (Sweep::apply_with_filter, hoomd-mc/src/sweep.rs:159-224) on the device.

One sequential random stream drives trials of the bodies in index order, each seeing every
earlier accepted move; the device must reproduce the oracle's chain bit for bit, with and
without a should_move_body filter, and leave a state the checkerboard sweep continues from.
"""
import numpy as np
import pytest

import oracle
from hoomd_rs_b200 import (FP32_RECHECK, TRANSLATE, Context, HardSphere, Microstate, PairwiseCutoff, Periodic,
                           lattice)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


def pair(ctx, dim, n, phi, seed, kind="auto"):
    pos, L = lattice.hard_sphere_box(n, phi, dim, seed, lattice=kind)
    g = Microstate(ctx, Periodic(1.0, [L] * dim), pos, PairwiseCutoff(HardSphere(1.0)), seed=seed, step=2)
    o = oracle.System(dim, [L] * dim, pos, seed=seed, step=2)
    return g, o


@pytest.mark.parametrize("dim,n,phi,d,kind", [(2, 1000, 0.60, 0.15, "auto"), (3, 2000, 0.45, 0.2, "auto"),
                                              (3, 8, 0.30, 0.3, "cubic")])
def test_serial_sweep_bit_identical(ctx, dim, n, phi, d, kind):
    g, o = pair(ctx, dim, n, phi, 61, kind)
    for _ in range(5):
        c = g.serial_sweep(d, increment_step=True)
        a, r = o.serial_sweep(oracle.TRANSLATE, d, 1.0)
        o.increment_step()
        assert (c.accepted, c.rejected) == (a, r)
    assert np.array_equal(g.positions(), o.state()[0])
    assert (g.step(), g.substep()) == (o.state()[2], o.state()[3])


def test_serial_sweep_filter_and_checkerboard_continuation(ctx):
    g, o = pair(ctx, 3, 1500, 0.48, 62)
    mask = (np.arange(1500) % 3) != 1
    c = g.serial_sweep(0.2, move_mask=mask)
    a, r = o.serial_sweep(oracle.TRANSLATE, 0.2, 1.0, mask=mask)
    assert (c.accepted, c.rejected) == (a, r) and a + r == mask.sum()
    start = o.state()[0]
    assert np.array_equal(g.positions(), start)
    # substep advanced once: the checkerboard sweep continues from the same counter
    c = g.sweep(TRANSLATE, 0.2, 1.0, FP32_RECHECK, n_sweeps=1, increment_step=True)
    a, r = o.parallel_sweep(oracle.TRANSLATE, 0.2, 1.0, 1.0)
    o.increment_step()
    assert (c.accepted, c.rejected) == (a, r)
    assert np.array_equal(g.positions(), o.state()[0])
    assert g.overlap_count() == 0
