"""GPU trajectories against the oracle at the configured workload sizes.

The smaller parity tests compare with the oracle up to a few thousand bodies; these run the
oracle's ParallelSweep (parallel_sweep.rs:390-421) on every host thread beside the GPU sweep at
the sizes the workloads are quoted on, so that what only appears at scale is compared too: colour
lists over hundreds of thousands of spaces, 32-bit slot offsets, the wrapped rows of 102^3 spaces
and the second colour set of a sweep. Each sweep's Count and the final state (positions and, for
cubes, versors) must equal the oracle's bit for bit, in both precision modes.
"""
import math
import os

import numpy as np
import pytest

import oracle
from hoomd_rs_b200 import (FP32_RECHECK, FP64, ROTATE, TRANSLATE, Context, ConvexPolyhedron, HardShape,
                           HardSphere, Isotropic, LennardJones, Microstate, PairwiseCutoff, Periodic, Shifted,
                           lattice)

pytestmark = pytest.mark.gpu

THREADS = max(1, os.cpu_count() or 1)
CUBE = np.array([[x, y, z] for x in (-0.5, 0.5) for y in (-0.5, 0.5) for z in (-0.5, 0.5)])


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


def sweep_both(g, o, moves, kt, precision, body_range):
    ambiguous = 0
    for move, maximum in moves:
        c = g.sweep(move, maximum, kt, precision, n_sweeps=1, increment_step=True)
        a, r = o.parallel_sweep(oracle.TRANSLATE if move == TRANSLATE else oracle.ROTATE, maximum, kt, body_range,
                                threads=THREADS)
        o.increment_step()
        assert (c.accepted, c.rejected) == (a, r), (move, maximum)
        ambiguous += c.order_ambiguous
    return ambiguous


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
def test_hard_spheres_2p20(ctx, precision):
    # 3-D hard spheres, N = 2^20, packing fraction 0.50, FCC start: 102^3 spaces, two colour
    # sets per sweep; the move size the bench's tuner picks (~0.235) and a larger one.
    pos, L = lattice.hard_sphere_box(1 << 20, 0.50, 3, 0x5EED0002)
    h = PairwiseCutoff(HardSphere(1.0))
    g = Microstate(ctx, Periodic(1.0, [L] * 3), pos, h, seed=0x5EED0002)
    o = oracle.System(3, [L] * 3, pos, diameter=1.0, seed=0x5EED0002)
    sweep_both(g, o, [(TRANSLATE, 0.235), (TRANSLATE, 0.235), (TRANSLATE, 0.4)], 1.0, precision, 1.0)
    assert np.array_equal(g.positions(), o.state()[0])
    assert g.overlap_count() == 0


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
def test_hard_disks_4096_thousand_sweeps(ctx, precision):
    # 2-D hard disks, N = 4096, area fraction 0.70, square-lattice start, translation 0.1:
    # 1000 ParallelSweep applies, compared after every 100.
    pos, L = lattice.hard_sphere_box(4096, 0.70, 2, 0x5EED0001)
    h = PairwiseCutoff(HardSphere(1.0))
    g = Microstate(ctx, Periodic(1.0, [L, L]), pos, h, seed=0x5EED0001)
    o = oracle.System(2, [L, L], pos, diameter=1.0, seed=0x5EED0001)
    acc = 0
    for block in range(10):
        c = g.sweep(TRANSLATE, 0.1, 1.0, precision, n_sweeps=100, increment_step=True)
        a = r = 0
        for _ in range(100):
            da, dr = o.parallel_sweep(oracle.TRANSLATE, 0.1, 1.0, 1.0)
            o.increment_step()
            a, r = a + da, r + dr
        assert (c.accepted, c.rejected) == (a, r), block
        acc += a
        assert np.array_equal(g.positions(), o.state()[0]), block
    assert acc > 0
    assert g.overlap_count() == 0 == o.overlap_count()


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
def test_hard_cubes_2p18(ctx, precision):
    # Cubes, N = 2^18, packing fraction 0.55, simple-cubic start with identity versors:
    # translate 0.08, rotate 0.1 (Gaussian sigma), twice each.
    n, phi, seed = 1 << 18, 0.55, 0x5EED0003
    L = (n / phi) ** (1.0 / 3.0)
    positions = lattice.cubic_lattice(n, L, 3, seed, jitter=0.01)
    h = PairwiseCutoff(HardShape(ConvexPolyhedron.with_vertices(CUBE)))
    g = Microstate(ctx, Periodic(math.sqrt(3.0), [L] * 3), positions, h, seed=seed)
    o = oracle.System(3, [L] * 3, positions, None, seed=seed, interaction=oracle.HARD_CONVEX_POLYHEDRON,
                      vertices=CUBE)
    sweep_both(g, o, [(TRANSLATE, 0.08), (ROTATE, 0.1)] * 2, 1.0, precision, math.sqrt(3.0))
    po, qo, _, _ = o.state()
    assert np.array_equal(g.positions(), po)
    assert np.array_equal(g.orientations(), qo)
    assert g.overlap_count() == 0


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
def test_lennard_jones_2p19(ctx, precision):
    # Lennard-Jones, N = 2^19, rho = 0.8, kT = 1, r_cut = r_shift = 2.5, translation 0.1, two
    # sweeps. The oracle sums pair energies in body order, the device in its stencil order; no
    # decision may lie inside the any-order summation bound (order_ambiguous == 0), and then every
    # decision equals the oracle's.
    n, rho, seed = 1 << 19, 0.8, 0x5EED0005
    pos, L = lattice.lennard_jones_box(n, rho, 3, seed)
    h = PairwiseCutoff(Isotropic(Shifted(LennardJones(1.0, 1.0), 2.5), 2.5))
    g = Microstate(ctx, Periodic(2.5, [L] * 3), pos, h, seed=seed)
    o = oracle.System(3, [L] * 3, pos, seed=seed, interaction=oracle.LENNARD_JONES, lj_r_cut=2.5, lj_r_shift=2.5)
    ambiguous = sweep_both(g, o, [(TRANSLATE, 0.1)] * 2, 1.0, precision, 2.5)
    assert ambiguous == 0
    assert np.array_equal(g.positions(), o.state()[0])
