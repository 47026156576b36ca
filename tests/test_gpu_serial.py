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


def test_serial_sweep_lennard_jones(ctx):
    # Sweep::apply_with_filter over Isotropic<Shifted<LennardJones>>: dH summed per stencil cell
    # and reduced over the warp; no decision may lie within the any-order summation bound, and
    # the chain (uniforms drawn only for 0 < dH < inf) equals the oracle's
    from hoomd_rs_b200 import Isotropic, LennardJones, Shifted
    pos, L = lattice.lennard_jones_box(1372, 0.8, 3, 63)
    h = PairwiseCutoff(Isotropic(Shifted(LennardJones(1.0, 1.0), 2.5), 2.5))
    g = Microstate(ctx, Periodic(2.5, [L] * 3), pos, h, seed=63, step=1)
    o = oracle.System(3, [L] * 3, pos, seed=63, step=1, interaction=oracle.LENNARD_JONES, lj_r_cut=2.5,
                      lj_r_shift=2.5)
    for kt in (1.0, 0.7, 1.5):
        c = g.serial_sweep(0.12, increment_step=True, temperature=kt)
        a, r = o.serial_sweep(oracle.TRANSLATE, 0.12, kt)
        o.increment_step()
        assert c.order_ambiguous == 0
        assert (c.accepted, c.rejected) == (a, r)
    assert np.array_equal(g.positions(), o.state()[0])


def test_serial_sweep_cubes_translate_and_rotate(ctx):
    import math
    from hoomd_rs_b200 import ROTATE, ConvexPolyhedron, HardShape
    cube = np.array([[x, y, z] for x in (-0.5, 0.5) for y in (-0.5, 0.5) for z in (-0.5, 0.5)])
    n, phi = 1000, 0.5
    L = (n / phi) ** (1 / 3)
    pos = lattice.cubic_lattice(n, L, 3, 64)
    g = Microstate(ctx, Periodic(math.sqrt(3), [L] * 3), pos,
                   PairwiseCutoff(HardShape(ConvexPolyhedron.with_vertices(cube))), seed=64)
    o = oracle.System(3, [L] * 3, pos, None, seed=64, interaction=oracle.HARD_CONVEX_POLYHEDRON, vertices=cube)
    mask = (np.arange(n) % 5) != 2
    for sweep in range(6):
        move, om, m = (TRANSLATE, oracle.TRANSLATE, 0.1) if sweep % 2 == 0 else (ROTATE, oracle.ROTATE, 0.2)
        use = mask if sweep == 3 else None
        c = g.serial_sweep(m, increment_step=True, move=move, move_mask=use)
        a, r = o.serial_sweep(om, m, 1.0, mask=use)
        o.increment_step()
        assert (c.accepted, c.rejected) == (a, r), sweep
    po, qo, _, _ = o.state()
    assert np.array_equal(g.positions(), po)
    assert np.array_equal(g.orientations(), qo)
    assert g.overlap_count() == 0


@pytest.mark.parametrize("kind", ["polygon", "mesh"])
def test_serial_sweep_polygons_translate_and_rotate(ctx, kind):
    import math
    from hoomd_rs_b200 import ROTATE, ConvexPolygon, ConvexSurfaceMesh2d, HardShape
    square = np.array([[-0.5, -0.5], [0.5, -0.5], [0.5, 0.5], [-0.5, 0.5]])
    shape = ConvexPolygon.with_vertices(square) if kind == "polygon" else ConvexSurfaceMesh2d.from_point_set(square)
    okind = oracle.HARD_CONVEX_POLYGON if kind == "polygon" else oracle.HARD_CONVEX_SURFACE_MESH_2D
    n = 900
    L = 30 * 1.5
    pos = lattice.cubic_lattice(n, L, 2, 65, jitter=0.0)
    ang = np.random.default_rng(65).uniform(-math.pi, math.pi, n)
    g = Microstate(ctx, Periodic(math.sqrt(2), [L, L]), pos, PairwiseCutoff(HardShape(shape)), seed=65,
                   orientations=ang)
    o = oracle.System(2, [L, L], pos, ang, seed=65, interaction=okind, vertices=square)
    for sweep in range(6):
        move, om, m = (TRANSLATE, oracle.TRANSLATE, 0.2) if sweep % 2 == 0 else (ROTATE, oracle.ROTATE, 0.4)
        c = g.serial_sweep(m, increment_step=True, move=move)
        a, r = o.serial_sweep(om, m, 1.0)
        o.increment_step()
        assert (c.accepted, c.rejected) == (a, r), sweep
    po, qo, _, _ = o.state()
    assert np.array_equal(g.positions(), po)
    assert np.array_equal(g.orientations(), qo.reshape(-1))
