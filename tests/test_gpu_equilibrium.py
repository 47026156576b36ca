"""The survey's oracle part (c) on the 3-D configurations: the checkerboard sweep visits bodies in
another order than the serial Sweep (hoomd-mc/src/sweep.rs:159-224), so their trajectories
differ, but the equilibrium they sample must not. A GPU ParallelSweep run and a CPU serial Sweep
run (the oracle, another seed) of the same system are compared within 2 sigma of blocked error
bars: the SDF pressure and g(r) of hard spheres at packing fraction 0.50, g(r) of hard cubes at
0.55, the potential energy per site and g(r) of Lennard-Jones sites at rho = 0.8, kT = 1; the
acceptance ratios are compared against a CPU ParallelSweep run with another seed (the same
algorithm, so the same acceptance).
"""
import math

import numpy as np
import pytest

import oracle
from hoomd_rs_b200 import (FP32_RECHECK, ROTATE, TRANSLATE, Context, ConvexPolyhedron, HardShape, HardSphere,
                           Isotropic, LennardJones, Microstate, PairwiseCutoff, Periodic, Shifted, gr_normalise,
                           lattice, sdf_pressure)

pytestmark = pytest.mark.gpu

CUBE = np.array([[x, y, z] for x in (-0.5, 0.5) for y in (-0.5, 0.5) for z in (-0.5, 0.5)])


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


def blocks(x, nb=10):
    x = np.asarray(x, dtype=np.float64)
    m = len(x) // nb * nb
    b = x[:m].reshape(nb, -1).mean(axis=1)
    return b.mean(), b.std(ddof=1) / np.sqrt(nb)


def agree(a, b):
    (m1, e1), (m2, e2) = blocks(a), blocks(b)
    return abs(m1 - m2) < 2.0 * math.hypot(e1, e2), (m1, e1, m2, e2)


def gr_agrees(ga, gb, first_bin):
    z = []
    for k in range(first_bin, ga.shape[1]):
        (m1, e1), (m2, e2) = blocks(ga[:, k]), blocks(gb[:, k])
        if e1 > 0 or e2 > 0:
            z.append((m1 - m2) / math.hypot(e1, e2))
    return float(np.mean(np.square(z))) < 4.0, z


def test_hard_spheres_phi_050(ctx):
    n, phi, d, equil, sweeps, every = 864, 0.50, 0.12, 300, 2300, 10
    pos, L = lattice.hard_sphere_box(n, phi, 3, 71, lattice="fcc")
    vol = L ** 3
    g = Microstate(ctx, Periodic(1.0, [L] * 3), pos, PairwiseCutoff(HardSphere(1.0)), seed=71)
    p_g, gr_g, acc_g = [], [], []
    for k in range(sweeps):
        c = g.sweep(TRANSLATE, d, 1.0, FP32_RECHECK, n_sweeps=1, increment_step=True)
        if k >= equil:
            acc_g.append(c.acceptance_ratio())
            if k % every == 0:
                p_g.append(sdf_pressure(g.sdf(0.02, 40), n, vol, 3, 0.02))
                gr_g.append(gr_normalise(g.gr_counts(2.5, 25), n, vol, 3, 2.5)[1])
    o = oracle.System(3, [L] * 3, pos, seed=72)
    p_c, gr_c = [], []
    for k in range(sweeps):
        o.serial_sweep(oracle.TRANSLATE, d, 1.0)
        o.increment_step()
        if k >= equil and k % every == 0:
            p_c.append(sdf_pressure(o.sdf(0.02, 40), n, vol, 3, 0.02))
            gr_c.append(gr_normalise(o.gr(2.5, 25), n, vol, 3, 2.5)[1])
    o2 = oracle.System(3, [L] * 3, pos, seed=73)
    acc_c = []
    for k in range(sweeps):
        a, r = o2.parallel_sweep(oracle.TRANSLATE, d, 1.0, 1.0, threads=4)
        o2.increment_step()
        if k >= equil:
            acc_c.append(a / (a + r))
    assert g.overlap_count() == 0 == o.overlap_count()
    ok, info = agree(p_g, p_c)
    assert ok, ("pressure", info)
    ok, info = agree(acc_g, acc_c)
    assert ok, ("acceptance", info)
    ok, z = gr_agrees(np.array(gr_g), np.array(gr_c), 10)  # r >= sigma
    assert ok, z


def test_hard_cubes_phi_055(ctx):
    n, phi, equil, sweeps, every = 512, 0.55, 200, 1400, 10
    L = (n / phi) ** (1.0 / 3.0)
    pos = lattice.cubic_lattice(n, L, 3, 74, jitter=0.01)
    vol = L ** 3
    h = PairwiseCutoff(HardShape(ConvexPolyhedron.with_vertices(CUBE)))
    g = Microstate(ctx, Periodic(math.sqrt(3.0), [L] * 3), pos, h, seed=74)
    moves = [(TRANSLATE, oracle.TRANSLATE, 0.08), (ROTATE, oracle.ROTATE, 0.1)]
    acc_g = {0: [], 1: []}
    gr_g = []
    for k in range(sweeps):
        mv, _, m = moves[k % 2]
        c = g.sweep(mv, m, 1.0, FP32_RECHECK, n_sweeps=1, increment_step=True)
        if k >= equil:
            acc_g[k % 2].append(c.acceptance_ratio())
            if k % every == 0:
                gr_g.append(gr_normalise(g.gr_counts(2.6, 26), n, vol, 3, 2.6)[1])
    o = oracle.System(3, [L] * 3, pos, None, seed=75, interaction=oracle.HARD_CONVEX_POLYHEDRON, vertices=CUBE)
    gr_c = []
    for k in range(sweeps):
        _, om, m = moves[k % 2]
        o.serial_sweep(om, m, 1.0)
        o.increment_step()
        if k >= equil and k % every == 0:
            gr_c.append(gr_normalise(o.gr(2.6, 26), n, vol, 3, 2.6)[1])
    o2 = oracle.System(3, [L] * 3, pos, None, seed=76, interaction=oracle.HARD_CONVEX_POLYHEDRON, vertices=CUBE)
    acc_c = {0: [], 1: []}
    for k in range(sweeps):
        _, om, m = moves[k % 2]
        a, r = o2.parallel_sweep(om, m, 1.0, math.sqrt(3.0), threads=4)
        o2.increment_step()
        if k >= equil:
            acc_c[k % 2].append(a / (a + r))
    assert g.overlap_count() == 0 == o.overlap_count()
    for kind in (0, 1):
        ok, info = agree(acc_g[kind], acc_c[kind])
        assert ok, (("translate", "rotate")[kind], info)
    ok, z = gr_agrees(np.array(gr_g), np.array(gr_c), 8)  # r >= 0.8: inside, no pair fits
    assert ok, z


def test_lennard_jones_rho_08(ctx):
    n, rho, kt, d, equil, sweeps, every = 500, 0.8, 1.0, 0.15, 100, 800, 5
    pos, L = lattice.lennard_jones_box(n, rho, 3, 77)
    vol = L ** 3
    h = PairwiseCutoff(Isotropic(Shifted(LennardJones(1.0, 1.0), 2.5), 2.5))
    g = Microstate(ctx, Periodic(2.5, [L] * 3), pos, h, seed=77)
    e_g, acc_g, gr_g = [], [], []
    for k in range(sweeps):
        c = g.sweep(TRANSLATE, d, kt, FP32_RECHECK, n_sweeps=1, increment_step=True)
        if k >= equil:
            acc_g.append(c.acceptance_ratio())
            if k % every == 0:
                e_g.append(g.total_energy() / n)
                gr_g.append(gr_normalise(g.gr_counts(2.5, 25), n, vol, 3, 2.5)[1])
    o = oracle.System(3, [L] * 3, pos, seed=78, interaction=oracle.LENNARD_JONES, lj_r_cut=2.5, lj_r_shift=2.5)
    e_c, gr_c = [], []
    for k in range(sweeps):
        o.serial_sweep(oracle.TRANSLATE, d, kt)
        o.increment_step()
        if k >= equil and k % every == 0:
            e_c.append(o.total_energy() / n)
            gr_c.append(gr_normalise(o.gr(2.5, 25), n, vol, 3, 2.5)[1])
    o2 = oracle.System(3, [L] * 3, pos, seed=79, interaction=oracle.LENNARD_JONES, lj_r_cut=2.5, lj_r_shift=2.5)
    acc_c = []
    for k in range(sweeps):
        a, r = o2.parallel_sweep(oracle.TRANSLATE, d, kt, 2.5)
        o2.increment_step()
        if k >= equil:
            acc_c.append(a / (a + r))
    ok, info = agree(e_g, e_c)
    assert ok, ("energy per site", info)
    ok, info = agree(acc_g, acc_c)
    assert ok, ("acceptance", info)
    ok, z = gr_agrees(np.array(gr_g), np.array(gr_c), 8)
    assert ok, z
