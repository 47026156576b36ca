"""Equilibrium estimators and the statistical agreement with CPU runs.

The scale distribution function (SDF) and g(r) histograms of the device must equal the
oracle's pair counts exactly for the same state. Because the checkerboard sweep orders its
trials differently from the serial Sweep, trajectories differ between the two; what must agree
is the equilibrium: SDF pressure and g(r) of a GPU ParallelSweep run against a CPU serial
Sweep run, and the acceptance ratio against a CPU ParallelSweep run with another seed, each
within 2 sigma of blocked error bars.
"""
import numpy as np
import pytest

import oracle
from hoomd_rs_b200 import (FP32_RECHECK, FP64, TRANSLATE, Context, HardSphere, Microstate, PairwiseCutoff, Periodic,
                           gr_normalise, lattice, sdf_pressure)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


@pytest.mark.parametrize("dim,n,phi", [(2, 2000, 0.65), (3, 3000, 0.45)])
def test_pair_histograms_equal_oracle(ctx, dim, n, phi):
    pos, L = lattice.hard_sphere_box(n, phi, dim, 41)
    g = Microstate(ctx, Periodic(1.0, [L] * dim), pos, PairwiseCutoff(HardSphere(1.0)), seed=41)
    g.sweep(TRANSLATE, 0.15, 1.0, FP32_RECHECK, n_sweeps=20, increment_step=True)
    o = oracle.System(dim, [L] * dim, g.positions())
    assert np.array_equal(g.sdf(0.02, 40), o.sdf(0.02, 40))
    assert np.array_equal(g.gr_counts(3.0, 60), o.gr(3.0, 60))
    assert g.sdf(0.02, 40).sum() > 0


def _blocks(x, nb=10):
    x = np.asarray(x, dtype=np.float64)
    m = len(x) // nb * nb
    b = x[:m].reshape(nb, -1).mean(axis=1)
    return b.mean(), b.std(ddof=1) / np.sqrt(nb)


def test_equilibrium_matches_cpu_serial_and_parallel_sweeps(ctx):
    dim, n, phi, d = 2, 1024, 0.60, 0.15
    pos, L = lattice.hard_sphere_box(n, phi, dim, 51)
    vol = L ** dim
    equil, sweeps, every = 200, 2200, 10
    # GPU ParallelSweep
    g = Microstate(ctx, Periodic(1.0, [L] * dim), pos, PairwiseCutoff(HardSphere(1.0)), seed=51)
    p_gpu, acc_gpu, gr_gpu = [], [], []
    for k in range(sweeps):
        c = g.sweep(TRANSLATE, d, 1.0, FP32_RECHECK, n_sweeps=1, increment_step=True)
        if k >= equil:
            acc_gpu.append(c.acceptance_ratio())
            if k % every == 0:
                p_gpu.append(sdf_pressure(g.sdf(0.02, 40), n, vol, dim, 0.02))
                gr_gpu.append(gr_normalise(g.gr_counts(3.0, 30), n, vol, dim, 3.0)[1])
    # CPU serial Sweep (Sweep::apply, sweep.rs:159-224): a different trial order, the same equilibrium
    o = oracle.System(dim, [L] * dim, pos, seed=52)
    p_cpu, gr_cpu = [], []
    for k in range(sweeps):
        o.serial_sweep(oracle.TRANSLATE, d, 1.0)
        o.increment_step()
        if k >= equil and k % every == 0:
            p_cpu.append(sdf_pressure(o.sdf(0.02, 40), n, vol, dim, 0.02))
            gr_cpu.append(gr_normalise(o.gr(3.0, 30), n, vol, dim, 3.0)[1])
    # CPU ParallelSweep with another seed: the acceptance of the same algorithm
    o2 = oracle.System(dim, [L] * dim, pos, seed=53)
    acc_cpu = []
    for k in range(sweeps):
        a, r = o2.parallel_sweep(oracle.TRANSLATE, d, 1.0, 1.0)
        o2.increment_step()
        if k >= equil:
            acc_cpu.append(a / (a + r))
    assert g.overlap_count() == 0 and o.overlap_count() == 0
    (mp_g, ep_g), (mp_c, ep_c) = _blocks(p_gpu), _blocks(p_cpu)
    assert abs(mp_g - mp_c) < 2.0 * np.hypot(ep_g, ep_c), (mp_g, ep_g, mp_c, ep_c)
    (ma_g, ea_g), (ma_c, ea_c) = _blocks(acc_gpu), _blocks(acc_cpu)
    assert abs(ma_g - ma_c) < 2.0 * np.hypot(ea_g, ea_c), (ma_g, ea_g, ma_c, ea_c)
    # g(r) over the first shells: the mean squared z-score of the bins stays near 1
    gg, gc = np.array(gr_gpu), np.array(gr_cpu)
    z = []
    for b in range(10, 30):  # r >= sigma: below it g(r) = 0 in both runs
        (m1, e1), (m2, e2) = _blocks(gg[:, b]), _blocks(gc[:, b])
        z.append((m1 - m2) / np.hypot(e1, e2))
    assert np.mean(np.square(z)) < 4.0, z
