"""GPU parity of the Lennard-Jones Metropolis sweep (Isotropic<Shifted<LennardJones>>).

delta_energy_one sums FP64 pair energies in an order the reference leaves to its cell
list; the device sums in its stencil order and the oracle in body-index order, so the
FP64 values agree to a few ulps and decisions can differ only when |dU/kT + ln u| is of
that size. The device bounds that difference for any order and counts the trials inside the
bound (Count.order_ambiguous, flag 4 of hmc_eval_trials); a decision may differ from the oracle's
only on such a trial. The FP32 + recheck pass must reproduce the device FP64 decisions exactly.
"""
import math

import numpy as np
import pytest

import oracle
from hoomd_rs_b200 import (FP32_RECHECK, FP64, TRANSLATE, Context, Isotropic, LennardJones, Microstate,
                           PairwiseCutoff, Periodic, Shifted, lattice)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


def lj(r_cut=2.5, r_shift=2.5):
    return PairwiseCutoff(Isotropic(Shifted(LennardJones(1.0, 1.0), r_shift), r_cut))


def make(ctx, dim, n, rho, seed, r_cut=2.5, r_shift=2.5, positions=None, L=None):
    if positions is None:
        pos, L = lattice.lennard_jones_box(n, rho, dim, seed)
    else:
        pos = positions
    g = Microstate(ctx, Periodic(r_cut, [L] * dim), pos, lj(r_cut, r_shift), seed=seed)
    o = oracle.System(dim, [L] * dim, pos, seed=seed, interaction=oracle.LENNARD_JONES, lj_epsilon=1.0, lj_sigma=1.0,
                      lj_r_cut=r_cut, lj_r_shift=r_shift)
    return g, o, L


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
@pytest.mark.parametrize("dim,n,rho,kt,d", [(3, 1372, 0.8, 1.0, 0.1), (2, 900, 0.7, 0.8, 0.15), (3, 1000, 0.4, 2.0, 0.3)])
def test_lj_trajectory_matches_oracle(ctx, dim, n, rho, kt, d, precision):
    g, o, L = make(ctx, dim, n, rho, seed=0x5EED0005)
    for _ in range(6):
        c = g.sweep(TRANSLATE, d, kt, precision, n_sweeps=1, increment_step=True)
        a, r = o.parallel_sweep(oracle.TRANSLATE, d, kt, 2.5)
        o.increment_step()
        assert c.order_ambiguous == 0
        assert (c.accepted, c.rejected) == (a, r)
    assert np.array_equal(g.positions(), o.state()[0])
    # total energy: the same pair sum in a different order
    assert math.isclose(g.total_energy(), o.total_energy(), rel_tol=1e-11, abs_tol=1e-9)


@pytest.mark.parametrize("dim,n,rho", [(3, 2048, 0.8), (2, 1600, 0.7)])
def test_lj_injected_decisions(ctx, dim, n, rho):
    g, o, L = make(ctx, dim, n, rho, seed=31)
    g.sweep(TRANSLATE, 0.1, 1.0, FP64, n_sweeps=2, increment_step=True)
    pos = g.positions()
    o = oracle.System(dim, [L] * dim, pos, interaction=oracle.LENNARD_JONES, lj_r_cut=2.5, lj_r_shift=2.5)
    # the oracle wraps on construction; compare against the GPU's own body positions
    rng = np.random.default_rng(7)
    m = 40_000
    bodies = rng.integers(0, n, m)
    disp = rng.normal(size=(m, dim)) * rng.choice([0.02, 0.1, 0.3], m)[:, None]
    trial = pos[bodies] + disp
    lam = trial / L
    lam = lam - np.round(lam)
    trial = np.where(lam == 0.5, -0.5, lam) * L
    # uniforms: random, plus a third placed next to the acceptance threshold exp(-dU/kT)
    _, dh_ref = o.eval_moves(bodies, trial, None, np.zeros(m), 1.0)
    u = rng.random(m)
    near = rng.random(m) < 0.33
    thr = np.exp(-np.clip(dh_ref, -50, 50))
    rel = np.exp(rng.uniform(math.log(1e-9), math.log(1e-2), m)) * rng.choice([-1.0, 1.0], m)
    u = np.where(near & (dh_ref > 0), np.clip(thr * (1 + rel), 0, 1 - 1e-16), u)
    want, dh_o = o.eval_moves(bodies, trial, None, u, 1.0)
    d64, _, dh64 = g.eval_moves(bodies, trial, u, 1.0, FP64, return_delta_h=True)
    d32, rech, _ = g.eval_moves(bodies, trial, u, 1.0, FP32_RECHECK, return_delta_h=True)
    assert np.array_equal(d32, d64), np.flatnonzero(d32 != d64)[:10]
    np.testing.assert_allclose(dh64, dh_o, rtol=1e-10, atol=1e-10)
    assert rech.sum() > 0
    # the colour passes' own decisions: every difference from the oracle is a trial the pass
    # flagged as order-ambiguous (its dU within the any-order summation bound of the threshold)
    for precision in (FP64, FP32_RECHECK):
        got, flags = g.eval_trials(bodies, trial, u, 1.0, precision)
        inside = (flags & 2) == 0
        amb = (flags & 4) != 0
        bad = inside & (got != want)
        assert not np.any(bad & ~amb), np.flatnonzero(bad & ~amb)[:10]
        assert np.array_equal(got[inside & ~amb], d64[inside & ~amb])
        assert amb.sum() < 0.01 * m


def test_delta_energy_consistent_with_total_energy(ctx):
    # pairwise_cutoff.rs:1329-1386: dU of a move equals the change of the total energy
    g, o, L = make(ctx, 3, 500, 0.6, seed=5)
    rng = np.random.default_rng(2)
    pos = g.positions()
    for _ in range(20):
        b = int(rng.integers(0, 500))
        t = pos[b] + rng.normal(size=3) * 0.2
        _, _, dh = g.eval_moves([b], [t], [0.5], 1.0, FP64, return_delta_h=True)
        e0 = g.total_energy()
        p2 = pos.copy()
        lam = t / L
        lam = lam - np.round(lam)
        p2[b] = np.where(lam == 0.5, -0.5, lam) * L
        g.set_state(p2, 0, 0)
        e1 = g.total_energy()
        g.set_state(pos, 0, 0)
        assert math.isclose(dh[0], e1 - e0, rel_tol=1e-9, abs_tol=1e-9)


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
def test_lj_overlapping_passes_equal_serialised_passes(ctx, monkeypatch, precision):
    # colour passes launched while the previous one finishes give the serialised trajectory
    pos, L = lattice.lennard_jones_box(1 << 16, 0.8, 3, 0x5EED0005)
    monkeypatch.setenv("HMC_B200_PDL", "1")
    a = Microstate(ctx, Periodic(2.5, [L] * 3), pos, lj(), seed=0x5EED0005)
    monkeypatch.setenv("HMC_B200_PDL", "0")
    b = Microstate(ctx, Periodic(2.5, [L] * 3), pos, lj(), seed=0x5EED0005)
    ca = a.sweep(TRANSLATE, 0.1, 1.0, precision, n_sweeps=3, increment_step=True)
    cb = b.sweep(TRANSLATE, 0.1, 1.0, precision, n_sweeps=3, increment_step=True)
    assert (ca.accepted, ca.rejected) == (cb.accepted, cb.rejected)
    assert np.array_equal(a.positions(), b.positions())


@pytest.mark.parametrize("dim,n,rho", [(3, 1372, 0.8), (2, 900, 0.7), (2, 1 << 18, 0.7)])
def test_lj_wide_bound_block_recheck_equals_fp64(ctx, monkeypatch, dim, n, rho):
    # Widening the FP32 error bound 10^4 times sends most trials of the FP32 pass to the
    # block-cooperative FP64 recheck (several per block, and in the 2^18 case more trials per
    # colour than the grid holds); the trajectory must equal the plain FP64 pass bit for bit.
    pos, L = lattice.lennard_jones_box(n, rho, dim, 0x5EED0012)
    monkeypatch.setenv("HMC_B200_FP32_BAND_SCALE", "1e4")
    a = Microstate(ctx, Periodic(2.5, [L] * dim), pos, lj(), seed=0x5EED0012)
    monkeypatch.delenv("HMC_B200_FP32_BAND_SCALE")
    b = Microstate(ctx, Periodic(2.5, [L] * dim), pos, lj(), seed=0x5EED0012)
    rechecks, trials = 0, 0
    for _ in range(3):
        ca = a.sweep(TRANSLATE, 0.1, 1.0, FP32_RECHECK, n_sweeps=1, increment_step=True)
        cb = b.sweep(TRANSLATE, 0.1, 1.0, FP64, n_sweeps=1, increment_step=True)
        assert (ca.accepted, ca.rejected) == (cb.accepted, cb.rejected)
        rechecks += ca.rechecks
        trials += ca.total()
    assert np.array_equal(a.positions(), b.positions())
    assert rechecks > trials // 4, (rechecks, trials)
