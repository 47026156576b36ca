"""GPU parity of the hard-disk / hard-sphere sweep against the CPU oracle.

The oracle restates ParallelSweep::apply (hoomd-mc/src/parallel_sweep.rs:390-421) with
the same counter-based random streams, so for the same initial state the GPU sweep must
reproduce the oracle's trajectory bit for bit, in both precision modes. Injected
near-contact moves check the accept/reject decision of delta_energy_one
(pairwise_cutoff.rs:919-941) and the FP32 forward-error bound directly.
"""
import math

import numpy as np
import pytest

import oracle
from hoomd_rs_b200 import (FP32_RECHECK, FP64, TRANSLATE, Context, HardSphere, HmcError, Isothermal, Microstate,
                           PairwiseCutoff, ParallelSweep, Periodic, Translate, lattice)
import hoomd_rs_b200 as hm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


def make(ctx, dim, n, phi, seed, L=None, body_range=0.0, positions=None, step=0, substep=0):
    if positions is None:
        pos, Lc = lattice.hard_sphere_box(n, phi, dim, seed)
    else:
        pos, Lc = positions, L
    Ls = list(L) if isinstance(L, (list, tuple)) else [L or Lc] * dim
    h = PairwiseCutoff(HardSphere(1.0))
    g = Microstate(ctx, Periodic(1.0, Ls), pos, h, seed=seed, step=step, substep=substep,
                   body_interaction_range=body_range)
    o = oracle.System(dim, Ls, pos, diameter=1.0, seed=seed, step=step, substep=substep)
    return g, o, Ls


def run_both(g, o, d, sweeps, precision, body_range=1.0):
    for _ in range(sweeps):
        c = g.sweep(TRANSLATE, d, 1.0, precision, n_sweeps=1, increment_step=True)
        a, r = o.parallel_sweep(oracle.TRANSLATE, d, 1.0, body_range)
        o.increment_step()
        assert (c.accepted, c.rejected) == (a, r)
    pg = g.positions()
    po = o.state()[0]
    return pg, po


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
@pytest.mark.parametrize("dim,n,phi,d,sweeps", [
    (2, 4096, 0.70, 0.1, 20),   # the 2-D hard-disk workload (N = 4096, area fraction 0.70)
    (3, 4000, 0.50, 0.15, 10),  # FCC spheres at packing fraction 0.50
    (3, 2048, 0.30, 0.60, 10),  # dilute, large moves: many boundary crossings
    (2, 1000, 0.45, 0.80, 10),
])
def test_trajectory_bit_identical_to_oracle(ctx, dim, n, phi, d, sweeps, precision):
    g, o, _ = make(ctx, dim, n, phi, seed=0x5EED0001 + dim)
    pg, po = run_both(g, o, d, sweeps, precision)
    assert np.array_equal(pg, po), np.abs(pg - po).max()
    assert g.overlap_count() == 0
    assert o.overlap_count() == 0


@pytest.mark.parametrize("dim,n,phi,d", [(3, 4000, 0.50, 0.15), (2, 4096, 0.70, 0.1)])
def test_wide_fp32_band_rechecks_in_fp64(ctx, monkeypatch, dim, n, phi, d):
    # Widening the FP32 band 10^5 times sends every pair within ~10 % of contact to the FP64
    # recheck inside the sweep; the trajectory must still equal the oracle's.
    monkeypatch.setenv("HMC_B200_FP32_BAND_SCALE", "1e5")
    g, o, _ = make(ctx, dim, n, phi, seed=0x5EED0011)
    monkeypatch.delenv("HMC_B200_FP32_BAND_SCALE")
    rechecks = 0
    for _ in range(6):
        c = g.sweep(TRANSLATE, d, 1.0, FP32_RECHECK, n_sweeps=1, increment_step=True)
        a, r = o.parallel_sweep(oracle.TRANSLATE, d, 1.0, 1.0)
        o.increment_step()
        assert (c.accepted, c.rejected) == (a, r)
        rechecks += c.rechecks
    assert rechecks > 100
    assert np.array_equal(g.positions(), o.state()[0])


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
def test_large_spaces_choose_among_several_bodies(ctx, precision):
    # body_interaction_range 2.5: ~5-15 bodies per space, exercising choose() and the
    # index order of each space's body list.
    g, o, _ = make(ctx, 3, 3000, 0.45, seed=77, body_range=2.5)
    pg, po = run_both(g, o, 0.2, 6, precision, body_range=2.5)
    assert np.array_equal(pg, po)


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
@pytest.mark.parametrize("dim,L,n", [(3, [2.4, 2.6, 4.4], 6), (2, [2.2, 2.9], 3), (2, [4.3, 2.1], 4)])
def test_two_spaces_per_axis(ctx, dim, L, n, precision):
    # floor(L / range) == 2 on some axes: both neighbours of a space are the same space.
    rng = np.random.default_rng(3)
    pos = []
    while len(pos) < n:
        p = (rng.random(dim) - 0.5) * np.array(L)
        ok = True
        for q in pos:
            dd = np.array(p) - q
            dd -= np.array(L) * np.round(dd / np.array(L))
            ok &= float(dd @ dd) > 1.05
        if ok:
            pos.append(p)
    pos = np.array(pos)
    g, o, _ = make(ctx, dim, n, 0.0, seed=5, L=L, positions=pos)
    pg, po = run_both(g, o, 0.5, 40, precision)
    assert np.array_equal(pg, po)


def test_single_body(ctx):
    g, o, _ = make(ctx, 3, 1, 0.0, seed=9, L=[3.0, 3.0, 3.0], positions=np.array([[0.1, 0.2, 0.3]]))
    pg, po = run_both(g, o, 0.4, 5, FP32_RECHECK)
    assert np.array_equal(pg, po)


def _near_contact_moves(o, n_moves, seed, spread):
    """Trial positions of body i placed at distance sigma*(1 + delta) from a neighbour j."""
    rng = np.random.default_rng(seed)
    pos = o.state()[0]
    n, dim = pos.shape
    L = o.L
    bodies = rng.integers(0, n, n_moves)
    js = rng.integers(0, n, n_moves)
    js = np.where(js == bodies, (js + 1) % n, js)
    v = rng.normal(size=(n_moves, dim))
    v /= np.linalg.norm(v, axis=1)[:, None]
    # delta log-uniform in [1e-17, spread], either sign; a tenth exactly at contact
    delta = np.exp(rng.uniform(math.log(1e-17), math.log(spread), n_moves)) * rng.choice([-1.0, 1.0], n_moves)
    delta[::10] = 0.0
    trial = pos[js] + v * (1.0 + delta)[:, None]
    # wrap like the trial move: wrap(propose(..)); the pair test wraps once more
    lam = trial / L
    lam = lam - np.round(lam)
    lam = np.where(lam == 0.5, -0.5, lam)
    return bodies, lam * L


@pytest.mark.parametrize("dim,n,phi", [(2, 4096, 0.70), (3, 8000, 0.50)])
def test_injected_near_contact_decisions(ctx, dim, n, phi):
    g, o, _ = make(ctx, dim, n, phi, seed=11)
    run_both(g, o, 0.12, 3, FP64)
    total = 0
    rechecked = 0
    for rep, spread in enumerate((1e-6, 1e-9, 1e-13)):
        bodies, trial = _near_contact_moves(o, 200_000, seed=100 + rep, spread=spread)
        want, _ = o.eval_moves(bodies, trial, None, np.zeros(len(bodies)), 1.0)
        got64, _ = g.eval_moves(bodies, trial, precision=FP64)
        got32, rech = g.eval_moves(bodies, trial, precision=FP32_RECHECK)
        assert np.array_equal(got64, want), np.flatnonzero(got64 != want)[:10]
        assert np.array_equal(got32, want), np.flatnonzero(got32 != want)[:10]
        total += len(bodies)
        rechecked += int(rech.sum())
    assert 0 < want.sum() < len(want)
    assert rechecked > 0  # the adversarial set exercises the FP64 recheck


def test_full_size_fp32_recheck_equals_fp64(ctx):
    # 2^20 spheres at packing fraction 0.50: FP32 + recheck reproduces FP64 bit for bit.
    pos, L = lattice.hard_sphere_box(1 << 20, 0.50, 3, 0x5EED0002)
    h = PairwiseCutoff(HardSphere(1.0))
    a = Microstate(ctx, Periodic(1.0, [L] * 3), pos, h, seed=0x5EED0002)
    b = Microstate(ctx, Periodic(1.0, [L] * 3), pos, h, seed=0x5EED0002)
    ca = a.sweep(TRANSLATE, 0.2, 1.0, FP64, n_sweeps=4, increment_step=True)
    cb = b.sweep(TRANSLATE, 0.2, 1.0, FP32_RECHECK, n_sweeps=4, increment_step=True)
    assert (ca.accepted, ca.rejected) == (cb.accepted, cb.rejected)
    assert np.array_equal(a.positions(), b.positions())
    assert b.overlap_count() == 0
    assert cb.rechecks < 1e-3 * cb.pair_checks


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
def test_overlapping_passes_equal_serialised_passes(ctx, monkeypatch, precision):
    # 2^20 spheres: colour passes launched while the previous pass finishes (programmatic
    # dependent launch) give the trajectory of passes launched one after another.
    pos, L = lattice.hard_sphere_box(1 << 20, 0.50, 3, 0x5EED0002)
    h = PairwiseCutoff(HardSphere(1.0))
    monkeypatch.setenv("HMC_B200_PDL", "1")
    a = Microstate(ctx, Periodic(1.0, [L] * 3), pos, h, seed=0x5EED0002)
    monkeypatch.setenv("HMC_B200_PDL", "0")
    b = Microstate(ctx, Periodic(1.0, [L] * 3), pos, h, seed=0x5EED0002)
    ca = a.sweep(TRANSLATE, 0.2, 1.0, precision, n_sweeps=4, increment_step=True)
    cb = b.sweep(TRANSLATE, 0.2, 1.0, precision, n_sweeps=4, increment_step=True)
    assert (ca.accepted, ca.rejected) == (cb.accepted, cb.rejected)
    assert np.array_equal(a.positions(), b.positions())
    assert a.overlap_count() == 0


def test_overlap_check_finds_planted_overlap(ctx):
    pos = np.array([[0.0, 0.0, 0.0], [0.5, 0.0, 0.0], [3.0, 3.0, 3.0], [-4.9, 0.0, 0.0], [4.6, 0.0, 0.0]])
    h = PairwiseCutoff(HardSphere(1.0))
    g = Microstate(ctx, Periodic(1.0, [10.0] * 3), pos, h)
    o = oracle.System(3, [10.0] * 3, pos, diameter=1.0)
    assert g.overlap_count() == o.overlap_count() == 2  # (0,1) and (3,4) through the boundary


def test_parallel_sweep_api_mirror(ctx):
    pos, L = lattice.hard_sphere_box(4096, 0.70, 2, 0x5EED0001)
    h = PairwiseCutoff(HardSphere(diameter=1.0))
    micro = Microstate(ctx, Periodic(1.0, [L, L]), pos, h, seed=0x5EED0001)
    sweep = ParallelSweep(1.0, Translate.with_maximum_distance(0.1))
    count = sweep.apply(micro, h, Isothermal(temperature=1.0))
    assert count.total() >= 4096
    assert 0.0 < count.acceptance_ratio() < 1.0


def test_errors_are_status_codes(ctx):
    h = PairwiseCutoff(HardSphere(1.0))
    with pytest.raises(HmcError) as e:
        Microstate(ctx, Periodic(1.0, [1.5, 1.5]), [[0.0, 0.0]], h)
    assert e.value.status == hm.RANGE_TOO_LARGE
    with pytest.raises(HmcError) as e:
        Microstate(ctx, Periodic(1.0, [5.0, 5.0]), [[0.0, float("nan")]], h)
    assert e.value.status == hm.NAN_STATE
    g = Microstate(ctx, Periodic(1.0, [5.0, 5.0]), [[0.0, 0.0]], h)
    with pytest.raises(HmcError) as e:
        g.sweep(TRANSLATE, -1.0, 1.0, FP64)
    assert e.value.status == hm.INVALID_ARGUMENT
    # the context stays usable after errors
    assert g.sweep(TRANSLATE, 0.3, 1.0, FP64).total() == 1


def test_context_released_after_its_last_system(ctx):
    # Destroying a context while a system still uses it defers the release to the
    # system's destruction; nothing leaks into later calls.
    c2 = Context(0)
    pos, L = lattice.hard_sphere_box(512, 0.4, 3, 21)
    g = Microstate(c2, Periodic(1.0, [L] * 3), pos, PairwiseCutoff(HardSphere(1.0)), seed=21)
    c2.close()
    assert g.sweep(TRANSLATE, 0.2, 1.0, FP32_RECHECK).total() >= 512
    g.close()
    h = Microstate(ctx, Periodic(1.0, [L] * 3), pos, PairwiseCutoff(HardSphere(1.0)), seed=21)
    assert h.overlap_count() == 0


def test_ten_million_injected_near_contact_moves(ctx):
    # 10^7 injected trials of the 3-D hard-sphere state (phi = 0.50), each placed at
    # sigma * (1 + delta) from another sphere with |delta| log-uniform down to 1e-17 (a tenth at
    # contact): FP64 and FP32 + recheck decisions equal the oracle's on every one.
    g, o, _ = make(ctx, 3, 32768, 0.50, seed=0x5EED0015)
    run_both(g, o, 0.12, 2, FP64)
    total, rechecked, accepted = 0, 0, 0
    for chunk in range(10):
        spread = (1e-3, 1e-6, 1e-9, 1e-12, 1e-15)[chunk % 5]
        bodies, trial = _near_contact_moves(o, 1_000_000, seed=1000 + chunk, spread=spread)
        want, _ = o.eval_moves(bodies, trial, None, np.zeros(len(bodies)), 1.0)
        got64, _ = g.eval_moves(bodies, trial, precision=FP64)
        got32, rech = g.eval_moves(bodies, trial, precision=FP32_RECHECK)
        assert np.array_equal(got64, want), (chunk, np.flatnonzero(got64 != want)[:10])
        assert np.array_equal(got32, want), (chunk, np.flatnonzero(got32 != want)[:10])
        total += len(bodies)
        rechecked += int(rech.sum())
        accepted += int(want.sum())
    assert total == 10_000_000
    assert 0 < accepted < total
    assert rechecked > 100_000
