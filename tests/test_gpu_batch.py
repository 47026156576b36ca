"""Batches of independent hard-sphere replicas (hmc_batch_*).

Each replica keeps its own box, checkerboard and Counter, so after any number of batched
sweeps replica k must equal, bit for bit, a single system built from the same description
and swept with the same move size (and hence the oracle).
"""
import numpy as np
import pytest

import oracle
from hoomd_rs_b200 import (FP32_RECHECK, FP64, TRANSLATE, Batch, Context, HardSphere, Microstate, PairwiseCutoff,
                           Periodic, lattice)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


def replicas(dim, specs):
    out = []
    for k, (n, phi, seed, step, kind) in enumerate(specs):
        pos, L = lattice.hard_sphere_box(n, phi, dim, seed, lattice=kind)
        # a valid hard-sphere start: the lattice spacing must exceed 1 + the jitter
        assert oracle.System(dim, [L] * dim, pos).overlap_count() == 0
        out.append({"boundary": Periodic(1.0, [L] * dim), "positions": pos, "seed": seed, "step": step})
    return out


# (N, packing fraction, seed, step, lattice); the last replica has two spaces per axis
SPECS3 = [(500, 0.40, 11, 0, "fcc"), (1024, 0.48, 12, 3, "fcc"), (2000, 0.45, 13, 0, "fcc"),
          (777, 0.50, 14, 9, "fcc"), (4096, 0.42, 15, 1, "fcc"), (8, 0.30, 16, 0, "cubic")]
SPECS2 = [(1000, 0.60, 21, 0, "auto"), (4096, 0.70, 22, 2, "auto"), (300, 0.45, 23, 0, "auto")]


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
@pytest.mark.parametrize("dim,specs", [(3, SPECS3), (2, SPECS2)])
def test_batch_replicas_equal_single_systems(ctx, dim, specs, precision):
    reps = replicas(dim, specs)
    maxima = np.linspace(0.08, 0.3, len(reps))
    b = Batch(ctx, reps)
    singles = [Microstate(ctx, r["boundary"], r["positions"], PairwiseCutoff(HardSphere(1.0)), seed=r["seed"],
                          step=r["step"]) for r in reps]
    for _ in range(5):
        counts, total = b.sweep(maxima, precision, increment_step=True)
        for k, m in enumerate(singles):
            c = m.sweep(TRANSLATE, float(maxima[k]), 1.0, precision, n_sweeps=1, increment_step=True)
            assert (counts[k].accepted, counts[k].rejected) == (c.accepted, c.rejected), k
        assert total.accepted == sum(c.accepted for c in counts)
    for k, m in enumerate(singles):
        pos, step, sub = b.state(k)
        assert np.array_equal(pos, m.positions()), k
        assert (step, sub) == (m.step(), m.substep())
    assert not b.overlap_counts().any()


def test_batch_replica_equals_oracle_and_overlap_counts(ctx):
    reps = replicas(3, SPECS3[:3])
    b = Batch(ctx, reps)
    r = reps[1]
    L = r["boundary"].edge_lengths[0]
    o = oracle.System(3, [L] * 3, r["positions"], seed=r["seed"], step=r["step"])
    for _ in range(4):
        b.sweep([0.2, 0.15, 0.2], FP32_RECHECK, increment_step=True)
        o.parallel_sweep(oracle.TRANSLATE, 0.15, 1.0, 1.0)
        o.increment_step()
    assert np.array_equal(b.positions(1), o.state()[0])
    # plant overlaps in replica 2 only; the oracle counts the same pairs
    p2, step, sub = b.state(2)
    L2 = reps[2]["boundary"].edge_lengths[0]
    moved = p2[0] + np.array([0.5, 0.0, 0.0])
    lam = moved / L2 - np.round(moved / L2)
    p2[1] = np.where(lam == 0.5, -0.5, lam) * L2
    b.set_state(2, p2, step, sub)
    want = oracle.System(3, [L2] * 3, p2).overlap_count()
    assert want >= 1
    assert list(b.overlap_counts()) == [0, 0, want]


def lj_replicas(dim, specs):
    from hoomd_rs_b200 import Isotropic, LennardJones, Shifted
    out = []
    for n, rho, seed, step, r_cut in specs:
        pos, L = lattice.lennard_jones_box(n, rho, dim, seed)
        h = PairwiseCutoff(Isotropic(Shifted(LennardJones(1.0, 1.0), r_cut), r_cut))
        out.append({"boundary": Periodic(r_cut, [L] * dim), "positions": pos, "seed": seed, "step": step,
                    "hamiltonian": h})
    return out


# (N, density, seed, step, r_cut); different sizes, densities and cut-offs per replica
LJ3 = [(1372, 0.8, 31, 0, 2.5), (864, 0.6, 32, 4, 2.5), (2048, 0.85, 33, 0, 2.2), (500, 0.5, 34, 1, 3.0)]
LJ2 = [(900, 0.7, 41, 0, 2.5), (1600, 0.6, 42, 2, 2.5), (400, 0.8, 43, 0, 2.0)]


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
@pytest.mark.parametrize("dim,specs", [(3, LJ3), (2, LJ2)])
def test_lj_batch_replicas_equal_single_systems(ctx, dim, specs, precision):
    # Lennard-Jones replicas, each at its own temperature: replica k equals, bit for bit, a
    # single system swept with the same move size and kT.
    reps = lj_replicas(dim, specs)
    maxima = np.linspace(0.08, 0.2, len(reps))
    kts = np.linspace(0.8, 2.0, len(reps))
    b = Batch(ctx, reps)
    singles = [Microstate(ctx, r["boundary"], r["positions"], r["hamiltonian"], seed=r["seed"], step=r["step"])
               for r in reps]
    for _ in range(4):
        counts, total = b.sweep(maxima, precision, increment_step=True, temperatures=kts)
        for k, m in enumerate(singles):
            c = m.sweep(TRANSLATE, float(maxima[k]), float(kts[k]), precision, n_sweeps=1, increment_step=True)
            assert (counts[k].accepted, counts[k].rejected) == (c.accepted, c.rejected), k
            assert 0 < c.accepted < c.total()
    for k, m in enumerate(singles):
        pos, step, sub = b.state(k)
        assert np.array_equal(pos, m.positions()), k
        assert (step, sub) == (m.step(), m.substep())


def test_lj_batch_fp32_equals_fp64_and_rejects_overlap_check(ctx):
    # 64 replicas of 8192 bodies at kT in [0.8, 2.0]: the FP32 + recheck batch gives the FP64
    # batch's trajectory; the hard-sphere overlap check does not apply to a soft potential.
    from hoomd_rs_b200 import HmcError
    specs = [(8192, 0.8, 0x5EED0050 + k, 0, 2.5) for k in range(64)]
    kts = np.random.default_rng(5).uniform(0.8, 2.0, 64)
    a = Batch(ctx, lj_replicas(3, specs))
    b = Batch(ctx, lj_replicas(3, specs))
    for _ in range(2):
        ca, ta = a.sweep(0.1, FP32_RECHECK, increment_step=True, temperatures=kts)
        cb, tb = b.sweep(0.1, FP64, increment_step=True, temperatures=kts)
        assert [(c.accepted, c.rejected) for c in ca] == [(c.accepted, c.rejected) for c in cb]
    for k in (0, 17, 63):
        assert np.array_equal(a.positions(k), b.positions(k))
    with pytest.raises(HmcError):
        a.overlap_counts()


def test_batch_sdf_equals_single_system_sdf(ctx):
    # the scale distribution of every replica equals hmc_sdf of the same state in its own system
    reps = replicas(3, SPECS3[:5])
    b = Batch(ctx, reps)
    maxima = np.linspace(0.08, 0.2, len(reps))
    b.sweep(maxima, FP32_RECHECK, n_sweeps=3, increment_step=True)
    counts = b.sdf(0.05, 25)
    assert counts.shape == (len(reps), 25) and counts.sum() > 0
    p = b.pressures(0.05, 25)
    for k, r in enumerate(reps):
        pos, step, sub = b.state(k)
        m = Microstate(ctx, r["boundary"], pos, PairwiseCutoff(HardSphere(1.0)), seed=r["seed"], step=step)
        assert np.array_equal(counts[k], m.sdf(0.05, 25)), k
        assert p[k] == m.pressure(0.05, 25)
    # the batch keeps sweeping correctly after the histograms reused its arrays
    single = Microstate(ctx, reps[0]["boundary"], b.positions(0), PairwiseCutoff(HardSphere(1.0)),
                        seed=reps[0]["seed"], step=b.state(0)[1], substep=b.state(0)[2])
    c, _ = b.sweep(maxima, FP64, increment_step=True)
    cs = single.sweep(TRANSLATE, float(maxima[0]), 1.0, FP64, n_sweeps=1, increment_step=True)
    assert (c[0].accepted, c[0].rejected) == (cs.accepted, cs.rejected)
    assert np.array_equal(b.positions(0), single.positions())


def test_lj_batch_wide_bound_block_recheck_equals_fp64(ctx, monkeypatch):
    # With the FP32 error bound widened 10^4 times most trials of the FP32 batch pass are
    # rechecked by their whole block (several per block, from different replicas); the
    # trajectories must equal the FP64 batch's bit for bit.
    reps = lj_replicas(3, LJ3)
    kts = np.linspace(0.8, 2.0, len(reps))
    monkeypatch.setenv("HMC_B200_FP32_BAND_SCALE", "1e4")
    a = Batch(ctx, reps)
    monkeypatch.delenv("HMC_B200_FP32_BAND_SCALE")
    b = Batch(ctx, reps)
    rechecks, trials = 0, 0
    for _ in range(3):
        ca, ta = a.sweep(0.1, FP32_RECHECK, increment_step=True, temperatures=kts)
        cb, tb = b.sweep(0.1, FP64, increment_step=True, temperatures=kts)
        assert [(c.accepted, c.rejected) for c in ca] == [(c.accepted, c.rejected) for c in cb]
        rechecks += ta.rechecks
        trials += ta.total()
    for k in range(len(reps)):
        assert np.array_equal(a.positions(k), b.positions(k)), k
    assert rechecks > trials // 4, (rechecks, trials)


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
def test_batch_tune_equals_single_system_tune(ctx, precision):
    # every replica's tuned move size equals Microstate.tune on the same state, for hard-sphere
    # and Lennard-Jones batches (per-replica start sizes and temperatures)
    reps = replicas(3, SPECS3[:4])
    b = Batch(ctx, reps)
    b.sweep(0.1, precision, n_sweeps=2, increment_step=True)
    start = np.linspace(0.05, 0.4, len(reps))
    tuned = b.tune(start, precision, 0.3, 3000, 8)
    for k, r in enumerate(reps):
        pos, step, sub = b.state(k)
        m = Microstate(ctx, r["boundary"], pos, PairwiseCutoff(HardSphere(1.0)), seed=r["seed"], step=step,
                       substep=sub)
        assert tuned[k] == m.tune(TRANSLATE, float(start[k]), 1.0, precision, 0.3, 3000, 8), k
    lreps = lj_replicas(3, LJ3)
    lb = Batch(ctx, lreps)
    kts = np.linspace(0.8, 2.0, len(lreps))
    ltuned = lb.tune(0.1, precision, 0.4, 2000, 6, temperatures=kts)
    for k, r in enumerate(lreps):
        m = Microstate(ctx, r["boundary"], r["positions"], r["hamiltonian"], seed=r["seed"], step=r["step"])
        assert ltuned[k] == m.tune(TRANSLATE, 0.1, float(kts[k]), precision, 0.4, 2000, 6), k
    # the batch still sweeps exactly like a single system afterwards
    single = Microstate(ctx, reps[1]["boundary"], b.positions(1), PairwiseCutoff(HardSphere(1.0)),
                        seed=reps[1]["seed"], step=b.state(1)[1], substep=b.state(1)[2])
    c, _ = b.sweep(tuned, precision, increment_step=True)
    cs = single.sweep(TRANSLATE, float(tuned[1]), 1.0, precision, n_sweeps=1, increment_step=True)
    assert (c[1].accepted, c[1].rejected) == (cs.accepted, cs.rejected)
    assert np.array_equal(b.positions(1), single.positions())


def test_batch_of_many_spaces_equals_single_systems(ctx):
    # 64 replicas of 65536 spheres: 5.45 M spaces in the batch, whose space counts are scanned in
    # three kernels (more than 2048 blocks of 2048 spaces); replicas 0 and 63 against single systems
    specs = [(65536, 0.40, 0x5EED0080 + k, 0, "fcc") for k in range(64)]
    reps = replicas(3, specs)
    b = Batch(ctx, reps)
    picks = (0, 63)
    singles = {k: Microstate(ctx, reps[k]["boundary"], reps[k]["positions"], PairwiseCutoff(HardSphere(1.0)),
                             seed=reps[k]["seed"]) for k in picks}
    for _ in range(2):
        counts, _ = b.sweep(0.3, FP32_RECHECK, increment_step=True)
        for k, m in singles.items():
            c = m.sweep(TRANSLATE, 0.3, 1.0, FP32_RECHECK, n_sweeps=1, increment_step=True)
            assert (counts[k].accepted, counts[k].rejected) == (c.accepted, c.rejected), k
    for k, m in singles.items():
        assert np.array_equal(b.positions(k), m.positions()), k


@pytest.mark.parametrize("captured", [False, True])
@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
def test_batch_with_replicas_of_more_colour_sets(ctx, precision, captured):
    # replicas whose checkerboard spaces are 2 or 3 diameters wide hold several bodies per space
    # and run more colour sets per sweep than the others (which run two): the later sets take
    # only their spaces (the late lists); every replica equals its single system
    specs = [(2000, 0.45, 61, 1.0), (3000, 0.50, 62, 2.0), (1500, 0.40, 63, 1.0), (2500, 0.48, 64, 3.0),
             (800, 0.35, 65, 1.0)]
    reps = []
    for n, phi, seed, rng in specs:
        pos, L = lattice.hard_sphere_box(n, phi, 3, seed)
        reps.append({"boundary": Periodic(rng, [L] * 3), "positions": pos, "seed": seed})
    b = Batch(ctx, reps)
    b.set_captured_sweeps(captured)
    singles = [Microstate(ctx, r["boundary"], r["positions"], PairwiseCutoff(HardSphere(1.0)), seed=r["seed"])
               for r in reps]
    for _ in range(3):
        counts, _ = b.sweep(0.2, precision, increment_step=True)
        for k, m in enumerate(singles):
            c = m.sweep(TRANSLATE, 0.2, 1.0, precision, n_sweeps=1, increment_step=True)
            assert (counts[k].accepted, counts[k].rejected) == (c.accepted, c.rejected), k
            assert c.total() >= specs[k][0]  # full colour sets until at least N trials
    for k, m in enumerate(singles):
        assert np.array_equal(b.positions(k), m.positions()), k
        assert m.substep() == 0 and b.state(k)[1:] == (m.step(), m.substep())
