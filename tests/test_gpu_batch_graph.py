"""Captured batch sweeps (hmc_batch_set_captured_sweeps): each sweep is one launch of a CUDA graph
whose rounds loop, checkerboard origins, counts and Counters stay on the device. The sweeps of a
call then run back to back with one wait at the end, and must give the launched sweeps' trajectory,
counts and Counters bit for bit."""
import numpy as np
import pytest

from hoomd_rs_b200 import FP32_RECHECK, FP64, Batch, Context

from test_gpu_batch import LJ2, LJ3, SPECS2, SPECS3, lj_replicas, replicas

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


def fields(c):
    return (c.accepted, c.rejected, c.rechecks, c.pair_checks, c.max_fp32_error, c.order_ambiguous)


def same_state(a, b, n):
    for k in range(n):
        pa, sa, ua = a.state(k)
        pb, sb, ub = b.state(k)
        assert np.array_equal(pa, pb), k
        assert (sa, ua) == (sb, ub), k


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
@pytest.mark.parametrize("dim,specs", [(3, SPECS3), (2, SPECS2)])
def test_captured_hard_sphere_sweeps_equal_launched(ctx, dim, specs, precision):
    reps = replicas(dim, specs)
    maxima = np.linspace(0.08, 0.3, len(reps))
    a, b = Batch(ctx, reps), Batch(ctx, reps)
    b.set_captured_sweeps(True)
    for increment_step, n_sweeps in ((True, 4), (False, 3), (True, 1)):
        want = [[0, 0] for _ in reps]
        tot = [0, 0, 0, 0, 0.0, 0]
        for _ in range(n_sweeps):
            ca, ta = a.sweep(maxima, precision, increment_step=increment_step)
            for k, c in enumerate(ca):
                want[k][0] += c.accepted
                want[k][1] += c.rejected
            f = fields(ta)
            tot = [x + y for x, y in zip(tot[:4], f[:4])] + [max(tot[4], f[4]), tot[5] + f[5]]
        cb, tb = b.sweep(maxima, precision, n_sweeps=n_sweeps, increment_step=increment_step)
        assert [[c.accepted, c.rejected] for c in cb] == want
        assert list(fields(tb)) == tot
        same_state(a, b, len(reps))
    assert not b.overlap_counts().any()


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
@pytest.mark.parametrize("dim,specs", [(3, LJ3), (2, LJ2)])
def test_captured_lj_sweeps_equal_launched(ctx, dim, specs, precision):
    reps = lj_replicas(dim, specs)
    maxima = np.linspace(0.08, 0.2, len(reps))
    kts = np.linspace(0.8, 2.0, len(reps))
    a, b = Batch(ctx, reps), Batch(ctx, reps)
    b.set_captured_sweeps(True)
    want = [[0, 0] for _ in reps]
    for _ in range(3):
        ca, _ = a.sweep(maxima, precision, increment_step=True, temperatures=kts)
        for k, c in enumerate(ca):
            want[k][0] += c.accepted
            want[k][1] += c.rejected
    cb, tb = b.sweep(maxima, precision, n_sweeps=3, increment_step=True, temperatures=kts)
    assert [[c.accepted, c.rejected] for c in cb] == want
    assert tb.order_ambiguous == 0
    same_state(a, b, len(reps))


def test_captured_graph_follows_precision_variant_and_mode_changes(ctx):
    # the graph is rebuilt when the precision, the launch variant or increment_step changes, and
    # captured and launched sweeps can follow one another on the same batch
    reps = replicas(3, SPECS3[:4])
    maxima = np.full(len(reps), 0.2)
    a, b = Batch(ctx, reps), Batch(ctx, reps)
    plan = [(FP32_RECHECK, None, True, True), (FP64, None, True, True), (FP32_RECHECK, 2, True, True),
            (FP64, None, False, False), (FP32_RECHECK, 1, True, False), (FP64, 0, False, True)]
    for precision, variant, captured, inc in plan:
        for x in (a, b):
            x.set_launch_variant(precision, variant)
        b.set_captured_sweeps(captured)
        ca, ta = a.sweep(maxima, precision, n_sweeps=1, increment_step=inc)
        cb, tb = b.sweep(maxima, precision, n_sweeps=1, increment_step=inc)
        assert [(c.accepted, c.rejected) for c in ca] == [(c.accepted, c.rejected) for c in cb]
        assert fields(ta) == fields(tb)
    same_state(a, b, len(reps))


def test_captured_sweeps_count_their_kernels(ctx):
    reps = replicas(3, SPECS3[:3])
    b = Batch(ctx, reps)
    b.set_captured_sweeps(True)
    k0 = b.kernel_launches()
    _, t = b.sweep(np.full(len(reps), 0.2), FP32_RECHECK, n_sweeps=2, increment_step=True)
    # per sweep: origins, the six rebuild kernels, rounds, the loop's first test, the end; per
    # colour set: 8 colour passes and the step to the next set
    launched = b.kernel_launches() - k0
    assert launched >= 2 * 10 + 2 * 9
    assert (launched - 20) % 9 == 0


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
def test_one_replica_batch_captured_equals_single_system(ctx, precision):
    # a single system run as a one-replica batch with captured sweeps: the same trajectory as
    # the Microstate's own sweeps (2-D disks at area fraction 0.70, 40 sweeps in one call)
    from hoomd_rs_b200 import TRANSLATE, HardSphere, Microstate, PairwiseCutoff, Periodic, lattice
    pos, L = lattice.hard_sphere_box(4096, 0.70, 2, 0x5EED0061)
    b = Batch(ctx, [{"boundary": Periodic(1.0, [L, L]), "positions": pos, "seed": 0x5EED0061}])
    b.set_captured_sweeps(True)
    m = Microstate(ctx, Periodic(1.0, [L, L]), pos, PairwiseCutoff(HardSphere(1.0)), seed=0x5EED0061)
    counts, total = b.sweep(0.1, precision, n_sweeps=40, increment_step=True)
    c = m.sweep(TRANSLATE, 0.1, 1.0, precision, n_sweeps=40, increment_step=True)
    assert (counts[0].accepted, counts[0].rejected) == (c.accepted, c.rejected)
    assert np.array_equal(b.positions(0), m.positions())
    assert b.state(0)[1:] == (m.step(), m.substep())
