"""GPU state preparation against the oracle: the overlap-penalty sphere (ParallelSweep and the
serial Sweep), QuickInsert (one warp, sequential insertions) and QuickCompress (host state
machine, device mapping and energies), and the benchmark placement loop built from them
(benchmarks/src/place.rs:31-110). Positions, counters and boxes must equal the oracle's bit
for bit (the penalty's energy sums are formed in another order than the oracle's; a decision
could differ only where |dH| or |u - exp(-dH)| is below ~1e-12)."""
import math

import numpy as np
import pytest

import oracle
from hoomd_rs_b200 import (FP32_RECHECK, FP64, TRANSLATE, Context, Expanded, HardSphere, HmcError, Isotropic,
                           Microstate, OverlapPenalty, PairwiseCutoff, Periodic, QuickCompress, QuickInsert, lattice,
                           place_single_site_point_bodies)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


def penalty_h(d=1.0, k=10000.0, dmax=0.2, eps=100.0):
    return PairwiseCutoff(Isotropic(Expanded(d, OverlapPenalty(k, dmax, eps)), d))


def pair(ctx, dim, L, pos, seed, capacity=0, d=1.0):
    g = Microstate(ctx, Periodic(d, L), pos, penalty_h(d), seed=seed, capacity=capacity)
    o = oracle.System(dim, L, pos, seed=seed, interaction=oracle.OVERLAP_PENALTY, diameter=d)
    return g, o


def same_state(g, o):
    po, _, step, sub = o.state()
    pg = g.positions()
    assert g.n == o.n_bodies
    assert np.array_equal(pg, po)
    assert g._counter() == (step, sub)


def test_penalty_pair_energy_known_answers(ctx):
    # overlap_penalty.rs tests (shoulder, core, harmonic) through the device total energy
    for x, k, dmax, eps, want in [(-0.5, 0.0, 1.0, 15.0, 15.0), (-2.0 ** -53, 0.0, 1.0, 15.0, 15.0),
                                  (0.0, 0.0, 1.0, 15.0, 0.0), (-0.5 - 2.0 ** -53, 0.0, 0.5, 0.0, math.inf),
                                  (-0.125, 6.0, 10.0, 0.0, 0.5 * 6.0 * 0.125 ** 2)]:
        g = Microstate(ctx, Periodic(1.0, [10.0] * 3), [[0.0, 0.0, 0.0], [1.0 + x, 0.0, 0.0]],
                       PairwiseCutoff(Isotropic(Expanded(1.0, OverlapPenalty(k, dmax, eps)), 1.0)))
        assert g.total_energy() == want


@pytest.mark.parametrize("dim", [2, 3])
def test_penalty_sweeps_bit_identical(ctx, dim):
    n = 2000
    rho = 0.9 if dim == 3 else 0.8
    L = (n / rho) ** (1.0 / dim)
    pos = (np.random.default_rng(dim).random((n, dim)) - 0.5) * L  # random: many penalty overlaps
    g, o = pair(ctx, dim, [L] * dim, pos, seed=21 + dim)
    assert g.total_energy() == pytest.approx(o.total_energy(), rel=1e-12)
    for sweep in range(6):
        if sweep % 2 == 0:
            c = g.serial_sweep(0.1, n_sweeps=1)
            a, r = o.serial_sweep(oracle.TRANSLATE, 0.1, 1.0)
        else:
            c = g.sweep(TRANSLATE, 0.1, 1.0, FP32_RECHECK, n_sweeps=1)  # the penalty runs in FP64
            a, r = o.parallel_sweep(oracle.TRANSLATE, 0.1, 1.0, 1.0)
        assert (c.accepted, c.rejected) == (a, r), sweep
        same_state(g, o)
    assert g.total_energy() == pytest.approx(o.total_energy(), rel=1e-9)


@pytest.mark.parametrize("soft", [False, True])
def test_quick_insert_bit_identical(ctx, soft):
    n, L = 3000, 16.0
    h = penalty_h() if soft else PairwiseCutoff(HardSphere(1.0))
    g = Microstate(ctx, Periodic(1.0, [L] * 3), np.zeros((0, 3)), h, seed=5, capacity=n)
    o = oracle.System(3, [L] * 3, np.zeros((0, 3)), seed=5,
                      interaction=oracle.OVERLAP_PENALTY if soft else oracle.HARD_SPHERE)
    qi = QuickInsert(n)
    oq = {"target": n, "allowed_overlaps": max(n // 8, 1), "inserted": 0, "complete": 0}
    for k in range(40):
        c = qi.apply(g)
        a, r = o.quick_insert(oq)
        assert (c.accepted, c.rejected) == (a, r), k
        assert (qi.inserted, qi.is_complete()) == (oq["inserted"], bool(oq["complete"]))
        same_state(g, o)
        if qi.is_complete():
            break
        g.serial_sweep(0.1)
        o.serial_sweep(oracle.TRANSLATE, 0.1, 1.0)
    assert g.n > 0


def test_quick_insert_reference_case(ctx):
    # quick_insert.rs tests::hard_spheres in a periodic 6 x 6 box
    g = Microstate(ctx, Periodic(1.0, [6.0, 6.0]), [[0.0, 0.0]], PairwiseCutoff(HardSphere(1.0)), capacity=11)
    qi = QuickInsert(10)
    for _ in range(100):
        qi.apply(g)
        if qi.is_complete():
            break
    g.serial_sweep(0.1)
    assert qi.inserted == 10 and qi.is_complete()
    assert g.n == 11
    assert g.total_energy() == 0.0
    with pytest.raises(HmcError):
        QuickInsert(5).apply(g)  # no capacity left


def test_set_box_bit_identical(ctx):
    rng = np.random.default_rng(8)
    L = np.array([7.0, 9.0, 11.0])
    pos = (rng.random((500, 3)) - 0.5) * L
    g, o = pair(ctx, 3, L, pos, seed=3)
    for f in (0.97, 1.05, 0.9):
        L = L * f
        g.set_box(L)
        o.set_box(L)
        same_state(g, o)
        assert np.array_equal(g.box(), o.box())


def _place_pair(g, o, n, rho, dim, sweeps, max_steps=4000):
    qi, qc = QuickInsert(n), QuickCompress.with_target_volume(n / rho)
    oqi = {"target": n, "allowed_overlaps": max(n // 8, 1), "inserted": 0, "complete": 0}
    oqc = {"target_volume": n / rho, "maximum_energy_per_site": 1000.0, "maximum_delta": 0.05, "state": 0,
           "is_final": 0, "boundary": [0.0, 0.0, 0.0]}
    for step in range(max_steps):
        if step % 20 == 0:
            if qi.is_complete():
                qc.apply(g)
                o.quick_compress(oqc)
                assert qc.state == oqc["state"]
                assert np.array_equal(g.box(), o.box())
            else:
                qi.apply(g)
                o.quick_insert(oqi)
        if sweeps == "serial":
            g.serial_sweep(0.1)
            o.serial_sweep(oracle.TRANSLATE, 0.1, 1.0)
        else:
            g.sweep(TRANSLATE, 0.1, 1.0, FP64, n_sweeps=1)
            o.parallel_sweep(oracle.TRANSLATE, 0.1, 1.0, 1.0)
        g.increment_step()
        o.increment_step()
        if qc.is_complete():
            break
    return qi, qc


@pytest.mark.parametrize("dim,sweeps", [(2, "serial"), (3, "parallel")])
def test_placement_loop_bit_identical(ctx, dim, sweeps):
    n, rho = 400, (0.8 if dim == 2 else 0.85)
    L0 = (n / (0.7 * rho)) ** (1.0 / dim)
    g, o = pair(ctx, dim, [L0] * dim, np.zeros((0, dim)), seed=0x5EED0002, capacity=n)
    qi, qc = _place_pair(g, o, n, rho, dim, sweeps)
    assert qi.is_complete() and qc.is_complete()
    same_state(g, o)
    assert g.volume() == pytest.approx(n / rho, rel=1e-12)
    assert g.total_energy() == 0.0 == o.total_energy()


def test_placement_large_reaches_target(ctx):
    # device only: 2^14 spheres to the headline density, ParallelSweep between applications
    n, phi = 1 << 14, 0.50
    rho = phi / (math.pi / 6.0)
    L0 = (n / (0.7 * rho)) ** (1.0 / 3.0)
    g = Microstate(ctx, Periodic(1.0, [L0] * 3), np.zeros((0, 3)), penalty_h(), seed=9, capacity=n)
    qi, qc = QuickInsert(n), QuickCompress.with_target_volume(n / rho)
    for step in range(20000):
        if step % 20 == 0:
            (qc if qi.is_complete() else qi).apply(g)
        g.sweep(TRANSLATE, 0.1, 1.0, FP64, n_sweeps=1)
        g.increment_step()
        if qc.is_complete():
            break
    assert qc.is_complete() and g.n == n
    assert g.volume() == pytest.approx(n / rho, rel=1e-12)
    hard = Microstate(ctx, Periodic(1.0, list(g.box())), g.positions(), PairwiseCutoff(HardSphere(1.0)))
    assert hard.overlap_count() == 0


def test_grand_canonical_reference_case(ctx):
    # grand_canonical.rs tests::hard_spheres_fugacity in a periodic 6 x 6 box
    from hoomd_rs_b200 import GrandCanonical, IsothermalIsofugacity
    g = Microstate(ctx, Periodic(1.0, [6.0, 6.0]), [[0.0, 0.0]], PairwiseCutoff(HardSphere(1.0)), capacity=64)
    qi = QuickInsert(10)
    for _ in range(100):
        qi.apply(g)
        if qi.is_complete():
            break
    g.serial_sweep(0.1)
    assert qi.is_complete() and g.n == 11 and g.total_energy() == 0.0
    gc = GrandCanonical()
    c = gc.apply(g, None, IsothermalIsofugacity(1.0, 0.0), n_trials=100)
    assert g.n == 0 and c.remove_accepted == 11 and c.insert_accepted == 0
    gc.apply(g, None, IsothermalIsofugacity(1.0, 1.0), n_trials=100)
    assert g.n > 0 and g.total_energy() == 0.0


@pytest.mark.parametrize("soft", [False, True])
def test_grand_canonical_bit_identical(ctx, soft, tmp_path):
    from hoomd_rs_b200 import GrandCanonical, IsothermalIsofugacity
    from hoomd_rs_b200.gsd import GsdFile, HoomdGsdFile
    n, L = 600, 12.0
    pos = lattice.cubic_lattice(n, L, 3, 4, jitter=0.01)
    h = penalty_h() if soft else PairwiseCutoff(HardSphere(1.0))
    g = Microstate(ctx, Periodic(1.0, [L] * 3), pos, h, seed=17, capacity=4000)
    o = oracle.System(3, [L] * 3, pos, seed=17, interaction=oracle.OVERLAP_PENALTY if soft else oracle.HARD_SPHERE)
    gc = GrandCanonical()
    path = tmp_path / "gc.gsd"
    f = HoomdGsdFile.create(path)
    for k, (fug, trials) in enumerate([(0.05, 300), (0.5, 500), (0.0, 200), (2.0, 700), (0.2, 400)]):
        c = gc.apply(g, None, IsothermalIsofugacity(1.0, fug), n_trials=trials)
        oc = o.grand_canonical(1.0, fug, trials)
        assert (c.insert_accepted, c.insert_rejected, c.remove_accepted, c.remove_rejected) == oc, k
        same_state(g, o)
        f.append_microstate(g).end()
        want, _ = o.gsd_frame()  # rows in tag order
        f.sync_all()
        got = GsdFile.open(path).iter_arrays(k, "particles/position", np.float32, 3)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
        g.serial_sweep(0.1)
        o.serial_sweep(oracle.TRANSLATE, 0.1, 1.0)
        same_state(g, o)
    f.close()


def test_place_single_site_point_bodies_equals_the_oracle(ctx):
    # the library's place.rs:31-110 loop against the same loop on the oracle
    n, rho, dim = 300, 0.8, 2
    g = place_single_site_point_bodies(ctx, n, rho, 1.0, penalty_h(), dim, seed=0x5EED0043)
    L0 = (n / (0.7 * rho)) ** (1.0 / dim)
    o = oracle.System(dim, [L0] * dim, np.zeros((0, dim)), seed=0x5EED0043, interaction=oracle.OVERLAP_PENALTY,
                      diameter=1.0)
    oqi = {"target": n, "allowed_overlaps": max(n // 8, 1), "inserted": 0, "complete": 0}
    oqc = {"target_volume": n / rho, "maximum_energy_per_site": 1000.0, "maximum_delta": 0.05, "state": 0,
           "is_final": 0, "boundary": [0.0, 0.0, 0.0]}
    while oqc["state"] != 3:
        if o.state()[2] % 20 == 0:
            (o.quick_compress if oqi["complete"] else o.quick_insert)(oqc if oqi["complete"] else oqi)
        o.serial_sweep(oracle.TRANSLATE, 0.1, 1.0)
        o.increment_step()
    same_state(g, o)
    assert g.total_energy() == 0.0 == o.total_energy()
