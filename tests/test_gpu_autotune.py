"""Launch variants and the autotuner (hmc_autotune, hmc_batch_autotune).

Every colour-pass kernel is compiled in a few launch shapes (register cap, trials per warp,
candidates a lane tests before its warp takes over); each makes the same pair tests, so every
variant must give the identical trajectory. The autotuner times the variants from a saved state
and must leave the state and the counter as it found them, and record its choice for other
systems with the same pass, dimension, precision and density band.
"""
import math

import numpy as np
import pytest

from hoomd_rs_b200 import (FP32_RECHECK, FP64, ROTATE, TRANSLATE, Batch, Context, ConvexPolyhedron, HardShape,
                           HardSphere, Isotropic, LennardJones, Microstate, PairwiseCutoff, Periodic, Shifted,
                           lattice)

pytestmark = pytest.mark.gpu

CUBE = np.array([[x, y, z] for x in (-0.5, 0.5) for y in (-0.5, 0.5) for z in (-0.5, 0.5)])


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


def spheres(ctx, dim=3, n=32768, phi=0.5, seed=0x5EED0021):
    pos, L = lattice.hard_sphere_box(n, phi, dim, seed)
    return lambda: Microstate(ctx, Periodic(1.0, [L] * dim), pos, PairwiseCutoff(HardSphere(1.0)), seed=seed)


def lj(ctx, n=4096, seed=0x5EED0022):
    pos, L = lattice.lennard_jones_box(n, 0.8, 3, seed)
    h = PairwiseCutoff(Isotropic(Shifted(LennardJones(1.0, 1.0), 2.5), 2.5))
    return lambda: Microstate(ctx, Periodic(2.5, [L] * 3), pos, h, seed=seed)


def cubes(ctx, n=4096, phi=0.55, seed=0x5EED0023):
    L = (n / phi) ** (1.0 / 3.0)
    pos = lattice.cubic_lattice(n, L, 3, seed, jitter=0.01)
    h = PairwiseCutoff(HardShape(ConvexPolyhedron.with_vertices(CUBE)))
    return lambda: Microstate(ctx, Periodic(math.sqrt(3.0), [L] * 3), pos, h, seed=seed)


def squares(ctx, n=4096, seed=0x5EED0024):
    from hoomd_rs_b200 import ConvexPolygon
    sq = np.array([[-0.5, -0.5], [0.5, -0.5], [0.5, 0.5], [-0.5, 0.5]])
    L = math.sqrt(n / 0.6)
    pos = lattice.cubic_lattice(n, L, 2, seed, jitter=0.0)
    ang = np.random.default_rng(seed).uniform(-0.2, 0.2, n)
    h = PairwiseCutoff(HardShape(ConvexPolygon.with_vertices(sq)))
    return lambda: Microstate(ctx, Periodic(math.sqrt(2.0), [L, L]), pos, h, seed=seed, orientations=ang)


def run(g, moves, precision, kt=1.0):
    counts = []
    for move, maximum in moves:
        c = g.sweep(move, maximum, kt, precision, n_sweeps=1, increment_step=True)
        counts.append((c.accepted, c.rejected))
    return counts


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
@pytest.mark.parametrize("kind", ["spheres3", "disks", "lj", "cubes", "squares"])
def test_every_variant_gives_the_same_trajectory(ctx, kind, precision):
    make, moves = {
        "spheres3": (spheres(ctx), [(TRANSLATE, 0.2)] * 3),
        "disks": (spheres(ctx, 2, 4096, 0.7), [(TRANSLATE, 0.1)] * 4),
        "lj": (lj(ctx), [(TRANSLATE, 0.1)] * 3),
        "cubes": (cubes(ctx), [(TRANSLATE, 0.08), (ROTATE, 0.1), (TRANSLATE, 0.08)]),
        "squares": (squares(ctx), [(TRANSLATE, 0.1), (ROTATE, 0.1), (TRANSLATE, 0.1)]),
    }[kind]
    ref = make()
    count = ref.launch_variant(precision)["count"]
    ref.set_launch_variant(precision, 0)
    want = run(ref, moves, precision)
    pos, ori = ref.positions(), (ref.orientations() if kind in ("cubes", "squares") else None)
    for v in range(1, count):
        g = make()
        g.set_launch_variant(precision, v)
        assert g.launch_variant(precision)["index"] == v
        assert run(g, moves, precision) == want, v
        assert np.array_equal(g.positions(), pos), v
        if ori is not None:
            assert np.array_equal(g.orientations(), ori), v
        g.close()


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
def test_autotune_restores_state_and_records_its_choice(ctx, precision):
    make = spheres(ctx, 3, 65536, 0.5, seed=0x5EED0024)
    g = make()
    g.sweep(TRANSLATE, 0.2, 1.0, precision, n_sweeps=2, increment_step=True)
    before, step, sub = g.state()
    chosen, ms = g.autotune(TRANSLATE, 0.2, 1.0, precision, sweeps=3)
    assert len(ms) == chosen["count"] and np.all(ms > 0)
    assert ms[chosen["index"]] == ms.min()
    after, step2, sub2 = g.state()
    assert np.array_equal(before, after) and (step, sub) == (step2, sub2)
    assert g.launch_variant(precision)["index"] == chosen["index"]
    # the sweep after autotuning equals a fresh system's from the same state
    twin = make()
    twin.set_state(before, step, sub)
    c1 = g.sweep(TRANSLATE, 0.2, 1.0, precision, n_sweeps=2, increment_step=True)
    c2 = twin.sweep(TRANSLATE, 0.2, 1.0, precision, n_sweeps=2, increment_step=True)
    assert (c1.accepted, c1.rejected) == (c2.accepted, c2.rejected)
    assert np.array_equal(g.positions(), twin.positions())
    # the recorded choice (pass and variant) applies to another system of the same workload
    # (same density band)
    assert twin.cooperative_pass(precision) == g.cooperative_pass(precision)
    assert twin.launch_variant(precision)["index"] == chosen["index"]


def test_batch_variants_and_autotune(ctx):
    rng = np.random.default_rng(5)
    reps = []
    for k in range(12):
        n = int(np.exp(rng.uniform(math.log(512), math.log(4096))))
        pos, L = lattice.hard_sphere_box(n, float(rng.uniform(0.40, 0.54)), 3, 300 + k)
        reps.append({"boundary": Periodic(1.0, [L] * 3), "positions": pos, "seed": 300 + k})
    maxima = np.full(len(reps), 0.15)
    ref = Batch(ctx, reps)
    ref.set_launch_variant(FP32_RECHECK, 0)
    want, _ = ref.sweep(maxima, FP32_RECHECK, n_sweeps=2, increment_step=True)
    for v in (1, 2, 3, 4, 5):
        b = Batch(ctx, reps)
        b.set_launch_variant(FP32_RECHECK, v)
        got, _ = b.sweep(maxima, FP32_RECHECK, n_sweeps=2, increment_step=True)
        assert [(c.accepted, c.rejected) for c in got] == [(c.accepted, c.rejected) for c in want], v
        for k in range(len(reps)):
            assert np.array_equal(b.positions(k), ref.positions(k)), (v, k)
    b = Batch(ctx, reps)
    before = [b.state(k) for k in range(len(reps))]
    chosen, ms = b.autotune(maxima, FP32_RECHECK, sweeps=2)
    assert len(ms) == chosen["count"] == 6 and ms[chosen["index"]] == ms.min()
    for k in range(len(reps)):
        pos, step, sub = b.state(k)
        assert np.array_equal(pos, before[k][0]) and (step, sub) == before[k][1:]


def test_lj_batch_variants_give_the_same_trajectory(ctx):
    # the Lennard-Jones replica pass in every compiled launch shape, both precision modes
    h = PairwiseCutoff(Isotropic(Shifted(LennardJones(1.0, 1.0), 2.5), 2.5))
    reps = []
    for k in range(6):
        pos, L = lattice.lennard_jones_box(2048, 0.8, 3, 400 + k)
        reps.append({"boundary": Periodic(2.5, [L] * 3), "positions": pos, "seed": 400 + k, "hamiltonian": h})
    kts = np.linspace(0.8, 2.0, len(reps))
    for precision in (FP64, FP32_RECHECK):
        ref = Batch(ctx, reps)
        ref.set_launch_variant(precision, 0)
        want, _ = ref.sweep(0.1, precision, n_sweeps=2, increment_step=True, temperatures=kts)
        for v in (1, 2, 3, 4):
            b = Batch(ctx, reps)
            b.set_launch_variant(precision, v)
            got, _ = b.sweep(0.1, precision, n_sweeps=2, increment_step=True, temperatures=kts)
            assert [(c.accepted, c.rejected) for c in got] == [(c.accepted, c.rejected) for c in want], (precision, v)
            for k in range(len(reps)):
                assert np.array_equal(b.positions(k), ref.positions(k)), (precision, v, k)


@pytest.mark.parametrize("dim,n,phi", [(3, 32768, 0.5), (2, 4096, 0.7)])
def test_cooperative_and_one_lane_passes_give_the_same_trajectory(ctx, dim, n, phi):
    make = spheres(ctx, dim, n, phi, seed=0x5EED0025)
    for precision in (FP64, FP32_RECHECK):
        runs = []
        for coop in (False, True):
            g = make()
            g.set_cooperative_pass(precision, coop)
            runs.append((run(g, [(TRANSLATE, 0.2 if dim == 3 else 0.1)] * 3, precision), g.positions()))
            g.close()
        assert runs[0][0] == runs[1][0], precision
        assert np.array_equal(runs[0][1], runs[1][1]), precision
