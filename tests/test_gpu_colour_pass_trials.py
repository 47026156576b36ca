"""Decisions of the colour-pass kernels themselves on injected trials (hmc_eval_trials).

hmc_sweep's passes draw each trial from the counter (generate_trial_moves,
hoomd-mc/src/parallel_sweep.rs:231-278). hmc_eval_trials hands the same kernels a list of
injected trials instead: the FP32 sphere pass decides them with its own row walk, its warp
settling of trials inside the FP32 bound and its warp walk of the wrapped rows at the
fast-axis ends; the FP64 sphere pass with its warp-cooperative walk; the Lennard-Jones passes
with their FP32 sums, block-cooperative FP64 recheck and Metropolis test; the cube pass with its
four-trials-per-warp XenoCollide lists. Every decision is compared with the oracle's
delta_energy_one + Metropolis (pairwise_cutoff.rs:919-941, parallel_sweep.rs:267-268) on
adversarial near-contact and near-threshold trials, and the space flag with the checkerboard the
next sweep lays out (hypercuboid.rs:85-128).
"""
import math

import numpy as np
import pytest

import oracle
from hoomd_rs_b200 import (FP32_RECHECK, FP64, ROTATE, TRANSLATE, Context, ConvexPolyhedron, HardShape,
                           HardSphere, Isotropic, LennardJones, Microstate, PairwiseCutoff, Periodic, Shifted,
                           lattice)

pytestmark = pytest.mark.gpu

OUTSIDE, RECHECKED, AMBIGUOUS = 2, 1, 4
CUBE = np.array([[x, y, z] for x in (-0.5, 0.5) for y in (-0.5, 0.5) for z in (-0.5, 0.5)])


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


def wrap(x, L):
    """Periodic<Hypercuboid>::wrap (cuboid.rs:91-103): round half away from zero, 0.5 -> -0.5."""
    lam = x / L
    lam = lam - np.trunc(lam + np.copysign(0.5, lam))
    return np.where(lam == 0.5, -0.5, lam) * L


def space_of(o, x, body_range):
    """Multi-index of each point's checkerboard space for the oracle system's current counter."""
    _, _, step, substep = o.state()
    origin, width, shape = oracle.checkerboard_for_counter(o.L, body_range, step, substep, o.seed)
    idx = np.floor((x - origin) / width)
    idx = np.where(idx == shape.astype(float), 0.0, idx)
    return idx.astype(np.int64)


def near_contact(pos, L, bodies, partners, rng, spread):
    """Trial of body i at sigma (1 + delta) from partner j, delta log-uniform in [1e-17, spread]
    of either sign (a tenth exactly at contact), wrapped like wrap(propose(..))."""
    m = len(bodies)
    v = rng.normal(size=(m, pos.shape[1]))
    v /= np.linalg.norm(v, axis=1)[:, None]
    delta = np.exp(rng.uniform(math.log(1e-17), math.log(spread), m)) * rng.choice([-1.0, 1.0], m)
    delta[::10] = 0.0
    return wrap(pos[partners] + v * (1.0 + delta)[:, None], L)


def sphere_trials(pos, L, n_moves, seed, spread):
    """Half of the trials next to a random other body anywhere in the box, half next to a
    neighbour of the body itself (mostly inside the body's own space, as the sweep's are)."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    n = len(pos)
    half = n_moves // 2
    b1 = rng.integers(0, n, half)
    j1 = (b1 + rng.integers(1, n, half)) % n
    tree = cKDTree(pos + np.asarray(L) / 2, boxsize=np.asarray(L))
    b2 = rng.integers(0, n, n_moves - half)
    _, nb = tree.query(pos[b2] + np.asarray(L) / 2, k=4)
    j2 = nb[np.arange(len(b2)), rng.integers(1, 4, len(b2))]
    bodies = np.concatenate([b1, b2])
    partners = np.concatenate([j1, j2])
    return bodies, near_contact(pos, L, bodies, partners, rng, spread)


@pytest.mark.parametrize("dim,n,phi,total,chunk", [(3, 32768, 0.50, 10_000_000, 1_000_000),
                                                   (2, 4096, 0.70, 10_000_000, 1_000_000)])
def test_sphere_trials_through_the_colour_passes(ctx, dim, n, phi, total, chunk):
    pos0, L = lattice.hard_sphere_box(n, phi, dim, 0x5EED0015)
    h = PairwiseCutoff(HardSphere(1.0))
    g = Microstate(ctx, Periodic(1.0, [L] * dim), pos0, h, seed=0x5EED0015)
    o = oracle.System(dim, [L] * dim, pos0, diameter=1.0, seed=0x5EED0015)
    for _ in range(2):
        c = g.sweep(TRANSLATE, 0.12, 1.0, FP64, n_sweeps=1, increment_step=True)
        a, r = o.parallel_sweep(oracle.TRANSLATE, 0.12, 1.0, 1.0)
        o.increment_step()
        assert (c.accepted, c.rejected) == (a, r)
    pos = o.state()[0]
    assert np.array_equal(g.positions(), pos)
    done, rechecked, accepted, outside = 0, 0, 0, 0
    for k in range(total // chunk):
        spread = (1e-3, 1e-6, 1e-9, 1e-12, 1e-15)[k % 5]
        bodies, trial = sphere_trials(pos, [L] * dim, chunk, seed=2000 + k, spread=spread)
        want, _ = o.eval_moves(bodies, trial, None, np.zeros(chunk), 1.0)
        away = np.any(space_of(o, trial, 1.0) != space_of(o, pos[bodies], 1.0), axis=1)
        for precision in (FP64, FP32_RECHECK):
            got, flags = g.eval_trials(bodies, trial, precision=precision)
            assert np.array_equal(got, want), (precision, k, np.flatnonzero(got != want)[:10])
            assert np.array_equal((flags & OUTSIDE) != 0, away), (precision, k)
            if precision == FP32_RECHECK:
                rechecked += int(((flags & RECHECKED) != 0).sum())
        done += chunk
        accepted += int(want.sum())
        outside += int(away.sum())
    assert done == total
    assert 0 < accepted < total
    assert 0 < outside < total  # both kinds of trial: inside and outside the body's own space
    assert rechecked > total // 1000  # the adversarial set reaches the FP64 settling in the warp


def cube_trials(pos, ori, L, n_moves, seed):
    """Adversarial cube trials: (a) the body's versor equal to a neighbour's up to a rotation of
    1e-k rad, displaced from it along one of its face normals to 1 + delta (faces touching to
    within delta); (b) a random versor next to a random neighbour at 0.95-1.75 (edges and
    vertices); (c) a small translation and rotation of the body's own pose."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    n = len(pos)
    tree = cKDTree(pos + L / 2, boxsize=[L] * 3)
    bodies = rng.integers(0, n, n_moves)
    _, nb = tree.query(pos[bodies] + L / 2, k=6)
    js = nb[np.arange(n_moves), rng.integers(1, 6, n_moves)]
    kind = rng.integers(0, 3, n_moves)
    trial = np.empty((n_moves, 3))
    q = np.empty((n_moves, 4))
    # (a) face contact: the j frame's axis e_a, sign s
    axis = rng.integers(0, 3, n_moves)
    sign = rng.choice([-1.0, 1.0], n_moves)
    delta = np.exp(rng.uniform(math.log(1e-16), math.log(1e-3), n_moves)) * rng.choice([-1.0, 1.0], n_moves)
    delta[::7] = 0.0
    e = np.zeros((n_moves, 3))
    e[np.arange(n_moves), axis] = sign
    qj = ori[js]
    # e rotated by qj: v + s t + x cross t with t = 2 x cross v
    s, x = qj[:, :1], qj[:, 1:]
    t = 2.0 * np.cross(x, e)
    normal = e + s * t + np.cross(x, t)
    tilt_angle = np.exp(rng.uniform(math.log(1e-12), math.log(1e-2), n_moves))
    tilt_axis = rng.normal(size=(n_moves, 3))
    tilt_axis /= np.linalg.norm(tilt_axis, axis=1)[:, None]
    tilt = np.concatenate([np.cos(tilt_angle / 2)[:, None], np.sin(tilt_angle / 2)[:, None] * tilt_axis], axis=1)
    qa = _qmul(tilt, qj)
    pa = pos[js] + normal * (1.0 + delta)[:, None]
    # (b) random versor near a neighbour
    rq = rng.normal(size=(n_moves, 4))
    rq /= np.linalg.norm(rq, axis=1)[:, None]
    v = rng.normal(size=(n_moves, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    pb = pos[js] + v * rng.uniform(0.95, 1.75, n_moves)[:, None]
    # (c) own pose, small move
    small = rng.normal(size=(n_moves, 3)) * 0.05
    sa = np.exp(rng.uniform(math.log(1e-6), math.log(0.2), n_moves))
    sq = np.concatenate([np.cos(sa / 2)[:, None], np.sin(sa / 2)[:, None] * tilt_axis], axis=1)
    pc = pos[bodies] + small
    qc = _qmul(sq, ori[bodies])
    trial = np.where((kind == 0)[:, None], pa, np.where((kind == 1)[:, None], pb, pc))
    q = np.where((kind == 0)[:, None], qa, np.where((kind == 1)[:, None], rq, qc))
    return bodies, wrap(trial, L), q


def _qmul(a, b):
    s1, v1 = a[:, :1], a[:, 1:]
    s2, v2 = b[:, :1], b[:, 1:]
    return np.concatenate([s1 * s2 - np.sum(v1 * v2, axis=1, keepdims=True), s1 * v2 + s2 * v1 + np.cross(v1, v2)],
                          axis=1)


def test_cube_trials_through_the_packed_pass(ctx):
    # 10^7 cube trials (face contacts within 1e-16..1e-3, random edges and vertices, small
    # moves of the body's own pose) decided by the packed XenoCollide pass in both precisions.
    n, phi, seed = 4096, 0.55, 0x5EED0003
    L = (n / phi) ** (1.0 / 3.0)
    positions = lattice.cubic_lattice(n, L, 3, seed, jitter=0.01)
    h = PairwiseCutoff(HardShape(ConvexPolyhedron.with_vertices(CUBE)))
    g = Microstate(ctx, Periodic(math.sqrt(3.0), [L] * 3), positions, h, seed=seed)
    o = oracle.System(3, [L] * 3, positions, None, seed=seed, interaction=oracle.HARD_CONVEX_POLYHEDRON,
                      vertices=CUBE)
    for sweep in range(4):
        move, maximum = (TRANSLATE, 0.08) if sweep % 2 == 0 else (ROTATE, 0.1)
        c = g.sweep(move, maximum, 1.0, FP64, n_sweeps=1, increment_step=True)
        a, r = o.parallel_sweep(oracle.TRANSLATE if move == TRANSLATE else oracle.ROTATE, maximum, 1.0,
                                math.sqrt(3.0))
        o.increment_step()
        assert (c.accepted, c.rejected) == (a, r)
    pos, ori, _, _ = o.state()
    total, chunk = 10_000_000, 1_000_000
    accepted = 0
    for k in range(total // chunk):
        bodies, trial, q = cube_trials(pos, ori, L, chunk, seed=3000 + k)
        want, _ = o.eval_moves(bodies, trial, q, np.zeros(chunk), 1.0)
        away = np.any(space_of(o, trial, math.sqrt(3.0)) != space_of(o, pos[bodies], math.sqrt(3.0)), axis=1)
        for precision in (FP64, FP32_RECHECK):
            got, flags = g.eval_trials(bodies, trial, precision=precision, orientations=q)
            assert np.array_equal(got, want), (precision, k, np.flatnonzero(got != want)[:10])
            assert np.array_equal((flags & OUTSIDE) != 0, away), (precision, k)
        accepted += int(want.sum())
    assert 0 < accepted < total


def test_lj_trials_through_the_colour_passes(ctx):
    # 10^7 Lennard-Jones trials (rho = 0.8, r_cut = 2.5): small moves of each body, a third with
    # u within 1e-16..1e-3 of the threshold exp(-dU/kT) and some exactly at it. Where the oracle
    # (which sums the same pair energies in body order) and the pass disagree, the pass must have
    # flagged the trial order-ambiguous: its dU lies within the any-order summation bound of the
    # threshold. Trials outside the body's space are rejected unevaluated, as in the sweep.
    n, rho, kt, seed = 1 << 14, 0.8, 1.0, 0x5EED0005
    pos0, L = lattice.lennard_jones_box(n, rho, 3, seed)
    h = PairwiseCutoff(Isotropic(Shifted(LennardJones(1.0, 1.0), 2.5), 2.5))
    g = Microstate(ctx, Periodic(2.5, [L] * 3), pos0, h, seed=seed)
    o = oracle.System(3, [L] * 3, pos0, seed=seed, interaction=oracle.LENNARD_JONES, lj_r_cut=2.5, lj_r_shift=2.5)
    for _ in range(2):
        c = g.sweep(TRANSLATE, 0.1, kt, FP64, n_sweeps=1, increment_step=True)
        a, r = o.parallel_sweep(oracle.TRANSLATE, 0.1, kt, 2.5)
        o.increment_step()
        assert (c.accepted, c.rejected) == (a, r)
        assert c.order_ambiguous == 0
    pos = o.state()[0]
    total, chunk = 10_000_000, 1_000_000
    stats = {"ambiguous": 0, "ambiguous_off_edge": 0, "disagree": 0, "outside": 0, "rechecked": 0, "edge": 0}
    for k in range(total // chunk):
        rng = np.random.default_rng(4000 + k)
        bodies = rng.integers(0, n, chunk)
        disp = rng.normal(size=(chunk, 3)) * rng.choice([0.02, 0.1, 0.25], chunk)[:, None]
        trial = wrap(pos[bodies] + disp, L)
        _, dh = o.eval_moves(bodies, trial, None, np.zeros(chunk), kt)
        u = rng.random(chunk)
        thr = np.exp(-np.clip(dh, -700, 700) / kt)
        pick = rng.random(chunk)
        rel = np.exp(rng.uniform(math.log(1e-16), math.log(1e-3), chunk)) * rng.choice([-1.0, 1.0], chunk)
        near = (pick < 0.33) & (dh > 0)
        exact = (pick > 0.95) & (dh > 0)
        u = np.where(near, np.clip(thr * (1 + rel), 0.0, 1.0 - 2.0 ** -53), u)
        u = np.where(exact, np.minimum(thr, 1.0 - 2.0 ** -53), u)
        want, _ = o.eval_moves(bodies, trial, None, u, kt)
        away = np.any(space_of(o, trial, 2.5) != space_of(o, pos[bodies], 2.5), axis=1)
        want = want & ~away
        for precision in (FP64, FP32_RECHECK):
            got, flags = g.eval_trials(bodies, trial, u, kt, precision)
            assert np.array_equal((flags & OUTSIDE) != 0, away), (precision, k)
            amb = (flags & AMBIGUOUS) != 0
            bad = got != want
            assert not np.any(bad & ~amb), (precision, k, np.flatnonzero(bad & ~amb)[:10])
            stats["ambiguous"] += int(amb.sum())
            stats["ambiguous_off_edge"] += int((amb & ~(near | exact)).sum())
            stats["disagree"] += int(bad.sum())
            if precision == FP32_RECHECK:
                stats["rechecked"] += int(((flags & RECHECKED) != 0).sum())
        stats["outside"] += int(away.sum())
        stats["edge"] += int((near | exact).sum())
    print("lj trials:", stats)
    assert stats["rechecked"] > 0
    # the flag marks the trials built to sit within ~1e-12 of the threshold; among the others
    # (uniform u) it is all but absent
    assert stats["ambiguous"] < stats["edge"] * 2
    assert stats["ambiguous_off_edge"] < 1e-5 * 2 * (total - stats["edge"])
