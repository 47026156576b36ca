"""The trial-move samplers, pinned by the reference's own statistical tests and by distribution
tests, on the oracle's restatement (the device's samples equal the oracle's bit for bit:
tests/test_gpu_samplers.py).

The reference draws its normals and uniforms through rand 0.10.4 and rand_distr 0.6.0, which are
not part of the reference tree; no reference test pins their outputs bit for bit, only
statistically (hoomd-mc/src/translate/cartesian.rs:65-100, rotate/versor.rs:151-184,
rotate/angle.rs:83-119). Those tests are restated here with their sample sizes and tolerances, on
the counter streams the sweep draws from (Counter(step, substep, seed).index(i), one sample per
index), together with Kolmogorov-Smirnov tests of the distributions each sampler must produce,
and a derivation of the 256-layer ziggurat tables from the ZIGNOR construction (Doornik 2005).
"""
import math

import numpy as np
import pytest
from scipy import stats

import oracle

TRANSLATE, ROTATE, NORMAL = 0, 1, 2


def arc_distance_from_identity(q):
    """Versor::arc_distance (hoomd-vector/src/quaternion.rs:622-625) of q from the identity:
    atan2(|vector part|, scalar)."""
    return np.arctan2(np.linalg.norm(q[:, 1:], axis=1), q[:, 0])


@pytest.mark.parametrize("d", [0.1, 1.0])
def test_translate_reference_statistics(d):
    # translate/cartesian.rs:65-100: N = 2048 proposals from a body at (1, -5, 2.5)
    n = 2048
    dv = oracle.sample_moves(3, TRANSLATE, d, n, seed=1)
    norm = np.linalg.norm(dv, axis=1)
    assert norm.max() <= d
    assert norm.min() < d * 0.1
    assert norm.max() > d * 0.9
    assert np.all(np.abs(dv.mean(axis=0)) < d * 0.1)


@pytest.mark.parametrize("a", [0.1, 1.0, 1.53])
def test_rotate_versor_reference_statistics(a):
    # rotate/versor.rs:151-184: N = 65536, mean arc distance within 0.1 a of 0.75 a
    q = oracle.sample_moves(3, ROTATE, a, 65536, seed=1)
    mean = abs(arc_distance_from_identity(q).mean())
    assert abs(mean - 0.75 * a) < 0.1 * a


@pytest.mark.parametrize("a", [0.1, 1.0])
def test_rotate_angle_reference_statistics(a):
    # rotate/angle.rs:83-119: N = 1024
    th = oracle.sample_moves(2, ROTATE, a, 1024, seed=1)
    assert np.abs(th).max() <= a
    assert np.abs(th).min() < a * 0.1
    assert np.abs(th).max() > a * 0.9
    assert abs(th.mean()) < a * 0.1


def test_standard_normal_distribution():
    # StandardNormal (rand_distr's ziggurat): KS against the normal CDF, and the tails
    z = oracle.sample_moves(3, NORMAL, 1.0, 400_000, seed=7)
    assert stats.kstest(z, "norm").pvalue > 1e-3
    assert abs(z.mean()) < 5 / math.sqrt(len(z))
    assert abs(z.var() - 1.0) < 5 * math.sqrt(2.0 / len(z))
    # beyond the base layer's R = 3.654 the tail sampler runs: its share matches 2 (1 - Phi(R))
    tail = np.mean(np.abs(z) > 3.6541528853610088)
    want = 2 * stats.norm.sf(3.6541528853610088)
    assert abs(tail - want) < 6 * math.sqrt(want / len(z))


@pytest.mark.parametrize("dim", [2, 3])
def test_ball_sample_is_uniform_in_the_ball(dim):
    # Ball::sample (distribution.rs:41-69): |v| / d has CDF r^dim, directions are uniform
    d = 0.3
    v = oracle.sample_moves(dim, TRANSLATE, d, 200_000, seed=11)
    r = np.linalg.norm(v, axis=1) / d
    assert r.max() < 1.0
    assert stats.kstest(r ** dim, "uniform").pvalue > 1e-3
    unit = v / np.linalg.norm(v, axis=1)[:, None]
    if dim == 3:
        assert stats.kstest(unit[:, 2], "uniform", args=(-1, 2)).pvalue > 1e-3
    ang = np.arctan2(unit[:, 1], unit[:, 0])
    assert stats.kstest(ang, "uniform", args=(-math.pi, 2 * math.pi)).pvalue > 1e-3


def test_versor_rotation_vector_distribution():
    # Rotate<Versor> (rotate/versor.rs:40-71): the rotation vector s ~ N(0, sigma^2 I) redrawn
    # while |s| > pi; the rotation angle is 2 arc_distance = |s|: a Maxwell law of scale sigma
    # truncated at pi
    sigma = 0.8
    q = oracle.sample_moves(3, ROTATE, sigma, 200_000, seed=13)
    theta = 2.0 * arc_distance_from_identity(q)
    assert theta.max() <= math.pi
    cut = stats.maxwell.cdf(math.pi, scale=sigma)
    cdf = lambda x: stats.maxwell.cdf(np.minimum(x, math.pi), scale=sigma) / cut
    assert stats.kstest(theta, cdf).pvalue > 1e-3
    # the versors are unit up to rounding (the move composes without renormalising)
    assert np.abs(np.linalg.norm(q, axis=1) - 1.0).max() < 1e-15 * 8


def test_rotate_angle_is_uniform():
    a = 0.7
    th = oracle.sample_moves(2, ROTATE, a, 200_000, seed=17)
    assert stats.kstest(th, "uniform", args=(-a, 2 * a)).pvalue > 1e-3


def test_ziggurat_tables_follow_the_zignor_construction():
    # ZIGNOR (Doornik 2005, "An improved ziggurat method to generate normal random samples"):
    # 256 layers of equal area V under f(x) = exp(-x^2/2), base layer [0, R] plus the tail.
    # x[1] = R, x[i] = f^-1(V / x[i-1] + f(x[i-1])), x[0] = V / f(R), x[256] = 0, f[i] = f(x[i]).
    R, V = 3.6541528853610088, 0.00492867323399
    f = lambda t: math.exp(-0.5 * t * t)
    x = [0.0] * 257
    x[0] = V / f(R)
    x[1] = R
    for i in range(2, 256):
        x[i] = math.sqrt(-2.0 * math.log(V / x[i - 1] + f(x[i - 1])))
    fx = [f(t) for t in x]
    ox, of = oracle.ziggurat_tables()
    assert np.array_equal(ox, np.array(x)), np.flatnonzero(ox != np.array(x))[:5]
    assert np.array_equal(of, np.array(fx))
    # each layer's rectangle x[i] (f[i+1] - f[i]) has area V (to rounding), the top one
    # (f[256] = f(0) = 1) included, and the base layer R f(R) plus the tail integral too
    areas = np.array([x[i] * (fx[i + 1] - fx[i]) for i in range(1, 256)])
    assert np.abs(areas / V - 1.0).max() < 1e-6
    base = R * f(R) + math.sqrt(math.pi / 2.0) * math.erfc(R / math.sqrt(2.0))
    assert abs(base / V - 1.0) < 1e-9
    assert fx[256] == 1.0
