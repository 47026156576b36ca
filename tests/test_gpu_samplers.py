"""The device's trial-move samplers equal the oracle's bit for bit (hmc_sample_moves against
oracle.sample_moves, sample i from Counter(step, substep, seed).index(i)); the oracle's samplers
are pinned by the reference's statistical tests in tests/test_samplers_cpu.py, which are also run
here on the device's own samples."""
import math

import numpy as np
import pytest

import oracle
from hoomd_rs_b200 import Context

pytestmark = pytest.mark.gpu

TRANSLATE, ROTATE, NORMAL = 0, 1, 2


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


@pytest.mark.parametrize("dim,kind,maximum", [(3, TRANSLATE, 0.235), (2, TRANSLATE, 0.1), (3, ROTATE, 0.1),
                                              (3, ROTATE, 1.53), (2, ROTATE, 0.7), (3, NORMAL, 1.0)])
def test_device_samples_equal_the_oracle(ctx, dim, kind, maximum):
    n = 1_000_000
    got = ctx.sample_moves(dim, kind, maximum, n, step=12, substep=3, seed=0x5EED0002)
    want = oracle.sample_moves(dim, kind, maximum, n, step=12, substep=3, seed=0x5EED0002)
    assert np.array_equal(got, want), np.flatnonzero(np.any(np.atleast_2d(got.T).T != np.atleast_2d(want.T).T,
                                                            axis=-1))[:10]


@pytest.mark.parametrize("d", [0.1, 1.0])
def test_device_translate_reference_statistics(ctx, d):
    # translate/cartesian.rs:65-100 on the device's samples
    dv = ctx.sample_moves(3, TRANSLATE, d, 2048, seed=1)
    norm = np.linalg.norm(dv, axis=1)
    assert norm.max() <= d and norm.min() < d * 0.1 and norm.max() > d * 0.9
    assert np.all(np.abs(dv.mean(axis=0)) < d * 0.1)


@pytest.mark.parametrize("a", [0.1, 1.0, 1.53])
def test_device_rotate_versor_reference_statistics(ctx, a):
    # rotate/versor.rs:151-184 on the device's samples
    q = ctx.sample_moves(3, ROTATE, a, 65536, seed=1)
    arc = np.arctan2(np.linalg.norm(q[:, 1:], axis=1), q[:, 0])
    assert abs(abs(arc.mean()) - 0.75 * a) < 0.1 * a


@pytest.mark.parametrize("a", [0.1, 1.0])
def test_device_rotate_angle_reference_statistics(ctx, a):
    th = ctx.sample_moves(2, ROTATE, a, 1024, seed=1)
    assert np.abs(th).max() <= a and np.abs(th).min() < a * 0.1 and np.abs(th).max() > a * 0.9
    assert abs(th.mean()) < a * 0.1
    assert math.isfinite(float(th.sum()))
