"""The oracle's univariate energies for Isotropic (hoomd-interaction/src/univariate/) against the
reference's own tests of them, with their tolerances: weeks_chandler_anderson.rs
special_points_12_6, harmonic.rs zero_energy_point / general_case, harmonic_repulsion.rs
outside_rcut / general_case, boxcar.rs general_case, xplor.rs special_points_12_6 and
lennard_jones_gauss.rs select_points_first_set / select_points_second_set; and
Isotropic's cut-off (isotropic.rs:147-156) through two-body systems."""
import math

import numpy as np
import pytest

import oracle

EPS = 2.220446049250313e-16  # f64::EPSILON, the default tolerance of the approx assertions


def rel_eq(a, b, rel=EPS):
    # approxim's assert_relative_eq with its defaults (epsilon = max_relative = f64::EPSILON)
    return a == b or abs(a - b) <= EPS or abs(a - b) <= rel * max(abs(a), abs(b))


def e(kind, params, r, wrap=oracle.UVW_NONE, wrap_params=()):
    return oracle.univariate_energy(kind, params, r, wrap, wrap_params)


@pytest.mark.parametrize("eps", [1.0, 2.0, 12.125, 0.25])
@pytest.mark.parametrize("sigma", [1.0, 2.0, 0.5])
def test_wca_special_points(eps, sigma):
    wca = oracle.UV_WEEKS_CHANDLER_ANDERSON
    assert rel_eq(e(wca, [eps, sigma], sigma), eps)  # the zero crossing, shifted by epsilon
    assert abs(e(wca, [eps, sigma], 2.0 ** (1.0 / 6.0) * sigma) - 0.0) <= EPS  # the bottom of the well
    assert e(wca, [eps, sigma], 2.0 * sigma) == 0.0


@pytest.mark.parametrize("k", [1.0, 2.0, 5.0, 10.0])
@pytest.mark.parametrize("r_0", [0.0, 1.0, 2.0])
def test_harmonic(k, r_0):
    assert e(oracle.UV_HARMONIC, [k, r_0], r_0) == 0.0
    r = 5.0
    assert rel_eq(e(oracle.UV_HARMONIC, [k, r_0], r), 0.5 * k * (r - r_0) * (r - r_0))


@pytest.mark.parametrize("a", [1.0, 2.0, 5.0, 10.0])
@pytest.mark.parametrize("r_cut", [1.0, 2.0, 3.0])
def test_harmonic_repulsion(a, r_cut):
    assert e(oracle.UV_HARMONIC_REPULSION, [a, r_cut], r_cut + 1.0) == 0.0
    r = 0.5
    want = a * (r_cut - r) - 0.5 * a / r_cut * (r_cut * r_cut - r * r)
    assert math.isclose(e(oracle.UV_HARMONIC_REPULSION, [a, r_cut], r), want, rel_tol=1e-15, abs_tol=EPS)


@pytest.mark.parametrize("eps", [1.0, -2.0, 12.125, 0.25])
@pytest.mark.parametrize("left", [1.0, 2.0, 0.5])
@pytest.mark.parametrize("w", [0.5, 0.125])
def test_boxcar(eps, left, w):
    right = left + w
    box = lambda r: e(oracle.UV_BOXCAR, [eps, left, right], r)
    assert box(0.0) == 0.0
    assert box(np.nextafter(left, -np.inf)) == 0.0
    assert box(left) == eps
    assert box(np.nextafter(left, np.inf)) == eps
    assert box(left + w / 2.0) == eps
    assert box(np.nextafter(right, -np.inf)) == eps
    assert box(right) == 0.0
    assert box(right * 10.0) == 0.0


@pytest.mark.parametrize("eps", [1.0, 2.0, 12.125, 0.25])
@pytest.mark.parametrize("sigma", [1.0, 2.0, 0.5])
def test_xplor_lj_special_points(eps, sigma):
    lj = oracle.UV_LENNARD_JONES
    r_smooth, r_cut = 1.0, 2.5 * sigma
    x = lambda r: e(lj, [eps, sigma], r, oracle.UVW_XPLOR, [r_cut, r_smooth])
    f = lambda r: e(lj, [eps, sigma], r)
    # not smoothed below r_smooth
    assert abs(x(r_smooth / 2.0) - f(r_smooth / 2.0)) <= EPS
    assert abs(x(np.nextafter(r_smooth, -np.inf)) - f(np.nextafter(r_smooth, -np.inf))) <= EPS
    if sigma < r_smooth:
        assert abs(x(sigma)) <= EPS
    # zero at and above r_cut
    for r in (r_cut, np.nextafter(r_cut, np.inf), 2.0 * r_cut):
        assert abs(x(r)) <= EPS
    # smoothed between
    mid = 0.5 * (r_smooth + r_cut)
    assert abs(x(mid) - f(mid)) > EPS


def test_shifted_and_expanded():
    # Shifted: F(r) - F(r_shift); Expanded: F(r - delta)
    wca, h = oracle.UV_WEEKS_CHANDLER_ANDERSON, oracle.UV_HARMONIC
    assert e(h, [2.0, 1.0], 1.7, oracle.UVW_SHIFTED, [2.0]) == e(h, [2.0, 1.0], 1.7) - e(h, [2.0, 1.0], 2.0)
    assert e(wca, [1.0, 1.0], 1.9, oracle.UVW_EXPANDED, [1.0]) == e(wca, [1.0, 1.0], 0.9)


def test_isotropic_cut_off_and_sum():
    # Isotropic: 0 at r^2 >= r_cut^2, else F(sqrt(r^2)); the total energy sums the pairs once
    iso = {"kind": oracle.UV_HARMONIC_REPULSION, "params": [3.0, 1.5], "r_cut": 1.5}
    pos = [[0.0, 0.0], [1.2, 0.0], [0.0, 1.5], [4.0, 4.0]]
    o = oracle.System(2, [10.0, 10.0], pos, interaction=oracle.ISOTROPIC, isotropic=iso)
    want = e(oracle.UV_HARMONIC_REPULSION, [3.0, 1.5], 1.2) + e(oracle.UV_HARMONIC_REPULSION, [3.0, 1.5],
                                                                 math.sqrt(1.2 ** 2 + 1.5 ** 2))
    assert o.total_energy() == pytest.approx(want, rel=1e-15)
    # the pair at exactly r_cut contributes nothing
    assert e(oracle.UV_HARMONIC_REPULSION, [3.0, 1.5], 1.5) == 0.0


@pytest.mark.parametrize("params,r,want", [([2.0, 0.5, 3.0, 1.0], 1.5, -0.378_674_092_892_274),
                                           ([2.0, 0.5, 3.0, 1.0], 3.2, -1.923_440_656_092_139),
                                           ([10.0, 0.1, 5.0, 1.0], 1.5, -0.167_875_643_768_546),
                                           ([10.0, 0.1, 5.0, 1.0], 3.2, -0.001_862_699_147_576_425)])
def test_lennard_jones_gauss_select_points(params, r, want):
    # lennard_jones_gauss.rs: assert_relative_eq!(energy, want, epsilon = 1e-12)
    got = e(oracle.UV_LENNARD_JONES_GAUSS, params, r)
    assert abs(got - want) <= 1e-12 or abs(got - want) <= EPS * max(abs(got), abs(want))
