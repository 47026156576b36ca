"""GPU parity of the other built-in isotropic potentials: PairwiseCutoff(Isotropic { W(F), r_cut })
with F one of WeeksChandlerAnderson, Harmonic, HarmonicRepulsion, Boxcar, LennardJones,
OverlapPenalty and W none, Shifted, Expanded or Xplor (HMC_ISOTROPIC). They run through the
warp-per-trial energy pass of the Lennard-Jones kernels in FP64 (both precision modes), the serial
Sweep, the tuner and the total energy. Pair energies equal the oracle's bit for bit; sums are
formed in another order, so decisions may differ only inside the order bound, which is counted
(Count.order_ambiguous) and is zero in these runs."""
import math

import numpy as np
import pytest

import oracle
from hoomd_rs_b200 import (FP32_RECHECK, FP64, TRANSLATE, Boxcar, Context, Expanded, Harmonic, HarmonicRepulsion,
                           Isotropic, LennardJones, LennardJonesGauss, Microstate, OverlapPenalty, PairwiseCutoff,
                           Periodic, Shifted, WeeksChandlerAnderson, Xplor, lattice)

pytestmark = pytest.mark.gpu

C6 = 2.0 ** (1.0 / 6.0)


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


# (name, device interaction, oracle description, r_cut)
CASES = {
    "wca": (WeeksChandlerAnderson(1.0, 1.0), {"kind": oracle.UV_WEEKS_CHANDLER_ANDERSON, "params": [1.0, 1.0]}, C6),
    "shifted_wca": (Shifted(WeeksChandlerAnderson(1.5, 1.0), 1.0),
                    {"kind": oracle.UV_WEEKS_CHANDLER_ANDERSON, "params": [1.5, 1.0], "wrap": oracle.UVW_SHIFTED,
                     "wrap_params": [1.0]}, 1.2),
    "harmonic_repulsion": (HarmonicRepulsion(20.0, 1.0),
                           {"kind": oracle.UV_HARMONIC_REPULSION, "params": [20.0, 1.0]}, 1.0),
    "xplor_lj": (Xplor(LennardJones(1.0, 1.0), 2.5, 2.0),
                 {"kind": oracle.UV_LENNARD_JONES, "params": [1.0, 1.0], "wrap": oracle.UVW_XPLOR,
                  "wrap_params": [2.5, 2.0]}, 2.5),
    "boxcar": (Boxcar(-0.5, 1.0, 1.4), {"kind": oracle.UV_BOXCAR, "params": [-0.5, 1.0, 1.4]}, 1.5),
    "expanded_harmonic": (Expanded(0.2, Harmonic(5.0, 1.0)),
                          {"kind": oracle.UV_HARMONIC, "params": [5.0, 1.0], "wrap": oracle.UVW_EXPANDED,
                           "wrap_params": [0.2]}, 1.5),
    "penalty": (OverlapPenalty(100.0, 0.3, 2.0), {"kind": oracle.UV_OVERLAP_PENALTY, "params": [100.0, 0.3, 2.0]},
                1.0),
    "lj_gauss": (Shifted(LennardJonesGauss(1.5, 0.02, 1.5, 1.0), 2.0),
                 {"kind": oracle.UV_LENNARD_JONES_GAUSS, "params": [1.5, 0.02, 1.5, 1.0], "wrap": oracle.UVW_SHIFTED,
                  "wrap_params": [2.0]}, 2.0),
}
# the potentials whose pair energy uses exp: the device's, within a few ulp of the platform's
EXP = {"lj_gauss"}


def systems(ctx, name, dim, pos, L, seed):
    e, iso, r_cut = CASES[name]
    g = Microstate(ctx, Periodic(r_cut, [L] * dim), pos, PairwiseCutoff(Isotropic(e, r_cut)), seed=seed)
    o = oracle.System(dim, [L] * dim, pos, seed=seed, interaction=oracle.ISOTROPIC, isotropic=dict(iso, r_cut=r_cut))
    return g, o


def start(dim, n, rho, seed):
    pos, L = lattice.lennard_jones_box(n, rho, dim, seed)
    return pos, L


@pytest.mark.parametrize("name", list(CASES))
def test_pair_energies_equal_the_oracle(ctx, name):
    # two-body systems over distances that cross every branch: the total energy is one pair
    e, iso, r_cut = CASES[name]
    for r in np.concatenate([np.linspace(0.05, r_cut * 1.05, 97), [1.0, C6, r_cut, np.nextafter(r_cut, 0.0)]]):
        pos = [[0.0, 0.0, 0.0], [float(r), 0.0, 0.0]]
        g, o = systems(ctx, name, 3, pos, 10.0, 1)
        got, want = g.total_energy(), o.total_energy()
        if name in EXP:
            assert math.isclose(got, want, rel_tol=1e-14, abs_tol=1e-14 * 1.5), (name, r, got, want)
        else:
            assert got == want or (math.isnan(got) and math.isnan(want)), (name, r, got, want)
        g.close()


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
@pytest.mark.parametrize("name,dim,n,rho,kt,d", [("wca", 3, 1000, 0.7, 1.0, 0.12), ("shifted_wca", 2, 900, 0.6, 1.0, 0.15),
                                                  ("harmonic_repulsion", 2, 800, 0.9, 0.5, 0.15),
                                                  ("xplor_lj", 3, 1372, 0.8, 1.0, 0.1),
                                                  ("boxcar", 3, 800, 0.5, 1.0, 0.2),
                                                  ("lj_gauss", 3, 1000, 0.7, 1.0, 0.1),
                                                  ("expanded_harmonic", 3, 600, 0.3, 1.0, 0.2)])
def test_trajectory_matches_oracle(ctx, name, dim, n, rho, kt, d, precision):
    pos, L = start(dim, n, rho, 0x5EED0051)
    g, o = systems(ctx, name, dim, pos, L, 0x5EED0051)
    r_cut = CASES[name][2]
    for _ in range(6):
        c = g.sweep(TRANSLATE, d, kt, precision, n_sweeps=1, increment_step=True)
        a, r = o.parallel_sweep(oracle.TRANSLATE, d, kt, r_cut)
        o.increment_step()
        assert c.order_ambiguous == 0
        assert (c.accepted, c.rejected) == (a, r)
    assert np.array_equal(g.positions(), o.state()[0])
    assert math.isclose(g.total_energy(), o.total_energy(), rel_tol=1e-11, abs_tol=1e-9)


@pytest.mark.parametrize("name", ["wca", "harmonic_repulsion"])
def test_serial_sweep_matches_oracle(ctx, name):
    pos, L = start(2, 400, 0.6, 0x5EED0052)
    g, o = systems(ctx, name, 2, pos, L, 0x5EED0052)
    for _ in range(4):
        c = g.serial_sweep(0.15, increment_step=True)
        a, r = o.serial_sweep(oracle.TRANSLATE, 0.15, 1.0)
        o.increment_step()
        assert (c.accepted, c.rejected) == (a, r)
    assert np.array_equal(g.positions(), o.state()[0])


def test_tune_matches_oracle(ctx):
    pos, L = start(3, 500, 0.7, 0x5EED0053)
    g, o = systems(ctx, "wca", 3, pos, L, 0x5EED0053)
    got = g.tune(TRANSLATE, 0.1, 1.0, FP64, 0.3, samples=200, steps=8)
    want = o.tune_stream(oracle.TRANSLATE, 0.1, 1.0, 0.3, 200, 8)
    assert got == want
