"""Large systems: 2^27 hard spheres (512^3 simple-cubic sites, packing fraction 0.40), about 21 GB
of device arrays per system and every double4 array past 4 GB, so that slot and byte offsets
beyond 32 bits, grids of half a million blocks and 512^3 checkerboard spaces are exercised. The
oracle cannot follow at this size; the checks are the size-independent ones: the FP32 + recheck
trajectory equals the FP64 trajectory bit for bit (counts and positions), no pair overlaps
afterwards, and the sweep's trial count is rounds x non-empty spaces over the whole box."""
import math

import numpy as np
import pytest

from hoomd_rs_b200 import FP32_RECHECK, FP64, TRANSLATE, Context, HardSphere, Microstate, PairwiseCutoff, Periodic, lattice

pytestmark = pytest.mark.gpu

N = 1 << 27


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


def test_two_to_the_27_spheres_fp32_equals_fp64(ctx):
    import torch
    free, _ = torch.cuda.mem_get_info(0)
    if free < 60e9:
        pytest.skip(f"needs about 45 GB of device memory, {free / 1e9:.0f} GB free")
    spacing = (math.pi / 6.0 / 0.40) ** (1.0 / 3.0)  # 1.094: no pair closer than the diameter
    L = 512 * spacing
    pos = lattice.cubic_lattice(N, L, 3, 0, jitter=0.0)
    h = PairwiseCutoff(HardSphere(1.0))
    runs = {}
    for precision in (FP32_RECHECK, FP64):
        g = Microstate(ctx, Periodic(1.0, [L] * 3), pos, h, seed=0x5EED0070)
        counts = []
        for d in (0.15, 0.3):
            c = g.sweep(TRANSLATE, d, 1.0, precision, n_sweeps=1, increment_step=True)
            assert c.total() >= N  # full colour sets until at least N trials (parallel_sweep.rs:402)
            counts.append((c.accepted, c.rejected))
        runs[precision] = (counts, g.positions())
        if precision == FP64:
            assert g.overlap_count() == 0
        g.close()
    assert runs[FP32_RECHECK][0] == runs[FP64][0]
    assert np.array_equal(runs[FP32_RECHECK][1], runs[FP64][1])
    # the bodies moved and stayed in the box
    moved = np.any(runs[FP64][1] != pos, axis=1)
    assert moved.mean() > 0.3
    assert np.all(np.abs(runs[FP64][1]) <= L / 2.0)


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
@pytest.mark.parametrize("dim,shape", [(2, 2100), (3, 166)])
def test_space_count_scan_of_many_blocks_matches_oracle(ctx, dim, shape, precision):
    # more than 2048 blocks of 2048 spaces: the space counts are scanned in three kernels (the
    # block totals by k_scan_block_sums); 2^19 bodies in a dilute box of shape^dim spaces, two
    # sweeps against the oracle's ParallelSweep bit for bit
    import os

    import oracle
    assert shape ** dim > 2048 * 2048
    n = 1 << 19
    L = float(shape) + 0.5  # spaces of width L / shape >= 1
    phi = n * (math.pi / 4.0 if dim == 2 else math.pi / 6.0) / L ** dim
    pos, L2 = lattice.hard_sphere_box(n, phi, dim, 0x5EED0071)
    assert abs(L2 - L) < 1e-9 * L
    g = Microstate(ctx, Periodic(1.0, [L] * dim), pos, PairwiseCutoff(HardSphere(1.0)), seed=0x5EED0071)
    o = oracle.System(dim, [L] * dim, pos, seed=0x5EED0071)
    threads = max(1, os.cpu_count() or 1)
    for d in (0.5, 1.5):
        c = g.sweep(TRANSLATE, d, 1.0, precision, n_sweeps=1, increment_step=True)
        a, r = o.parallel_sweep(oracle.TRANSLATE, d, 1.0, 1.0, threads=threads)
        o.increment_step()
        assert (c.accepted, c.rejected) == (a, r)
    assert np.array_equal(g.positions(), o.state()[0])
