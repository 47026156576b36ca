"""The oracle's threaded ParallelSweep gives the same trajectory for every thread count.

The trials of one colour pass only read the pre-colour state (parallel_sweep.rs:209-279 runs
them under rayon), and the accepted moves are applied in space-list order, so hard-sphere and
Lennard-Jones trajectories must be identical bit for bit.
"""
import numpy as np
import pytest

import oracle
from hoomd_rs_b200 import lattice


@pytest.mark.parametrize("interaction", [oracle.HARD_SPHERE, oracle.LENNARD_JONES])
def test_thread_count_does_not_change_the_trajectory(interaction):
    if interaction == oracle.HARD_SPHERE:
        pos, L = lattice.hard_sphere_box(4000, 0.5, 3, 11)
        rng, d = 1.0, 0.2
    else:
        pos, L = lattice.lennard_jones_box(2048, 0.8, 3, 11)
        rng, d = 2.5, 0.1
    out = []
    for threads in (1, 3, 8):
        o = oracle.System(3, [L] * 3, pos, seed=21, interaction=interaction)
        counts = []
        for _ in range(3):
            counts.append(o.parallel_sweep(oracle.TRANSLATE, d, 1.0, rng, threads=threads))
            o.increment_step()
        out.append((counts, o.state()[0]))
    for counts, p in out[1:]:
        assert counts == out[0][0]
        assert np.array_equal(p, out[0][1])
