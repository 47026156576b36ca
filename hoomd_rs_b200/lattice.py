"""Seeded synthetic initial configurations for the sweep workloads.

The reference's benchmarks build their states with QuickInsert/QuickCompress
(benchmarks/src/place.rs); these workloads start instead from lattices with a small
seeded jitter so that every run is reproducible from (N, packing fraction, seed):

* square (2-D) and simple-cubic (3-D) lattices with ceil(N^(1/d)) sites per side;
* FCC with m = ceil((N/4)^(1/3)) cells per side and the first N sites in (i, j, k, basis)
  order;
* each coordinate gets U[-jitter, jitter) drawn from hoomd-rand's counter stream
  Counter(0, 0, seed).index(i) (SFC64, hoomd-rand/src/counter.rs:160-167), one uniform per
  coordinate in axis order.
"""
from __future__ import annotations

import math

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _sfc64_streams(step: int, substep: int, seed: int, index: np.ndarray):
    """Vectorised SFC64 states after Counter::make_rng (12 discarded outputs)."""
    n = index.shape[0]
    s0 = np.full(n, np.uint64(step), dtype=np.uint64)
    s1 = np.full(n, np.uint64((substep << 32) | seed), dtype=np.uint64)
    s2 = index.astype(np.uint64).copy()
    ctr = np.zeros(n, dtype=np.uint64)
    st = [s0, s1, s2, ctr]
    for _ in range(12):
        _sfc64_next(st)
    return st


def _sfc64_next(st):
    s0, s1, s2, ctr = st
    with np.errstate(over="ignore"):
        out = s0 + s1 + ctr
        n0 = s1 ^ (s1 >> np.uint64(11))
        n1 = s2 + (s2 << np.uint64(3))
        n2 = ((s2 << np.uint64(24)) | (s2 >> np.uint64(40))) + out
        st[0], st[1], st[2], st[3] = n0, n1, n2, ctr + np.uint64(1)
    return out


def counter_uniforms(seed: int, n: int, per_index: int) -> np.ndarray:
    """U[0,1) values: row i holds the first `per_index` draws of Counter(0,0,seed).index(i)."""
    st = _sfc64_streams(0, 0, seed, np.arange(n, dtype=np.uint64))
    out = np.empty((n, per_index))
    for k in range(per_index):
        out[:, k] = (_sfc64_next(st) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return out


def _jitter(pos: np.ndarray, seed: int, jitter: float) -> np.ndarray:
    if jitter <= 0:
        return pos
    u = counter_uniforms(seed, pos.shape[0], pos.shape[1])
    return pos + (u * 2.0 - 1.0) * jitter


def box_length(n: int, number_density: float, dim: int) -> float:
    return (n / number_density) ** (1.0 / dim)


def sphere_number_density(packing_fraction: float, dim: int, diameter: float = 1.0) -> float:
    v = math.pi / 4.0 * diameter ** 2 if dim == 2 else math.pi / 6.0 * diameter ** 3
    return packing_fraction / v


def cubic_lattice(n: int, L: float, dim: int, seed: int, jitter: float = 0.01) -> np.ndarray:
    """Square (2-D) or simple-cubic (3-D) lattice in [-L/2, L/2)^dim."""
    m = int(math.ceil(n ** (1.0 / dim) - 1e-9))
    a = L / m
    idx = np.indices([m] * dim).reshape(dim, -1).T[:n].astype(np.float64)
    pos = -L / 2.0 + (idx + 0.5) * a
    return _jitter(pos, seed, jitter)


def fcc_lattice(n: int, L: float, seed: int, jitter: float = 0.01) -> np.ndarray:
    """FCC lattice with m = ceil((n/4)^(1/3)) cells per side, first n sites."""
    m = int(math.ceil((n / 4.0) ** (1.0 / 3.0) - 1e-9))
    a = L / m
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    cells = np.indices([m, m, m]).reshape(3, -1).T.astype(np.float64)
    pos = (cells[:, None, :] + basis[None, :, :]).reshape(-1, 3)[:n]
    pos = -L / 2.0 + (pos + 0.25) * a
    return _jitter(pos, seed, jitter)


def hard_sphere_box(n: int, packing_fraction: float, dim: int, seed: int, lattice: str = "auto",
                    jitter: float = 0.01):
    """(positions, L) for hard disks/spheres of diameter 1 at the given packing fraction."""
    rho = sphere_number_density(packing_fraction, dim)
    L = box_length(n, rho, dim)
    if dim == 3 and lattice in ("auto", "fcc"):
        return fcc_lattice(n, L, seed, jitter), L
    return cubic_lattice(n, L, dim, seed, jitter), L


def lennard_jones_box(n: int, number_density: float, dim: int, seed: int, jitter: float = 0.01):
    """(positions, L) for Lennard-Jones sites (sigma = 1) at the given number density."""
    L = box_length(n, number_density, dim)
    if dim == 3:
        return fcc_lattice(n, L, seed, jitter), L
    return cubic_lattice(n, L, dim, seed, jitter), L
