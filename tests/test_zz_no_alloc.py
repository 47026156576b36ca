"""hmc_overlap_count_noalloc: the overlap count into caller-owned device buffers.

Some callers cannot call cudaMalloc when they want this check (all their device memory
comes from a pool they reserved up front, or they may not grow the process's device
footprint after start-up). This entry point keeps its cell list in a fixed device array
inside the library and writes only to the caller's buffers. These tests compare it with
hmc_overlap_check, which builds a full system, on two calls in a row, so the second call
also shows that state left in the shared array by the first one does not leak into its
result. The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import hoomd_rs_b200 as hm
from hoomd_rs_b200 import Context, HardSphere, Microstate, PairwiseCutoff, Periodic

pytestmark = pytest.mark.gpu


def _random_system(ctx, dim, n, L, seed, boundary_range=1.0):
    rng = np.random.default_rng(seed)
    Ls = np.broadcast_to(np.asarray(L, dtype=np.float64), (dim,))
    pos = (rng.random((n, dim)) - 0.5) * Ls
    return Microstate(ctx, Periodic(boundary_range, list(Ls)), pos, PairwiseCutoff(HardSphere(1.0)))


def _noalloc_count(torch, lib, positions, L, diameter=1.0, boundary_range=1.0):
    dim = positions.shape[1]
    d_pos = torch.from_numpy(np.ascontiguousarray(positions)).to("cuda")
    d_out = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    Lh = np.ascontiguousarray(L, dtype=np.float64)
    stream = torch.cuda.current_stream().cuda_stream
    st = lib.hmc_overlap_count_noalloc(C.c_void_p(d_pos.data_ptr()), positions.shape[0], dim,
                                       Lh.ctypes.data_as(C.POINTER(C.c_double)), diameter, boundary_range,
                                       C.c_void_p(d_out.data_ptr()), C.c_void_p(stream))
    torch.cuda.synchronize()
    return st, int(d_out.item())


@pytest.mark.parametrize("dim,n,L", [(3, 5000, 14.0), (2, 3000, 50.0)])
def test_noalloc_matches_overlap_check_twice(dim, n, L):
    torch = pytest.importorskip("torch")
    lib = hm.load_library()
    ctx = Context(0)
    for call, seed in enumerate((11, 12)):
        sysm = _random_system(ctx, dim, n, L, seed + 10 * dim)
        want = sysm.overlap_count()  # the existing entry point
        assert want > 0
        st, got = _noalloc_count(torch, lib, sysm.positions(), [L] * dim)
        assert st == hm.OK, call
        assert got == want, (call, got, want)
        sysm.close()


@pytest.mark.parametrize("dim,n,L,boundary_range", [
    (3, 40, [2.5, 2.6, 2.7], 1.0),   # fewer than 3 cells on every axis: each neighbour cell once
    (2, 30, [2.2, 9.0], 1.0),        # two cells on one axis
    (3, 65536, 200.0, 1.0),          # 200^3 cells exceed the fixed 65,536: the cells are widened
    (3, 3000, 12.0, 1.6),            # a boundary range wider than the diameter (ghost rule)
])
def test_noalloc_geometries_match_overlap_check(dim, n, L, boundary_range):
    torch = pytest.importorskip("torch")
    lib = hm.load_library()
    ctx = Context(0)
    sysm = _random_system(ctx, dim, n, L, 7, boundary_range)
    want = sysm.overlap_count()
    assert want > 0
    Ls = list(np.broadcast_to(np.asarray(L, dtype=np.float64), (dim,)))
    for call in range(2):
        st, got = _noalloc_count(torch, lib, sysm.positions(), Ls, boundary_range=boundary_range)
        assert st == hm.OK, call
        assert got == want, (call, got, want)
    sysm.close()


def test_noalloc_empty_input_and_no_device_memory_growth():
    # n_bodies = 0 gives 0 (the output is still written); after that first call has set the
    # library up on the device, further calls leave the device's free memory unchanged.
    torch = pytest.importorskip("torch")
    lib = hm.load_library()
    ctx = Context(0)
    st, got = _noalloc_count(torch, lib, np.zeros((0, 3)), [10.0, 10.0, 10.0])
    assert (st, got) == (hm.OK, 0)
    sysm = _random_system(ctx, 3, 20000, 30.0, 5)
    pos = sysm.positions()
    want = sysm.overlap_count()
    d_pos = torch.from_numpy(np.ascontiguousarray(pos)).to("cuda")
    d_out = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    Lh = np.array([30.0, 30.0, 30.0])
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for call in range(2):
        st = lib.hmc_overlap_count_noalloc(C.c_void_p(d_pos.data_ptr()), len(pos), 3,
                                           Lh.ctypes.data_as(C.POINTER(C.c_double)), 1.0, 1.0,
                                           C.c_void_p(d_out.data_ptr()), None)
        assert st == hm.OK
        torch.cuda.synchronize()
        assert int(d_out.item()) == want, call
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    sysm.close()


def test_noalloc_rejects_more_bodies_than_its_scratch_holds():
    torch = pytest.importorskip("torch")
    lib = hm.load_library()
    n = 65536 + 1
    d_pos = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    d_out = torch.zeros(1, dtype=torch.int64, device="cuda")
    Lh = np.array([100.0, 100.0, 100.0])
    st = lib.hmc_overlap_count_noalloc(C.c_void_p(d_pos.data_ptr()), n, 3, Lh.ctypes.data_as(C.POINTER(C.c_double)),
                                       1.0, 1.0, C.c_void_p(d_out.data_ptr()), None)
    assert st == hm.INVALID_ARGUMENT
