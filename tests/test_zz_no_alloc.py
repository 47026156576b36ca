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


def _random_system(ctx, dim, n, L, seed):
    rng = np.random.default_rng(seed)
    pos = (rng.random((n, dim)) - 0.5) * L
    return Microstate(ctx, Periodic(1.0, [L] * dim), pos, PairwiseCutoff(HardSphere(1.0)))


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
