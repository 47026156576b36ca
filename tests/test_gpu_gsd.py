"""GSD frames written from device state (hmc_gsd_append_system) against the oracle.

AppendMicrostate::append_microstate (hoomd-microstate/src/append.rs:115-129) writes the
step, the FP32 site positions and orientations in tag order, the dimensions and the box.
The library converts the GPU-resident state on the device; the oracle restates the site
transform and the FP32 conversion on the host (oracle_gsd_frame) and the file layer in
Python (oracle/gsd_oracle.py). Frames must agree bit for bit and whole files byte for byte.
"""
import math

import numpy as np
import pytest

import oracle
from oracle import gsd_oracle as O
from hoomd_rs_b200 import (FP32_RECHECK, FP64, ROTATE, TRANSLATE, Context, ConvexPolygon, ConvexPolyhedron,
                           HardShape, HardSphere, Isotropic, LennardJones, Microstate, PairwiseCutoff, Periodic,
                           Shifted, lattice)
from hoomd_rs_b200.gsd import GsdFile, HoomdGsdFile

pytestmark = pytest.mark.gpu

CUBE = np.array([[x, y, z] for x in (-0.5, 0.5) for y in (-0.5, 0.5) for z in (-0.5, 0.5)])
SQUARE = np.array([[-0.5, -0.5], [0.5, -0.5], [0.5, 0.5], [-0.5, 0.5]])


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


def _frame_arrays(path, frame=0):
    r = GsdFile.open(path)
    pos = r.iter_arrays(frame, "particles/position", np.float32, 3)
    ori = (r.iter_arrays(frame, "particles/orientation", np.float32, 4)
           if r.find_chunk(frame, "particles/orientation") else None)
    return r, pos, ori


def _bits(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def test_point_periodic_rectangle_2d(ctx, tmp_path):
    # append.rs:300-338: two points in a periodic 12 x 18 rectangle at step 1234
    m = Microstate(ctx, Periodic(1.0, [12.0, 18.0]), [[1.0, 0.0], [-1.0, 2.0]], PairwiseCutoff(HardSphere(1.0)),
                   step=1234)
    path = tmp_path / "test.gsd"
    f = HoomdGsdFile.create(path)
    f.append_microstate(m).end()
    f.close()
    r = GsdFile.open(path)
    assert r.n_frames() == 1
    assert list(r.iter_scalars(0, "configuration/step", np.uint64)) == [1234]
    assert r.iter_arrays(0, "particles/position", np.float32, 3).tolist() == [[1.0, 0.0, 0.0], [-1.0, 2.0, 0.0]]
    assert list(r.iter_scalars(0, "configuration/dimensions", np.uint8)) == [2]
    assert list(r.iter_scalars(0, "configuration/box", np.float32)) == [12.0, 18.0, 0.0, 0.0, 0.0, 0.0]
    assert list(r.iter_scalars(0, "particles/N", np.uint32)) == [2]
    assert r.find_chunk(0, "particles/orientation") is None


def _run_pair(g, o, moves, precision, body_range):
    for move, maximum in moves:
        g.sweep(move, maximum, 1.0, precision, n_sweeps=1, increment_step=True)
        o.parallel_sweep(oracle.TRANSLATE if move == TRANSLATE else oracle.ROTATE, maximum, 1.0, body_range)
        o.increment_step()


def _check_file(tmp_path, g, o, dim, L, frames):
    """Write `frames` frames from both sides (a sweep between frames) and compare bytes."""
    path = tmp_path / "traj.gsd"
    f = HoomdGsdFile.create(path, "hoomd-rs-b200")
    w = O.Writer("hoomd-rs-b200", "hoomd", (1, 4))
    for k, (moves, precision, body_range) in enumerate(frames):
        _run_pair(g, o, moves, precision, body_range)
        f.append_microstate(g).log_scalar("frame", k, np.uint32).end()
        pos, ori = o.gsd_frame()
        w.append_microstate(o.state()[2], dim, L, pos, ori)
        w.write_scalars("log/frame", [k], O.U32)
        w.end_frame()
    f.close()
    image = w.close()
    assert path.read_bytes() == image
    r, pos_last, ori_last = _frame_arrays(path, len(frames) - 1)
    pos, ori = o.gsd_frame()
    assert np.array_equal(_bits(pos_last), _bits(pos))
    assert (ori is None and ori_last is None) or np.array_equal(_bits(ori_last), _bits(ori))
    return path


@pytest.mark.parametrize("precision", [FP64, FP32_RECHECK])
def test_spheres_3d_frames(ctx, tmp_path, precision):
    n, phi = 4000, 0.50
    L = (n / (phi * math.pi / 6.0)) ** (1.0 / 3.0)
    pos = lattice.fcc_lattice(n, L, seed=11, jitter=0.01)
    g = Microstate(ctx, Periodic(1.0, [L] * 3), pos, PairwiseCutoff(HardSphere(1.0)), seed=11)
    o = oracle.System(3, [L] * 3, pos, seed=11)
    frames = [([(TRANSLATE, 0.15)] * 2, precision, 1.0) for _ in range(4)]
    _check_file(tmp_path, g, o, 3, [L] * 3, frames)


def test_disks_2d_frames(ctx, tmp_path):
    n, phi = 4096, 0.70
    L = math.sqrt(n / (phi * math.pi / 4.0))
    pos = lattice.cubic_lattice(n, L, 2, seed=12, jitter=0.01)
    g = Microstate(ctx, Periodic(1.0, [L, L]), pos, PairwiseCutoff(HardSphere(1.0)), seed=12)
    o = oracle.System(2, [L, L], pos, seed=12)
    _check_file(tmp_path, g, o, 2, [L, L], [([(TRANSLATE, 0.1)] * 3, FP64, 1.0) for _ in range(3)])


def test_cubes_frames_with_signed_zero_versors(ctx, tmp_path):
    n, phi = 1728, 0.45
    L = (n / phi) ** (1.0 / 3.0)
    pos = lattice.cubic_lattice(n, L, 3, seed=13, jitter=0.01)
    rng = np.random.default_rng(13)
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    # signed zeros: the site versor combine(q, identity) turns -0 + 0 into +0 in some places
    q[0] = [1.0, -0.0, 0.0, -0.0]
    q[1] = [-0.0, 1.0, -0.0, 0.0]
    q[2] = [0.0, -0.0, -1.0, -0.0]
    q[3] = [-1.0, -0.0, -0.0, -0.0]
    g = Microstate(ctx, Periodic(math.sqrt(3.0), [L] * 3), pos, PairwiseCutoff(HardShape(
        ConvexPolyhedron.with_vertices(CUBE))), seed=13, orientations=q)
    o = oracle.System(3, [L] * 3, pos, q, seed=13, interaction=oracle.HARD_CONVEX_POLYHEDRON, vertices=CUBE)
    frames = [([], FP64, math.sqrt(3.0)),
              ([(TRANSLATE, 0.08), (ROTATE, 0.1)], FP64, math.sqrt(3.0)),
              ([(TRANSLATE, 0.08), (ROTATE, 0.1)], FP32_RECHECK, math.sqrt(3.0))]
    path = _check_file(tmp_path, g, o, 3, [L] * 3, frames)
    r = GsdFile.open(path)
    ori0 = r.iter_arrays(0, "particles/orientation", np.float32, 4)
    # combine(q, identity): scalar q.s; vector (0 q.s + v) + (v x 0). For q = (-1, -0, -0, -0):
    # 0 (-1) + (-0) = -0, and v x 0 has components (-0)0 - (-0)0 = +0, so the vector is +0.
    assert _bits(ori0[0]).tolist() == _bits(np.array([1.0, 0.0, 0.0, 0.0], np.float32)).tolist()
    assert _bits(ori0[3]).tolist() == _bits(np.array([-1.0, 0.0, 0.0, 0.0], np.float32)).tolist()


def test_polygons_2d_frames(ctx, tmp_path):
    n = 900
    shape = ConvexPolygon.with_vertices(SQUARE)
    R = shape.bounding_radius
    m = int(math.ceil(math.sqrt(n)))
    L = m * 1.05 * 2 * R
    pos = lattice.cubic_lattice(n, L, 2, 14, jitter=0.0)
    angles = np.random.default_rng(14).uniform(-math.pi, math.pi, n)
    angles[:4] = [-0.0, 0.0, 1.0e5, -3.0e5]
    g = Microstate(ctx, Periodic(2 * R, [L, L]), pos, PairwiseCutoff(HardShape(shape)), seed=14, orientations=angles)
    o = oracle.System(2, [L, L], pos, angles, seed=14, interaction=oracle.HARD_CONVEX_POLYGON,
                      vertices=shape.vertices)
    frames = [([], FP64, 2 * R), ([(TRANSLATE, 0.1), (ROTATE, 0.2)] * 2, FP64, 2 * R)]
    _check_file(tmp_path, g, o, 2, [L, L], frames)


def test_lennard_jones_frames(ctx, tmp_path):
    n, rho = 4000, 0.8
    L = (n / rho) ** (1.0 / 3.0)
    pos = lattice.fcc_lattice(n, L, seed=15, jitter=0.01)
    h = PairwiseCutoff(Isotropic(Shifted(LennardJones(epsilon=1.0, sigma=1.0), 2.5), 2.5))
    g = Microstate(ctx, Periodic(2.5, [L] * 3), pos, h, seed=15)
    o = oracle.System(3, [L] * 3, pos, seed=15, interaction=oracle.LENNARD_JONES)
    _check_file(tmp_path, g, o, 3, [L] * 3, [([(TRANSLATE, 0.1)] * 2, FP32_RECHECK, 2.5) for _ in range(2)])


def test_large_frame_round_trip(ctx, tmp_path):
    # a 2^18-sphere frame passes the 1 MiB write buffer: written straight from pinned memory
    n, phi = 1 << 18, 0.5
    L = (n / (phi * math.pi / 6.0)) ** (1.0 / 3.0)
    pos = lattice.fcc_lattice(n, L, seed=16, jitter=0.01)
    g = Microstate(ctx, Periodic(1.0, [L] * 3), pos, PairwiseCutoff(HardSphere(1.0)), seed=16)
    g.sweep(TRANSLATE, 0.1, 1.0, FP32_RECHECK, n_sweeps=2, increment_step=True)
    path = tmp_path / "big.gsd"
    f = HoomdGsdFile.create(path)
    for _ in range(3):
        p, step = g.positions(), g.step()
        f.append_microstate(g).end()
        g.sweep(TRANSLATE, 0.1, 1.0, FP32_RECHECK, n_sweeps=1, increment_step=True)
    f.close()
    r = GsdFile.open(path)
    assert r.n_frames() == 3
    want = np.zeros((n, 3), np.float32)
    w = p.copy()
    for a in range(3):  # wrap(B) with the reference's rounding (cuboid.rs:96-101), then FP32
        lam = w[:, a] / L
        lam = lam - np.where(np.abs(lam - np.trunc(lam)) >= 0.5, np.trunc(lam) + np.sign(lam), np.trunc(lam))
        lam = np.where(lam == 0.5, -0.5, lam)
        want[:, a] = (lam * L).astype(np.float32)
    got = r.iter_arrays(2, "particles/position", np.float32, 3)
    assert np.array_equal(got, want)
    assert list(r.iter_scalars(2, "configuration/step", np.uint64)) == [step]
