"""B200-native Monte Carlo sweep for hoomd-rs's hoomd-mc, driven through its C ABI.

The compute lives in ``libhmc_b200.so`` (CUDA kernels for sm_100a behind the C ABI in
``include/hmc.h``). This module loads that library with ctypes and mirrors the
reference's Rust API on the sweep path so that a caller reads like hoomd-rs code::

    from hoomd_rs_b200 import (Context, HardSphere, Isothermal, Microstate, PairwiseCutoff,
                               ParallelSweep, Periodic, Translate)

    ctx = Context()
    hamiltonian = PairwiseCutoff(HardSphere(diameter=1.0))
    microstate = Microstate(ctx, Periodic(1.0, [L, L, L]), positions, hamiltonian, seed=1)
    sweep = ParallelSweep(1.0, Translate.with_maximum_distance(0.1))
    count = sweep.apply(microstate, hamiltonian, Isothermal(temperature=1.0))
    microstate.increment_step()

There is no CPU fallback: if the library cannot be loaded, importing the module raises.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# HMC_B200_LIB selects another build of the library (for example a variant under test).
LIB_PATH = os.environ.get("HMC_B200_LIB", os.path.join(_HERE, "libhmc_b200.so"))

# hmc_status
OK, INVALID_ARGUMENT, RANGE_TOO_LARGE, OVERLAP_IN_INPUT, CELL_OVERFLOW, NAN_STATE, ITERATION_CAP, TIMEOUT, \
    CUDA_ERROR, OUT_OF_MEMORY, NOT_SUPPORTED, OUTSIDE_CHECKERBOARD, IO_ERROR = range(13)
# hmc_interaction / hmc_move / hmc_precision
HARD_SPHERE, HARD_CONVEX_POLYGON, HARD_CONVEX_POLYHEDRON, LENNARD_JONES, HARD_CONVEX_SURFACE_MESH_2D, \
    OVERLAP_PENALTY, ISOTROPIC = range(7)
# hmc_univariate / hmc_univariate_wrap
UV_LENNARD_JONES, UV_WEEKS_CHANDLER_ANDERSON, UV_HARMONIC, UV_HARMONIC_REPULSION, UV_BOXCAR, UV_OVERLAP_PENALTY, \
    UV_LENNARD_JONES_GAUSS = range(7)
UVW_NONE, UVW_SHIFTED, UVW_EXPANDED, UVW_XPLOR = range(4)
TRANSLATE, ROTATE = range(2)
FP64, FP32_RECHECK = range(2)
# hmc_sweep_params.flags of the tuners
TUNE_PER_SAMPLE_STREAMS = 1


class HmcError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"hmc status {status}: {message}")
        self.status = status


class hmc_device_opts(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("device", C.c_int32)]


class hmc_system_desc(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("dim", C.c_uint32), ("edge_lengths", C.c_double * 3),
                ("n_bodies", C.c_uint64), ("step", C.c_uint64), ("substep", C.c_uint32), ("seed", C.c_uint32),
                ("interaction", C.c_uint32), ("n_vertices", C.c_uint32), ("vertices", C.POINTER(C.c_double)),
                ("diameter", C.c_double), ("lj_epsilon", C.c_double), ("lj_sigma", C.c_double),
                ("lj_r_cut", C.c_double), ("lj_r_shift", C.c_double), ("boundary_range", C.c_double),
                ("body_interaction_range", C.c_double), ("penalty_k", C.c_double),
                ("penalty_maximum_overlap", C.c_double), ("penalty_shoulder", C.c_double),
                ("capacity", C.c_uint64), ("univariate", C.c_uint32), ("univariate_wrap", C.c_uint32),
                ("univariate_params", C.c_double * 4), ("wrap_params", C.c_double * 2),
                ("isotropic_r_cut", C.c_double)]


class hmc_shape_overlap_params(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("reserved", C.c_uint32), ("resolution", C.c_double),
                ("r_cut", C.c_double), ("penalty_k", C.c_double), ("penalty_maximum_overlap", C.c_double),
                ("penalty_shoulder", C.c_double)]


class hmc_sweep_params(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("move", C.c_uint32), ("maximum", C.c_double),
                ("temperature", C.c_double), ("precision", C.c_uint32), ("n_sweeps", C.c_uint32),
                ("increment_step", C.c_uint32), ("flags", C.c_uint32)]


class hmc_count(C.Structure):
    _fields_ = [("accepted", C.c_uint64), ("rejected", C.c_uint64), ("rechecks", C.c_uint64),
                ("pair_checks", C.c_uint64), ("max_fp32_error", C.c_double), ("order_ambiguous", C.c_uint64)]


_SWEEP_PARAMS_DTYPE = np.dtype(hmc_sweep_params)
_COUNT_DTYPE = np.dtype(hmc_count)


class hmc_launch_variant(C.Structure):
    _fields_ = [("index", C.c_uint32), ("count", C.c_uint32), ("blocks_per_sm", C.c_uint32),
                ("trials_per_warp", C.c_uint32), ("own_steps", C.c_uint32)]


class hmc_injected_move(C.Structure):
    _fields_ = [("body", C.c_uint64), ("position", C.c_double * 3), ("orientation", C.c_double * 4),
                ("u", C.c_double)]


class hmc_quick_insert(C.Structure):
    _fields_ = [("target", C.c_uint64), ("allowed_overlaps", C.c_uint64), ("inserted", C.c_uint64),
                ("complete", C.c_uint32), ("reserved", C.c_uint32)]


class hmc_quick_compress(C.Structure):
    _fields_ = [("target_volume", C.c_double), ("maximum_energy_per_site", C.c_double),
                ("maximum_delta", C.c_double), ("state", C.c_uint32), ("is_final", C.c_uint32),
                ("boundary", C.c_double * 3)]


class hmc_grand_canonical_params(C.Structure):
    _fields_ = [("temperature", C.c_double), ("fugacity", C.c_double), ("n_trials", C.c_uint32),
                ("reserved", C.c_uint32)]


class hmc_insert_remove_count(C.Structure):
    _fields_ = [("insert_accepted", C.c_uint64), ("insert_rejected", C.c_uint64), ("remove_accepted", C.c_uint64),
                ("remove_rejected", C.c_uint64)]


class hmc_gsd_chunk(C.Structure):
    _fields_ = [("frame", C.c_uint64), ("rows", C.c_uint64), ("location", C.c_uint64), ("columns", C.c_uint32),
                ("id", C.c_uint16), ("type", C.c_uint8), ("flags", C.c_uint8)]


class hmc_gsd_info(C.Structure):
    _fields_ = [("n_frames", C.c_uint64), ("buffer_frame", C.c_uint64), ("file_length", C.c_uint64),
                ("index_entries", C.c_uint64), ("index_allocated_entries", C.c_uint64),
                ("namelist_allocated_entries", C.c_uint64), ("n_names", C.c_uint32), ("schema_major", C.c_uint16),
                ("schema_minor", C.c_uint16), ("gsd_major", C.c_uint16), ("gsd_minor", C.c_uint16),
                ("writable", C.c_int), ("maximum_write_buffer_size", C.c_uint64),
                ("application", C.c_char * 64), ("schema", C.c_char * 64)]


class hmc_profile(C.Structure):
    _fields_ = [("kernel_launches", C.c_uint64), ("sweep_launches", C.c_uint64), ("sweep_ms", C.c_double),
                ("rebuild_launches", C.c_uint64), ("rebuild_ms", C.c_double), ("sweeps", C.c_uint64)]


# Every function that include/hmc.h declares: name -> (restype, argtypes).
_vp = C.c_void_p
_dp = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)
SIGNATURES = {
    "hmc_abi_version": (C.c_uint32, []),
    "hmc_status_string": (C.c_char_p, [C.c_int]),
    "hmc_last_error_message": (C.c_char_p, []),
    "hmc_context_create": (C.c_int, [C.POINTER(hmc_device_opts), C.POINTER(_vp)]),
    "hmc_context_destroy": (None, [_vp]),
    "hmc_system_create": (C.c_int, [_vp, C.POINTER(hmc_system_desc), _dp, _dp, C.POINTER(_vp)]),
    "hmc_system_destroy": (None, [_vp]),
    "hmc_system_set_stream": (C.c_int, [_vp, _vp]),
    "hmc_system_stream": (_vp, [_vp]),
    "hmc_set_state": (C.c_int, [_vp, _dp, _dp, C.c_uint64, C.c_uint32]),
    "hmc_get_state": (C.c_int, [_vp, _dp, _dp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)]),
    "hmc_increment_step": (C.c_int, [_vp]),
    "hmc_math_sincos": (C.c_int, [_vp, _dp, C.c_uint64, _dp, _dp]),
    "hmc_sdf": (C.c_int, [_vp, C.c_double, C.c_uint32, C.POINTER(C.c_uint64)]),
    "hmc_serial_sweep": (C.c_int, [_vp, C.POINTER(hmc_sweep_params), _u8p, C.POINTER(hmc_count)]),
    "hmc_gr": (C.c_int, [_vp, C.c_double, C.c_uint32, C.POINTER(C.c_uint64)]),
    "hmc_batch_create": (C.c_int, [_vp, C.c_uint32, C.POINTER(hmc_system_desc), C.POINTER(_dp), C.POINTER(_vp)]),
    "hmc_batch_destroy": (None, [_vp]),
    "hmc_batch_sweep": (C.c_int, [_vp, C.POINTER(hmc_sweep_params), C.POINTER(hmc_count), C.POINTER(hmc_count)]),
    "hmc_batch_get_state": (C.c_int, [_vp, C.c_uint32, _dp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)]),
    "hmc_batch_set_state": (C.c_int, [_vp, C.c_uint32, _dp, C.c_uint64, C.c_uint32]),
    "hmc_batch_overlap_check": (C.c_int, [_vp, C.POINTER(C.c_uint64)]),
    "hmc_batch_sdf": (C.c_int, [_vp, C.c_double, C.c_uint32, C.POINTER(C.c_uint64)]),
    "hmc_batch_tune": (C.c_int, [_vp, C.POINTER(hmc_sweep_params), C.c_double, C.c_uint32, C.c_uint32]),
    "hmc_batch_kernel_launches": (C.c_uint64, [_vp]),
    "hmc_sweep": (C.c_int, [_vp, C.POINTER(hmc_sweep_params), C.POINTER(hmc_count)]),
    "hmc_tune": (C.c_int, [_vp, C.POINTER(hmc_sweep_params), C.c_double, C.c_uint32, C.c_uint32]),
    "hmc_overlap_check": (C.c_int, [_vp, C.POINTER(C.c_uint64)]),
    "hmc_eval_moves": (C.c_int, [_vp, C.POINTER(hmc_injected_move), C.c_uint64, C.c_double, C.c_uint32, _u8p,
                                 _u8p, _dp]),
    "hmc_eval_trials": (C.c_int, [_vp, C.POINTER(hmc_injected_move), C.c_uint64, C.c_double, C.c_uint32, _u8p,
                                  _u8p]),
    "hmc_sample_moves": (C.c_int, [_vp, C.c_uint32, C.c_uint32, C.c_double, C.c_uint64, C.c_uint32, C.c_uint32,
                                   C.c_uint64, _dp]),
    "hmc_get_launch_variant": (C.c_int, [_vp, C.c_uint32, C.c_uint32, C.POINTER(hmc_launch_variant)]),
    "hmc_set_launch_variant": (C.c_int, [_vp, C.c_uint32, C.c_uint32]),
    "hmc_autotune": (C.c_int, [_vp, C.POINTER(hmc_sweep_params), C.c_uint32, C.POINTER(hmc_launch_variant), _dp]),
    "hmc_batch_autotune": (C.c_int, [_vp, C.POINTER(hmc_sweep_params), C.c_uint32, C.POINTER(hmc_launch_variant),
                                     _dp]),
    "hmc_batch_set_launch_variant": (C.c_int, [_vp, C.c_uint32, C.c_uint32]),
    "hmc_batch_set_captured_sweeps": (C.c_int, [_vp, C.c_uint32]),
    "hmc_total_energy": (C.c_int, [_vp, _dp]),
    "hmc_overlap_count_noalloc": (C.c_int, [_vp, C.c_uint64, C.c_uint32, _dp, C.c_double, C.c_double, _vp, _vp]),
    "hmc_quick_insert_apply": (C.c_int, [_vp, C.POINTER(hmc_quick_insert), C.POINTER(hmc_count)]),
    "hmc_quick_compress_apply": (C.c_int, [_vp, C.POINTER(hmc_quick_compress)]),
    "hmc_grand_canonical_apply": (C.c_int, [_vp, C.POINTER(hmc_grand_canonical_params),
                                            C.POINTER(hmc_insert_remove_count)]),
    "hmc_get_box": (C.c_int, [_vp, _dp]),
    "hmc_set_box": (C.c_int, [_vp, _dp]),
    "hmc_get_n_bodies": (C.c_int, [_vp, C.POINTER(C.c_uint64)]),
    "hmc_set_shape_overlap": (C.c_int, [_vp, C.POINTER(hmc_shape_overlap_params)]),
    "hmc_set_cooperative_pass": (C.c_int, [_vp, C.c_uint32, C.c_uint32]),
    "hmc_get_cooperative_pass": (C.c_int, [_vp, C.c_uint32, C.POINTER(C.c_uint32)]),
    "hmc_gsd_last_error": (C.c_int, []),
    "hmc_gsd_create": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_uint16, C.c_uint16, C.c_int,
                                 C.POINTER(_vp)]),
    "hmc_gsd_open": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(_vp)]),
    "hmc_gsd_close": (C.c_int, [_vp]),
    "hmc_gsd_write_chunk": (C.c_int, [_vp, C.c_char_p, C.c_uint32, C.c_uint64, C.c_uint32, _vp]),
    "hmc_gsd_write_strings": (C.c_int, [_vp, C.c_char_p, C.POINTER(C.c_char_p), C.c_uint64]),
    "hmc_gsd_end_frame": (C.c_int, [_vp]),
    "hmc_gsd_sync": (C.c_int, [_vp]),
    "hmc_gsd_set_maximum_write_buffer_size": (C.c_int, [_vp, C.c_uint64]),
    "hmc_gsd_get_info": (C.c_int, [_vp, C.POINTER(hmc_gsd_info)]),
    "hmc_gsd_name": (C.c_int, [_vp, C.c_uint32, C.c_char_p, C.c_uint64]),
    "hmc_gsd_find_chunk": (C.c_int, [_vp, C.c_uint64, C.c_char_p, C.POINTER(hmc_gsd_chunk), C.POINTER(C.c_int)]),
    "hmc_gsd_read_chunk": (C.c_int, [_vp, C.c_uint64, C.c_char_p, C.c_uint32, C.c_uint32, _vp, C.c_uint64,
                                     C.POINTER(C.c_uint64)]),
    "hmc_gsd_create_hoomd": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(_vp)]),
    "hmc_gsd_append_frame": (C.c_int, [_vp, C.c_uint64]),
    "hmc_gsd_frame_particles": (C.c_int, [_vp, C.c_char_p, C.c_uint32, C.c_uint64, C.c_uint32, _vp]),
    "hmc_gsd_frame_end": (C.c_int, [_vp]),
    "hmc_gsd_set_auto_sync_delay": (C.c_int, [_vp, C.c_double]),
    "hmc_gsd_append_system": (C.c_int, [_vp, _vp]),
    "hmc_profile_enable": (C.c_int, [_vp, C.c_int]),
    "hmc_profile_read": (C.c_int, [_vp, C.POINTER(hmc_profile), C.c_int]),
}

_lib = None


def load_library(path: str = LIB_PATH):
    """Load libhmc_b200.so and bind every C-ABI symbol. Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m hoomd_rs_b200.build` "
                          "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(status: int):
    if status != OK:
        msg = _lib.hmc_last_error_message().decode()
        raise HmcError(status, msg)


class Context:
    """A CUDA device context (hmc_context)."""

    def __init__(self, device: int = 0):
        lib = load_library()
        opts = hmc_device_opts(C.sizeof(hmc_device_opts), device)
        h = _vp()
        _check(lib.hmc_context_create(C.byref(opts), C.byref(h)))
        self._h = h
        self.device = device

    def sincos(self, x) -> "tuple[np.ndarray, np.ndarray]":
        """The correctly rounded sin and cos of the 2-D rotation path, evaluated on the device."""
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
        sn = np.empty_like(x)
        cs = np.empty_like(x)
        _check(_lib.hmc_math_sincos(self._h, x.ctypes.data_as(_dp), x.size, sn.ctypes.data_as(_dp),
                                    cs.ctypes.data_as(_dp)))
        return sn, cs

    def sample_moves(self, dim: int, kind: int, maximum: float, n: int, step: int = 0, substep: int = 0,
                     seed: int = 0) -> np.ndarray:
        """n proposals of the device samplers (hmc_sample_moves), sample i from
        Counter(step, substep, seed).index(i): kind 0 Translate displacements (n x dim), kind 1 Rotate
        (3-D versors n x 4, 2-D angles n), kind 2 StandardNormal draws (n)."""
        per = 1 if kind == 2 else (dim if kind == 0 else (4 if dim == 3 else 1))
        out = np.empty(n * per)
        _check(_lib.hmc_sample_moves(self._h, dim, kind, maximum, step, substep, seed, n, out.ctypes.data_as(_dp)))
        return out.reshape(n, per) if per > 1 else out

    def close(self):
        if getattr(self, "_h", None):
            _lib.hmc_context_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


# ---- mirrors of the reference's types ---------------------------------------------------------
@dataclass
class HardSphere:
    """hoomd_interaction::pairwise::HardSphere (hard_shape.rs:128-175)."""
    diameter: float = 1.0

    @property
    def maximum_interaction_range(self) -> float:
        return self.diameter


@dataclass
class LennardJones:
    """hoomd_interaction::univariate::LennardJones (lennard_jones.rs:79-124)."""
    epsilon: float = 1.0
    sigma: float = 1.0


@dataclass
class OverlapPenalty:
    """hoomd_interaction::univariate::OverlapPenalty (overlap_penalty.rs:42-116): inf below
    -maximum_allowed_overlap, (k/2) r^2 + epsilon_shoulder below 0, else 0. Defaults as
    OverlapPenalty::default()."""
    k: float = 10000.0
    maximum_allowed_overlap: float = 0.2
    epsilon_shoulder: float = 100.0


@dataclass
class WeeksChandlerAnderson:
    """hoomd_interaction::univariate::WeeksChandlerAnderson (weeks_chandler_anderson.rs): the
    Lennard-Jones energy plus epsilon below 2^(1/6) sigma, else 0."""
    epsilon: float = 1.0
    sigma: float = 1.0


@dataclass
class Harmonic:
    """hoomd_interaction::univariate::Harmonic (harmonic.rs): 0.5 k (r - r_0)^2."""
    k: float
    r_0: float


@dataclass
class HarmonicRepulsion:
    """hoomd_interaction::univariate::HarmonicRepulsion (harmonic_repulsion.rs): 0.5 a / r_cut
    (r - r_cut)^2 below r_cut, else 0."""
    a: float
    r_cut: float


@dataclass
class Boxcar:
    """hoomd_interaction::univariate::Boxcar (boxcar.rs): epsilon on [left, right), else 0."""
    epsilon: float
    left: float
    right: float


@dataclass
class LennardJonesGauss:
    """hoomd_interaction::univariate::LennardJonesGauss (lennard_jones_gauss.rs): r_inv^12 - 2 r_inv^6
    - epsilon exp(-(r / scale - r_0)^2 / (2 sigma_squared)), r_inv = scale / r."""
    epsilon: float
    sigma_squared: float
    r_0: float
    scale: float = 1.0


@dataclass
class Xplor:
    """hoomd_interaction::univariate::Xplor (xplor.rs): f(r) smoothed to 0 between r_smooth and
    r_cut."""
    f: object
    r_cut: float
    r_smooth: float


@dataclass
class Expanded:
    """hoomd_interaction::univariate::Expanded (expanded.rs:62-67): f(r - delta)."""
    delta: float
    f: OverlapPenalty


@dataclass
class Shifted:
    """hoomd_interaction::univariate::Shifted (shifted.rs:57-102): f(r) - f(r_shift)."""
    f: LennardJones
    r_shift: float


@dataclass
class Isotropic:
    """hoomd_interaction::pairwise::Isotropic (isotropic.rs:88-187)."""
    interaction: object  # Shifted(LennardJones) or Expanded(OverlapPenalty)
    r_cut: float

    @property
    def maximum_interaction_range(self) -> float:
        return self.r_cut


@dataclass
class ConvexPolyhedron:
    """hoomd_geometry::shape::ConvexPolyhedron (convex_polytope.rs:120): up to 32 vertices."""
    vertices: np.ndarray

    @classmethod
    def with_vertices(cls, vertices) -> "ConvexPolyhedron":
        v = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 3)
        return cls(v)

    @property
    def bounding_radius(self) -> float:
        return float(np.sqrt(max(float(np.dot(v, v)) for v in self.vertices)))


@dataclass
class ConvexPolygon:
    """hoomd_geometry::shape::ConvexPolygon (convex_polytope.rs:100): 3 to 32 vertices, any order
    (the support function's first maximum follows the given order); XenoCollide overlaps."""
    vertices: np.ndarray

    @classmethod
    def with_vertices(cls, vertices) -> "ConvexPolygon":
        return cls(np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 2))

    @classmethod
    def regular(cls, n: int) -> "ConvexPolygon":
        """ConvexPolygon::regular (convex_polytope.rs:137-152): vertex x at 0.5 (cos, sin) of
        theta = 2 pi x / n. The reference sets the bounding radius to 0.5; here it is computed
        from the vertices (0.5 up to the rounding of cos and sin)."""
        return cls(np.array([[0.5 * math.cos(2.0 * math.pi * x / n), 0.5 * math.sin(2.0 * math.pi * x / n)]
                             for x in range(n)]))

    @property
    def bounding_radius(self) -> float:
        return float(np.sqrt(max(float(np.dot(v, v)) for v in self.vertices)))


def convex_hull_2d(points) -> np.ndarray:
    """Counter-clockwise hull without collinear points, starting at the lowest (then leftmost)
    point, as ConvexSurfaceMesh2d::construct_convex_hull keeps it (convex_surface_mesh_2d.rs:166-260)."""
    pts = sorted({(float(x), float(y)) for x, y in np.asarray(points, dtype=np.float64).reshape(-1, 2)})

    def cross(o, a, b):
        return (a[0] - o[0]) * (b[1] - o[1]) - (a[1] - o[1]) * (b[0] - o[0])

    lower, upper = [], []
    for p in pts:
        while len(lower) >= 2 and cross(lower[-2], lower[-1], p) <= 0:
            lower.pop()
        lower.append(p)
    for p in reversed(pts):
        while len(upper) >= 2 and cross(upper[-2], upper[-1], p) <= 0:
            upper.pop()
        upper.append(p)
    hull = lower[:-1] + upper[:-1]
    if len(hull) < 3:
        raise HmcError(INVALID_ARGUMENT, "fewer than 3 non-collinear points")
    start = min(range(len(hull)), key=lambda i: (hull[i][1], hull[i][0]))
    return np.array(hull[start:] + hull[:start])


@dataclass
class ConvexSurfaceMesh2d:
    """hoomd_geometry::shape::ConvexSurfaceMesh2d (convex_surface_mesh_2d.rs): a convex polygon
    held as its counter-clockwise hull; separating-axis overlaps."""
    vertices: np.ndarray

    @classmethod
    def from_point_set(cls, points) -> "ConvexSurfaceMesh2d":
        return cls(convex_hull_2d(points))

    @property
    def bounding_radius(self) -> float:
        return float(np.sqrt(max(float(np.dot(v, v)) for v in self.vertices)))


@dataclass
class HardShape:
    """hoomd_interaction::pairwise::HardShape(Convex(shape)) or HardShape(ConvexSurfaceMesh2d)
    (hard_shape.rs:33-119)."""
    shape: object

    @property
    def maximum_interaction_range(self) -> float:
        return self.shape.bounding_radius * 2.0


@dataclass
class ApproximateShapeOverlap:
    """hoomd_interaction::pairwise::ApproximateShapeOverlap (approximate_shape_overlap.rs:52-171):
    the isotropic energy (an OverlapPenalty) at minus the approximate distance, in steps of
    `resolution`, that shape j must move along the line of centres to stop intersecting shape i.
    For Convex polyhedra and polygons; only for preparing states (QuickInsert, QuickCompress)."""
    shape: object  # ConvexPolyhedron or ConvexPolygon
    isotropic: OverlapPenalty
    resolution: float

    @classmethod
    def new(cls, shape, isotropic: OverlapPenalty, resolution: float) -> "ApproximateShapeOverlap":
        return cls(shape, isotropic, float(resolution))


@dataclass
class Anisotropic:
    """hoomd_interaction::pairwise::Anisotropic (anisotropic.rs:88-143): the pair energy in the
    local frame of site i, 0 at a centre distance >= r_cut."""
    interaction: ApproximateShapeOverlap
    r_cut: float

    @property
    def maximum_interaction_range(self) -> float:
        return self.r_cut


@dataclass
class PairwiseCutoff:
    """hoomd_interaction::PairwiseCutoff (pairwise_cutoff.rs:140)."""
    pair: object

    @property
    def maximum_interaction_range(self) -> float:
        return self.pair.maximum_interaction_range


@dataclass
class Periodic:
    """hoomd_microstate::boundary::Periodic<Hypercuboid<N>> (boundary/periodic.rs:65-107)."""
    maximum_interaction_range: float
    edge_lengths: Sequence[float]


@dataclass
class Isothermal:
    """hoomd_simulation::macrostate::Isothermal (macrostate.rs:109)."""
    temperature: float = 1.0


@dataclass
class Count:
    """hoomd_mc::Count (lib.rs:206-294), plus the FP32 recheck statistics."""
    accepted: int = 0
    rejected: int = 0
    rechecks: int = 0
    pair_checks: int = 0
    max_fp32_error: float = 0.0
    order_ambiguous: int = 0  # soft-potential decisions another summation order could change

    def total(self) -> int:
        return self.accepted + self.rejected

    def acceptance_ratio(self) -> Optional[float]:
        t = self.total()
        return self.accepted / t if t > 0 else None


@dataclass
class Rotate:
    """hoomd_mc::Rotate<Versor> (rotate/versor.rs:40-123): Gaussian rotation vector, sigma = maximum."""
    maximum_rotation: float

    @classmethod
    def with_maximum_rotation(cls, a: float) -> "Rotate":
        return cls(float(a))


@dataclass
class Translate:
    """hoomd_mc::Translate (translate.rs:41, translate/cartesian.rs:40-51)."""
    maximum_distance: float

    @classmethod
    def with_maximum_distance(cls, d: float) -> "Translate":
        return cls(float(d))


def sdf_pressure(counts, n: int, volume: float, dim: int, x_max: float, fit_bins: int = 12) -> float:
    """beta P = rho (1 + s(0+) / dim) from SDF pair counts (pairs counted once, s = counts/(N dx))."""
    counts = np.asarray(counts, dtype=np.float64)
    dx = x_max / counts.size
    x = (np.arange(counts.size) + 0.5) * dx
    sx = counts / (n * dx)
    k = min(fit_bins, counts.size)
    s0 = np.polyval(np.polyfit(x[:k], sx[:k], 2), 0.0)
    rho = n / volume
    return float(rho * (1.0 + s0 / dim))


def gr_normalise(counts, n: int, volume: float, dim: int, r_max: float) -> "tuple[np.ndarray, np.ndarray]":
    """(r, g(r)) from pair counts (pairs counted once)."""
    counts = np.asarray(counts, dtype=np.float64)
    edges = np.linspace(0.0, r_max, counts.size + 1)
    shell = (np.pi * (edges[1:] ** 2 - edges[:-1] ** 2) if dim == 2
             else 4.0 / 3.0 * np.pi * (edges[1:] ** 3 - edges[:-1] ** 3))
    ideal = 0.5 * n * (n - 1) / volume * shell
    return 0.5 * (edges[1:] + edges[:-1]), counts / ideal


def _univariate(e):
    """(hmc_univariate, its parameters, hmc_univariate_wrap, its parameters) of a univariate energy,
    plain or in one Shifted, Expanded or Xplor."""
    wrap, wparams = UVW_NONE, ()
    if isinstance(e, Shifted):
        wrap, wparams, e = UVW_SHIFTED, (e.r_shift,), e.f
    elif isinstance(e, Expanded):
        wrap, wparams, e = UVW_EXPANDED, (e.delta,), e.f
    elif isinstance(e, Xplor):
        wrap, wparams, e = UVW_XPLOR, (e.r_cut, e.r_smooth), e.f
    if isinstance(e, LennardJones):
        return UV_LENNARD_JONES, (e.epsilon, e.sigma), wrap, wparams
    if isinstance(e, WeeksChandlerAnderson):
        return UV_WEEKS_CHANDLER_ANDERSON, (e.epsilon, e.sigma), wrap, wparams
    if isinstance(e, Harmonic):
        return UV_HARMONIC, (e.k, e.r_0), wrap, wparams
    if isinstance(e, HarmonicRepulsion):
        return UV_HARMONIC_REPULSION, (e.a, e.r_cut), wrap, wparams
    if isinstance(e, Boxcar):
        return UV_BOXCAR, (e.epsilon, e.left, e.right), wrap, wparams
    if isinstance(e, OverlapPenalty):
        return UV_OVERLAP_PENALTY, (e.k, e.maximum_allowed_overlap, e.epsilon_shoulder), wrap, wparams
    if isinstance(e, LennardJonesGauss):
        return UV_LENNARD_JONES_GAUSS, (e.epsilon, e.sigma_squared, e.r_0, e.scale), wrap, wparams
    raise HmcError(NOT_SUPPORTED, f"univariate {type(e).__name__}")


class Microstate:
    """Bodies in a periodic box, resident on the GPU (one hmc_system)."""

    def __init__(self, ctx: Context, boundary: Periodic, positions, hamiltonian: PairwiseCutoff, *,
                 step: int = 0, substep: int = 0, seed: int = 0, body_interaction_range: float = 0.0,
                 orientations=None, capacity: int = 0):
        lib = load_library()
        L = [float(x) for x in boundary.edge_lengths]
        self.dim = len(L)
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, self.dim)
        self.n = pos.shape[0]
        d = hmc_system_desc()
        d.struct_size = C.sizeof(hmc_system_desc)
        d.dim = self.dim
        for a, x in enumerate(L):
            d.edge_lengths[a] = x
        d.n_bodies = self.n
        d.step, d.substep, d.seed = step, substep, seed
        pair = hamiltonian.pair
        if isinstance(pair, HardSphere):
            d.interaction = HARD_SPHERE
            d.diameter = pair.diameter
        elif isinstance(pair, HardShape):
            d.interaction = {ConvexPolyhedron: HARD_CONVEX_POLYHEDRON, ConvexPolygon: HARD_CONVEX_POLYGON,
                             ConvexSurfaceMesh2d: HARD_CONVEX_SURFACE_MESH_2D}[type(pair.shape)]
            verts = np.ascontiguousarray(pair.shape.vertices, dtype=np.float64)
            self._verts = verts  # keep alive during the call
            d.n_vertices = verts.shape[0]
            d.vertices = verts.ctypes.data_as(_dp)
        elif (isinstance(pair, Isotropic) and isinstance(pair.interaction, Expanded)
              and isinstance(pair.interaction.f, OverlapPenalty) and pair.interaction.delta == pair.r_cut):
            # the overlap-penalty sphere: Isotropic { Expanded { delta: d, OverlapPenalty }, r_cut: d }
            d.interaction = OVERLAP_PENALTY
            d.diameter = pair.r_cut
            d.penalty_k = pair.interaction.f.k
            d.penalty_maximum_overlap = pair.interaction.f.maximum_allowed_overlap
            d.penalty_shoulder = pair.interaction.f.epsilon_shoulder
        elif (isinstance(pair, Isotropic) and isinstance(pair.interaction, Shifted)
              and isinstance(pair.interaction.f, LennardJones)):
            d.interaction = LENNARD_JONES
            d.lj_epsilon = pair.interaction.f.epsilon
            d.lj_sigma = pair.interaction.f.sigma
            d.lj_r_cut = pair.r_cut
            d.lj_r_shift = pair.interaction.r_shift
        elif isinstance(pair, Isotropic):
            d.interaction = ISOTROPIC
            kind, params, wrap, wparams = _univariate(pair.interaction)
            d.univariate, d.univariate_wrap = kind, wrap
            for k, x in enumerate(params):
                d.univariate_params[k] = x
            for k, x in enumerate(wparams):
                d.wrap_params[k] = x
            d.isotropic_r_cut = pair.r_cut
        else:
            raise HmcError(NOT_SUPPORTED, f"{type(pair).__name__}")
        d.boundary_range = boundary.maximum_interaction_range
        d.body_interaction_range = body_interaction_range
        d.capacity = max(int(capacity), self.n)
        self.oriented = d.interaction in (HARD_CONVEX_POLYHEDRON, HARD_CONVEX_POLYGON, HARD_CONVEX_SURFACE_MESH_2D)
        self.ori_len = (4 if self.dim == 3 else 1) if self.oriented else 0
        ori = None
        if self.oriented:
            if orientations is None:
                orientations = np.tile([1.0, 0.0, 0.0, 0.0], (self.n, 1)) if self.dim == 3 else np.zeros(self.n)
            ori = np.ascontiguousarray(orientations, dtype=np.float64).reshape(self.n * self.ori_len)
        h = _vp()
        _check(lib.hmc_system_create(ctx._h, C.byref(d), pos.ctypes.data_as(_dp),
                                     None if ori is None else ori.ctypes.data_as(_dp), C.byref(h)))
        self._h = h
        self._ctx = ctx  # keep the context alive
        self.edge_lengths = L
        self.hamiltonian = hamiltonian

    def close(self):
        if getattr(self, "_h", None):
            _lib.hmc_system_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    # microstate.rs:412-455
    def state(self, out: Optional[np.ndarray] = None):
        """(positions, step, substep); `out` (n x dim float64, C-contiguous) receives the positions."""
        pos = np.empty((self.n, self.dim)) if out is None else out
        if pos.shape != (self.n, self.dim) or pos.dtype != np.float64 or not pos.flags.c_contiguous:
            raise HmcError(INVALID_ARGUMENT, "out must be a C-contiguous float64 array of shape (n, dim)")
        step = C.c_uint64()
        sub = C.c_uint32()
        _check(_lib.hmc_get_state(self._h, pos.ctypes.data_as(_dp), None, C.byref(step), C.byref(sub)))
        return pos, step.value, sub.value

    def orientations(self) -> np.ndarray:
        """Versors (n x 4: s, x, y, z) in 3-D, angles (n) in 2-D."""
        ori = np.zeros((self.n, 4)) if self.dim == 3 else np.zeros(self.n)
        _check(_lib.hmc_get_state(self._h, None, ori.ctypes.data_as(_dp), None, None))
        return ori

    def positions(self) -> np.ndarray:
        return self.state()[0]

    def _counter(self):
        step = C.c_uint64()
        sub = C.c_uint32()
        _check(_lib.hmc_get_state(self._h, None, None, C.byref(step), C.byref(sub)))
        return step.value, sub.value

    def step(self) -> int:
        return self._counter()[0]

    def substep(self) -> int:
        return self._counter()[1]

    def set_state(self, positions, step: int, substep: int, orientations=None):
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(self.n, self.dim)
        ori = None if orientations is None else np.ascontiguousarray(orientations, dtype=np.float64).reshape(
            self.n * (4 if self.dim == 3 else 1))
        _check(_lib.hmc_set_state(self._h, pos.ctypes.data_as(_dp), None if ori is None else ori.ctypes.data_as(_dp),
                                  step, substep))

    def increment_step(self):
        """Microstate::increment_step (microstate.rs:412-430): step += 1, substep = 0."""
        _check(_lib.hmc_increment_step(self._h))

    def tune(self, move: int, maximum: float, temperature: float, precision: int, target: float, samples: int,
             steps: int, per_sample_streams: bool = False) -> float:
        """Tune::tune_with_options: the reference's single-stream tuner (tune_local.rs:42-88), or
        with per_sample_streams the faster variant that gives every sample its own stream."""
        p = hmc_sweep_params(C.sizeof(hmc_sweep_params), move, maximum, temperature, precision, 1, 0,
                             TUNE_PER_SAMPLE_STREAMS if per_sample_streams else 0)
        _check(_lib.hmc_tune(self._h, C.byref(p), target, samples, steps))
        return p.maximum

    def sdf(self, x_max: float = 0.02, n_bins: int = 40) -> np.ndarray:
        """Pair counts (i < j) by x = 1 - sigma/r over [0, x_max) (hard spheres)."""
        out = np.zeros(n_bins, dtype=np.uint64)
        _check(_lib.hmc_sdf(self._h, x_max, n_bins, out.ctypes.data_as(C.POINTER(C.c_uint64))))
        return out

    def gr_counts(self, r_max: float, n_bins: int) -> np.ndarray:
        """Pair counts (i < j) by minimum-image distance over [0, r_max)."""
        out = np.zeros(n_bins, dtype=np.uint64)
        _check(_lib.hmc_gr(self._h, r_max, n_bins, out.ctypes.data_as(C.POINTER(C.c_uint64))))
        return out

    def pressure(self, x_max: float = 0.02, n_bins: int = 40, fit_bins: int = 12) -> float:
        """beta P from the scale distribution: rho (1 + s(0+) / dim), s(x) = counts / (N dx)
        extrapolated to x = 0 by a quadratic fit over the first fit_bins bins."""
        return sdf_pressure(self.sdf(x_max, n_bins), self.n, self.volume(), self.dim, x_max, fit_bins)

    def volume(self) -> float:
        return float(np.prod(self.edge_lengths))

    def overlap_count(self) -> int:
        n = C.c_uint64()
        _check(_lib.hmc_overlap_check(self._h, C.byref(n)))
        return n.value

    def stream(self) -> int:
        return _lib.hmc_system_stream(self._h) or 0

    def profile(self, enable: Optional[bool] = None, reset: bool = False) -> dict:
        if enable is not None:
            _check(_lib.hmc_profile_enable(self._h, int(enable)))
        p = hmc_profile()
        _check(_lib.hmc_profile_read(self._h, C.byref(p), int(reset)))
        return {f: getattr(p, f) for f, _ in hmc_profile._fields_}

    def set_stream(self, stream_ptr: int):
        _check(_lib.hmc_system_set_stream(self._h, C.c_void_p(stream_ptr)))

    def sweep(self, move: int, maximum: float, temperature: float, precision: int, n_sweeps: int = 1,
              increment_step: bool = False) -> Count:
        p = hmc_sweep_params(C.sizeof(hmc_sweep_params), move, maximum, temperature, precision, n_sweeps,
                             int(increment_step), 0)
        c = hmc_count()
        _check(_lib.hmc_sweep(self._h, C.byref(p), C.byref(c)))
        return Count(c.accepted, c.rejected, c.rechecks, c.pair_checks, c.max_fp32_error, c.order_ambiguous)

    def launch_variant(self, precision: int, index: Optional[int] = None) -> dict:
        """The launch variant the next sweep runs in this precision (or variant `index`)."""
        v = hmc_launch_variant()
        _check(_lib.hmc_get_launch_variant(self._h, precision, 0xFFFFFFFF if index is None else index, C.byref(v)))
        return {f: getattr(v, f) for f, _ in hmc_launch_variant._fields_}

    def set_launch_variant(self, precision: int, index: Optional[int]):
        """Force a launch variant (None: the autotuner's recorded choice for this workload, else 0)."""
        _check(_lib.hmc_set_launch_variant(self._h, precision, 0xFFFFFFFF if index is None else index))

    def set_cooperative_pass(self, precision: int, cooperative: bool):
        """Hard spheres: the warp-cooperative colour pass (the FP64 default) or one lane per trial
        (the FP32 default) for this precision; the trajectory is the same."""
        _check(_lib.hmc_set_cooperative_pass(self._h, precision, int(cooperative)))

    def cooperative_pass(self, precision: int) -> bool:
        """Hard spheres: whether the next sweep in this precision runs the warp-cooperative pass."""
        v = C.c_uint32()
        _check(_lib.hmc_get_cooperative_pass(self._h, precision, C.byref(v)))
        return bool(v.value)

    def autotune(self, move: int, maximum: float, temperature: float, precision: int, sweeps: int = 4):
        """hmc_autotune: time every launch variant of this system's pass from the current state
        (restored after), keep the fastest; returns (chosen variant, ms per sweep per variant)."""
        p = hmc_sweep_params(C.sizeof(hmc_sweep_params), move, maximum, temperature, precision, 1, 1, 0)
        v = hmc_launch_variant()
        ms = np.zeros(16)
        _check(_lib.hmc_autotune(self._h, C.byref(p), sweeps, C.byref(v), ms.ctypes.data_as(_dp)))
        return {f: getattr(v, f) for f, _ in hmc_launch_variant._fields_}, ms[: v.count].copy()

    def serial_sweep(self, maximum: float, n_sweeps: int = 1, increment_step: bool = False, move_mask=None,
                     temperature: float = 1.0, move: int = TRANSLATE) -> "Count":
        """Sweep::apply_with_filter (sweep.rs:159-224), any interaction: bodies in index order from
        one sequential stream; move_mask (n booleans) plays should_move_body; ROTATE for shapes."""
        p = hmc_sweep_params(C.sizeof(hmc_sweep_params), move, maximum, temperature, FP64, n_sweeps,
                             int(increment_step), 0)
        c = hmc_count()
        mask = None
        if move_mask is not None:
            mask = np.ascontiguousarray(np.asarray(move_mask, dtype=bool).astype(np.uint8))
        _check(_lib.hmc_serial_sweep(self._h, C.byref(p), None if mask is None else mask.ctypes.data_as(_u8p), C.byref(c)))
        return Count(c.accepted, c.rejected, 0, 0, 0.0, c.order_ambiguous)

    def eval_moves(self, bodies, positions, u=None, temperature: float = 1.0, precision: int = FP64,
                   return_delta_h: bool = False, orientations=None):
        bodies = np.asarray(bodies, dtype=np.uint64)
        pos = np.asarray(positions, dtype=np.float64).reshape(len(bodies), self.dim)
        n = len(bodies)
        arr = np.zeros(n, dtype=[("body", np.uint64), ("position", np.float64, 3), ("orientation", np.float64, 4),
                                 ("u", np.float64)])
        arr["body"] = bodies
        arr["position"][:, : self.dim] = pos
        arr["u"] = -1.0 if u is None else np.asarray(u, dtype=np.float64)
        if orientations is not None:
            if self.dim == 3:
                arr["orientation"] = np.asarray(orientations, dtype=np.float64).reshape(n, 4)
            else:
                arr["orientation"][:, 0] = np.asarray(orientations, dtype=np.float64).reshape(n)
        moves = arr.ctypes.data_as(C.POINTER(hmc_injected_move))
        dec = np.zeros(n, dtype=np.uint8)
        rech = np.zeros(n, dtype=np.uint8)
        dh = np.zeros(n)
        _check(_lib.hmc_eval_moves(self._h, moves, n, temperature, precision, dec.ctypes.data_as(_u8p),
                                   rech.ctypes.data_as(_u8p), dh.ctypes.data_as(_dp)))
        if return_delta_h:
            return dec.astype(bool), rech.astype(bool), dh
        return dec.astype(bool), rech.astype(bool)

    def eval_trials(self, bodies, positions, u=None, temperature: float = 1.0, precision: int = FP64,
                    orientations=None):
        """The colour pass's own decisions for injected trials (hmc_eval_trials): positions are
        W1 = wrap(propose(..)); returns (decisions, flags) with flag bit 0 = settled in FP64 by
        the FP32 pass, bit 1 = outside the body's checkerboard space."""
        bodies = np.asarray(bodies, dtype=np.uint64)
        n = len(bodies)
        arr = np.zeros(n, dtype=[("body", np.uint64), ("position", np.float64, 3), ("orientation", np.float64, 4),
                                 ("u", np.float64)])
        arr["body"] = bodies
        arr["position"][:, : self.dim] = np.asarray(positions, dtype=np.float64).reshape(n, self.dim)
        arr["u"] = -1.0 if u is None else np.asarray(u, dtype=np.float64)
        if orientations is not None:
            arr["orientation"] = np.asarray(orientations, dtype=np.float64).reshape(n, 4)
        moves = arr.ctypes.data_as(C.POINTER(hmc_injected_move))
        dec = np.zeros(n, dtype=np.uint8)
        flags = np.zeros(n, dtype=np.uint8)
        _check(_lib.hmc_eval_trials(self._h, moves, n, temperature, precision, dec.ctypes.data_as(_u8p),
                                    flags.ctypes.data_as(_u8p)))
        return dec.astype(bool), flags

    def refresh(self):
        """Re-read the body count (QuickInsert appends bodies on the device)."""
        n = C.c_uint64()
        _check(_lib.hmc_get_n_bodies(self._h, C.byref(n)))
        self.n = n.value

    def box(self) -> np.ndarray:
        L = np.zeros(3)
        _check(_lib.hmc_get_box(self._h, L.ctypes.data_as(_dp)))
        return L[:self.dim].copy()

    def set_box(self, edge_lengths):
        """Microstate::clone_with_boundary onto a periodic box with these edge lengths."""
        L = np.zeros(3)
        L[:self.dim] = edge_lengths
        _check(_lib.hmc_set_box(self._h, L.ctypes.data_as(_dp)))
        self.edge_lengths = [float(x) for x in L[:self.dim]]

    def volume(self) -> float:
        v = None
        for x in self.box():
            v = x if v is None else v * x
        return float(v)

    def total_energy(self) -> float:
        e = C.c_double()
        _check(_lib.hmc_total_energy(self._h, C.byref(e)))
        return e.value

    def set_hamiltonian(self, hamiltonian: PairwiseCutoff):
        """The hamiltonian the next sweeps, QuickInsert, QuickCompress and total_energy use: the
        system's own, or for convex shapes PairwiseCutoff(Anisotropic(ApproximateShapeOverlap)),
        the insertion hamiltonian of place_single_site_orientable_bodies (hmc_set_shape_overlap)."""
        pair = hamiltonian.pair
        if isinstance(pair, Anisotropic) and isinstance(pair.interaction, ApproximateShapeOverlap):
            a = pair.interaction
            own = self.hamiltonian.pair
            if not (isinstance(own, HardShape) and type(own.shape) is type(a.shape)
                    and np.array_equal(np.asarray(own.shape.vertices), np.asarray(a.shape.vertices))):
                raise HmcError(NOT_SUPPORTED, "the approximate shape overlap needs the system's own shape")
            prm = hmc_shape_overlap_params(C.sizeof(hmc_shape_overlap_params), 0, a.resolution, pair.r_cut,
                                           a.isotropic.k, a.isotropic.maximum_allowed_overlap,
                                           a.isotropic.epsilon_shoulder)
            _check(_lib.hmc_set_shape_overlap(self._h, C.byref(prm)))
        elif hamiltonian is self.hamiltonian or (
                isinstance(pair, HardShape) and isinstance(self.hamiltonian.pair, HardShape)
                and type(pair.shape) is type(self.hamiltonian.pair.shape)
                and np.array_equal(np.asarray(pair.shape.vertices), np.asarray(self.hamiltonian.pair.shape.vertices))):
            _check(_lib.hmc_set_shape_overlap(self._h, None))
        else:
            raise HmcError(NOT_SUPPORTED, f"{type(pair).__name__} on a system of {type(self.hamiltonian.pair).__name__}")


class QuickInsert:
    """hoomd_mc::QuickInsert (quick_insert.rs:94-280) with the distribution UniformIn over the
    microstate's box and one site at the body origin; the microstate needs the capacity
    (Microstate(..., capacity=N))."""

    def __init__(self, target: int, allowed_overlaps: Optional[int] = None):
        self._s = hmc_quick_insert(int(target), max(int(target) // 8, 1) if allowed_overlaps is None
                                   else int(allowed_overlaps), 0, 0, 0)

    @classmethod
    def new(cls, target: int) -> "QuickInsert":
        return cls(target)

    @property
    def target(self) -> int:
        return self._s.target

    @property
    def inserted(self) -> int:
        return self._s.inserted

    def is_complete(self) -> bool:
        return bool(self._s.complete)

    def apply(self, microstate: Microstate, hamiltonian=None) -> Count:
        if hamiltonian is not None:
            microstate.set_hamiltonian(hamiltonian)
        c = hmc_count()
        _check(_lib.hmc_quick_insert_apply(microstate._h, C.byref(self._s), C.byref(c)))
        microstate.refresh()
        return Count(c.accepted, c.rejected, 0, 0, 0.0)


class QuickCompress:
    """hoomd_mc::QuickCompress (quick_compress.rs:88-383)."""

    STARTUP, WAITING, COMPRESSING, COMPLETE = range(4)

    def __init__(self, target_volume: float):
        self._s = hmc_quick_compress(float(target_volume), 1000.0, 0.05, self.STARTUP, 0)

    @classmethod
    def with_target_volume(cls, target_volume: float) -> "QuickCompress":
        return cls(target_volume)

    @property
    def target_volume(self) -> float:
        return self._s.target_volume

    def set_target_volume(self, target_volume: float):
        """set_target_volume (quick_compress.rs:215-240): Startup and Complete restart, Waiting
        forgets that it was final, Compressing continues."""
        if self._s.target_volume != target_volume:
            if self._s.state in (self.STARTUP, self.COMPLETE):
                self._s.state = self.STARTUP
            elif self._s.state == self.WAITING:
                self._s.is_final = 0
        self._s.target_volume = float(target_volume)

    @property
    def maximum_energy_per_site(self) -> float:
        return self._s.maximum_energy_per_site

    @maximum_energy_per_site.setter
    def maximum_energy_per_site(self, v: float):
        self._s.maximum_energy_per_site = float(v)

    @property
    def maximum_delta(self) -> float:
        return self._s.maximum_delta

    @maximum_delta.setter
    def maximum_delta(self, v: float):
        self._s.maximum_delta = float(v)

    @property
    def state(self) -> int:
        return self._s.state

    def is_complete(self) -> bool:
        return self._s.state == self.COMPLETE

    def apply(self, microstate: Microstate, hamiltonian=None):
        if hamiltonian is not None:
            microstate.set_hamiltonian(hamiltonian)
        _check(_lib.hmc_quick_compress_apply(microstate._h, C.byref(self._s)))
        microstate.edge_lengths = [float(x) for x in microstate.box()]


def place_single_site_point_bodies(ctx: "Context", n: int, number_density: float, maximum_interaction_range: float,
                                   overlap_penalty_hamiltonian: PairwiseCutoff, dim: int, *, seed: int = 0,
                                   max_steps: int = 1_000_000) -> "Microstate":
    """place_single_site_point_bodies (benchmarks/src/place.rs:31-110): an empty periodic box at
    0.7 times the number density, QuickInsert of n bodies, then QuickCompress to the target
    density (either every 20 steps), and a serial translation Sweep (0.1, kT = 1) every step, all
    under the overlap-penalty hamiltonian. Returns that microstate; its positions start a system of
    the hard hamiltonian."""
    initial_box_length = (n / (0.7 * number_density)) ** (1.0 / dim)
    final_box_volume = n / number_density
    g = Microstate(ctx, Periodic(maximum_interaction_range, [initial_box_length] * dim), np.zeros((0, dim)),
                   overlap_penalty_hamiltonian, seed=seed, capacity=n)
    quick_insert = QuickInsert.new(n)
    quick_compress = QuickCompress.with_target_volume(final_box_volume)
    for _ in range(max_steps):
        if quick_compress.is_complete():
            break
        if g.step() % 20 == 0:
            if quick_insert.is_complete():
                quick_compress.apply(g)
            else:
                quick_insert.apply(g)
        g.serial_sweep(0.1)
        g.increment_step()
    else:
        raise HmcError(ITERATION_CAP, f"QuickCompress did not complete in {max_steps} steps")
    return g


def place_single_site_orientable_bodies(ctx: "Context", n: int, number_density: float,
                                        maximum_interaction_range: float, insert_hamiltonian: PairwiseCutoff,
                                        hamiltonian: PairwiseCutoff, dim: int, *, seed: int = 0,
                                        max_steps: int = 1_000_000) -> "Microstate":
    """place_single_site_orientable_bodies (benchmarks/src/place.rs:120-219): an empty periodic
    box at half the number density, QuickInsert of n bodies, then QuickCompress to the target
    density (either every 10 steps), a translation (0.03) and a rotation (0.1) ParallelSweep every
    step, all under insert_hamiltonian (PairwiseCutoff(Anisotropic(ApproximateShapeOverlap))) at
    kT = 1. Returns the microstate under `hamiltonian` (its HardShape)."""
    initial_box_length = (n / (0.5 * number_density)) ** (1.0 / dim)
    final_box_volume = n / number_density
    g = Microstate(ctx, Periodic(maximum_interaction_range, [initial_box_length] * dim), np.zeros((0, dim)),
                   hamiltonian, seed=seed, capacity=n,
                   body_interaction_range=insert_hamiltonian.maximum_interaction_range)
    g.set_hamiltonian(insert_hamiltonian)
    quick_insert = QuickInsert.new(n)
    quick_compress = QuickCompress.with_target_volume(final_box_volume)
    for _ in range(max_steps):
        if quick_compress.is_complete():
            break
        if g.step() % 10 == 0:
            if quick_insert.is_complete():
                quick_compress.apply(g)
            else:
                quick_insert.apply(g)
        g.sweep(TRANSLATE, 0.03, 1.0, FP64)
        g.sweep(ROTATE, 0.1, 1.0, FP64)
        g.increment_step()
    else:
        raise HmcError(ITERATION_CAP, f"QuickCompress did not complete in {max_steps} steps")
    g.set_hamiltonian(hamiltonian)
    return g


@dataclass
class IsothermalIsofugacity:
    """hoomd_simulation::macrostate::IsothermalIsofugacity: temperature and fugacity."""
    temperature: float = 1.0
    fugacity: float = 0.0


@dataclass
class InsertRemoveCount:
    """hoomd_mc::InsertRemoveCount (grand_canonical.rs)."""
    insert_accepted: int = 0
    insert_rejected: int = 0
    remove_accepted: int = 0
    remove_rejected: int = 0


class GrandCanonical:
    """hoomd_mc::GrandCanonical (grand_canonical.rs:49-110) with the distribution UniformIn over
    the microstate's box; apply(..., n_trials=k) runs k applies in sequence on the device."""

    def apply(self, microstate: Microstate, hamiltonian, macrostate: IsothermalIsofugacity,
              n_trials: int = 1) -> InsertRemoveCount:
        p = hmc_grand_canonical_params(float(macrostate.temperature), float(macrostate.fugacity), int(n_trials), 0)
        c = hmc_insert_remove_count()
        _check(_lib.hmc_grand_canonical_apply(microstate._h, C.byref(p), C.byref(c)))
        microstate.refresh()
        return InsertRemoveCount(c.insert_accepted, c.insert_rejected, c.remove_accepted, c.remove_rejected)


class Batch:
    """Independent replicas swept together (hmc_batch_*): one counting sort and one kernel per
    colour pass for all replicas. Replica k evolves exactly as a Microstate built from the same
    (boundary, positions, hamiltonian, seed, step, substep) would. All replicas hold hard spheres,
    or all hold Lennard-Jones bodies (each replica with its own parameters and temperature)."""

    def __init__(self, ctx: Context, replicas):
        """replicas: dicts with keys boundary (Periodic), positions, seed, step, substep (default
        0), and either diameter (hard spheres, default 1) or hamiltonian (PairwiseCutoff of
        HardSphere or of Isotropic(Shifted(LennardJones)))."""
        lib = load_library()
        self.n_replicas = len(replicas)
        descs = (hmc_system_desc * self.n_replicas)()
        self._pos = []
        self.dim = len(replicas[0]["boundary"].edge_lengths)
        self.sizes = []
        self.edge_lengths = []
        for k, r in enumerate(replicas):
            L = [float(x) for x in r["boundary"].edge_lengths]
            self.edge_lengths.append(L)
            pos = np.ascontiguousarray(r["positions"], dtype=np.float64).reshape(-1, len(L))
            self._pos.append(pos)
            self.sizes.append(pos.shape[0])
            d = descs[k]
            d.struct_size = C.sizeof(hmc_system_desc)
            d.dim = len(L)
            for a, x in enumerate(L):
                d.edge_lengths[a] = x
            d.n_bodies = pos.shape[0]
            d.step, d.substep, d.seed = r.get("step", 0), r.get("substep", 0), r.get("seed", 0)
            ham = r.get("hamiltonian")
            pair = None if ham is None else ham.pair
            if pair is None or isinstance(pair, HardSphere):
                d.interaction = HARD_SPHERE
                d.diameter = r.get("diameter", 1.0) if pair is None else pair.diameter
            elif isinstance(pair, Isotropic) and isinstance(pair.interaction, Shifted):
                d.interaction = LENNARD_JONES
                d.lj_epsilon = pair.interaction.f.epsilon
                d.lj_sigma = pair.interaction.f.sigma
                d.lj_r_cut = pair.r_cut
                d.lj_r_shift = pair.interaction.r_shift
            else:
                raise HmcError(NOT_SUPPORTED, f"batches of {type(pair).__name__}")
            d.boundary_range = r["boundary"].maximum_interaction_range
        ptrs = (_dp * self.n_replicas)(*[p.ctypes.data_as(_dp) for p in self._pos])
        h = _vp()
        _check(lib.hmc_batch_create(ctx._h, self.n_replicas, descs, ptrs, C.byref(h)))
        self._h = h
        self.ctx = ctx

    def sweep(self, maxima, precision: int = FP32_RECHECK, n_sweeps: int = 1, increment_step: bool = False,
              temperatures=1.0):
        """ParallelSweep::apply on every replica (replica k moves up to maxima[k] at kT =
        temperatures[k]); returns (per-replica Counts, batch total Count)."""
        # the per-replica parameters and counts as arrays of the C structs, filled without a Python
        # loop over the replicas (the batch's step would otherwise wait for it)
        ps = np.zeros(self.n_replicas, dtype=_SWEEP_PARAMS_DTYPE)
        ps["struct_size"] = C.sizeof(hmc_sweep_params)
        ps["move"] = TRANSLATE
        ps["maximum"] = maxima
        ps["temperature"] = temperatures
        ps["precision"] = precision
        ps["n_sweeps"] = n_sweeps
        ps["increment_step"] = int(increment_step)
        cs = np.zeros(self.n_replicas, dtype=_COUNT_DTYPE)
        tot = hmc_count()
        _check(_lib.hmc_batch_sweep(self._h, ps.ctypes.data_as(C.POINTER(hmc_sweep_params)),
                                    cs.ctypes.data_as(C.POINTER(hmc_count)), C.byref(tot)))
        counts = [Count(int(a), int(r), 0, 0, 0.0) for a, r in zip(cs["accepted"].tolist(), cs["rejected"].tolist())]
        return counts, Count(tot.accepted, tot.rejected, tot.rechecks, tot.pair_checks, tot.max_fp32_error,
                             tot.order_ambiguous)

    def state(self, k: int):
        pos = np.empty((self.sizes[k], self.dim))
        step = C.c_uint64()
        sub = C.c_uint32()
        _check(_lib.hmc_batch_get_state(self._h, k, pos.ctypes.data_as(_dp), C.byref(step), C.byref(sub)))
        return pos, step.value, sub.value

    def positions(self, k: int) -> np.ndarray:
        return self.state(k)[0]

    def set_state(self, k: int, positions, step: int, substep: int):
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(self.sizes[k], self.dim)
        _check(_lib.hmc_batch_set_state(self._h, k, pos.ctypes.data_as(_dp), step, substep))

    def overlap_counts(self) -> np.ndarray:
        out = np.zeros(self.n_replicas, dtype=np.uint64)
        _check(_lib.hmc_batch_overlap_check(self._h, out.ctypes.data_as(C.POINTER(C.c_uint64))))
        return out

    def tune(self, maxima, precision: int, target: float, samples: int, steps: int, temperatures=1.0,
             per_sample_streams: bool = False) -> np.ndarray:
        """Tune every replica's translation size towards the target acceptance (Microstate.tune on
        each replica's state); returns the tuned maxima."""
        maxima = np.broadcast_to(np.asarray(maxima, dtype=np.float64), (self.n_replicas,))
        kts = np.broadcast_to(np.asarray(temperatures, dtype=np.float64), (self.n_replicas,))
        ps = (hmc_sweep_params * self.n_replicas)()
        flags = TUNE_PER_SAMPLE_STREAMS if per_sample_streams else 0
        for k in range(self.n_replicas):
            ps[k] = hmc_sweep_params(C.sizeof(hmc_sweep_params), TRANSLATE, float(maxima[k]), float(kts[k]), precision,
                                     1, 0, flags)
        _check(_lib.hmc_batch_tune(self._h, ps, target, samples, steps))
        return np.array([ps[k].maximum for k in range(self.n_replicas)])

    def autotune(self, maxima, precision: int, sweeps: int = 3, temperatures=1.0):
        """hmc_batch_autotune: the fastest launch variant of the replica pass, from the current
        state (restored after); returns (chosen variant, ms per sweep per variant)."""
        maxima = np.broadcast_to(np.asarray(maxima, dtype=np.float64), (self.n_replicas,))
        kts = np.broadcast_to(np.asarray(temperatures, dtype=np.float64), (self.n_replicas,))
        ps = (hmc_sweep_params * self.n_replicas)()
        for k in range(self.n_replicas):
            ps[k] = hmc_sweep_params(C.sizeof(hmc_sweep_params), TRANSLATE, float(maxima[k]), float(kts[k]), precision,
                                     1, 1, 0)
        v = hmc_launch_variant()
        ms = np.zeros(16)
        _check(_lib.hmc_batch_autotune(self._h, ps, sweeps, C.byref(v), ms.ctypes.data_as(_dp)))
        return {f: getattr(v, f) for f, _ in hmc_launch_variant._fields_}, ms[: v.count].copy()

    def set_launch_variant(self, precision: int, index: Optional[int]):
        _check(_lib.hmc_batch_set_launch_variant(self._h, precision, 0xFFFFFFFF if index is None else index))

    def set_captured_sweeps(self, enable: bool = True):
        """hmc_batch_set_captured_sweeps: each sweep as one CUDA-graph launch, the sweeps of a call
        back to back with one wait at the end (same trajectory as the launched sweeps)."""
        _check(_lib.hmc_batch_set_captured_sweeps(self._h, 1 if enable else 0))

    def sdf(self, x_max: float = 0.02, n_bins: int = 40) -> np.ndarray:
        """Scale distributions of all replicas (hard spheres): (n_replicas, n_bins) pair counts."""
        out = np.zeros((self.n_replicas, n_bins), dtype=np.uint64)
        _check(_lib.hmc_batch_sdf(self._h, x_max, n_bins, out.ctypes.data_as(C.POINTER(C.c_uint64))))
        return out

    def pressures(self, x_max: float = 0.02, n_bins: int = 40, fit_bins: int = 12) -> np.ndarray:
        """beta P of every replica from its scale distribution (Microstate.pressure's estimator)."""
        counts = self.sdf(x_max, n_bins)
        return np.array([sdf_pressure(counts[k], self.sizes[k], float(np.prod(self.edge_lengths[k])), self.dim, x_max,
                                      fit_bins) for k in range(self.n_replicas)])

    def kernel_launches(self) -> int:
        return int(_lib.hmc_batch_kernel_launches(self._h))

    def close(self):
        if getattr(self, "_h", None):
            _lib.hmc_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


@dataclass
class TuneOptions:
    """hoomd_mc::TuneOptions (lib.rs:394-412)."""
    target_acceptance: float = 0.2
    samples: int = 8000
    steps: int = 32


class ParallelSweep:
    """hoomd_mc::ParallelSweep (parallel_sweep.rs:83-421) executed on the GPU.

    ``precision`` selects the plain FP64 pair test (``FP64``) or the FP32 test with FP64
    recheck inside the forward-error bound (``FP32_RECHECK``); both give the same decisions.
    """

    def __init__(self, body_interaction_range: float, local_trial, precision: int = FP32_RECHECK):
        self.body_interaction_range = float(body_interaction_range)
        self.local_trial = local_trial
        self.precision = precision
        self.last_count: Optional[Count] = None

    def apply(self, microstate: Microstate, hamiltonian: PairwiseCutoff, macrostate: Isothermal) -> Count:
        if hamiltonian is not microstate.hamiltonian and hamiltonian != microstate.hamiltonian:
            raise HmcError(INVALID_ARGUMENT, "the hamiltonian differs from the one the microstate was built with")
        if isinstance(self.local_trial, Translate):
            move, maximum = TRANSLATE, self.local_trial.maximum_distance
        elif isinstance(self.local_trial, Rotate):
            move, maximum = ROTATE, self.local_trial.maximum_rotation
        else:
            raise HmcError(NOT_SUPPORTED, type(self.local_trial).__name__)
        c = microstate.sweep(move, maximum, macrostate.temperature, self.precision)
        self.last_count = c
        return c

    def tune_with_options(self, microstate: "Microstate", hamiltonian: PairwiseCutoff, macrostate: Isothermal,
                          options: TuneOptions = TuneOptions()) -> None:
        """Tune::tune_with_options (lib.rs:430-449): rescales the local trial's maximum."""
        if isinstance(self.local_trial, Translate):
            move, maximum = TRANSLATE, self.local_trial.maximum_distance
        else:
            move, maximum = ROTATE, self.local_trial.maximum_rotation
        tuned = microstate.tune(move, maximum, macrostate.temperature, self.precision, options.target_acceptance,
                                options.samples, options.steps)
        if isinstance(self.local_trial, Translate):
            self.local_trial.maximum_distance = tuned
        else:
            self.local_trial.maximum_rotation = tuned


__all__ = ["Batch", "Context", "sdf_pressure", "gr_normalise", "ConvexPolygon", "ConvexPolyhedron", "ConvexSurfaceMesh2d", "Count", "convex_hull_2d", "HardShape", "HardSphere", "HmcError", "Isothermal", "Isotropic",
           "LennardJones", "Microstate", "PairwiseCutoff", "Rotate", "Shifted", "TuneOptions",
           "ParallelSweep", "Periodic", "Translate", "load_library", "SIGNATURES", "FP64", "FP32_RECHECK",
           "QuickInsert", "QuickCompress", "OverlapPenalty", "ApproximateShapeOverlap", "Anisotropic",
           "WeeksChandlerAnderson", "Harmonic", "HarmonicRepulsion", "Boxcar", "Xplor", "LennardJonesGauss",
           "place_single_site_orientable_bodies", "place_single_site_point_bodies", "Expanded", "GrandCanonical", "IsothermalIsofugacity",
           "InsertRemoveCount",
           "TRANSLATE", "ROTATE", "HARD_SPHERE", "HARD_CONVEX_POLYGON", "HARD_CONVEX_POLYHEDRON", "LENNARD_JONES",
           "HARD_CONVEX_SURFACE_MESH_2D"]
