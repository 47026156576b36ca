"""ctypes bindings for the CPU oracle (test infrastructure only).

The oracle is a plain FP64 C++ restatement of the reference's Monte Carlo sweep
(glotzerlab/hoomd-rs v1.4.0, ``hoomd-mc``), built by ``oracle/Makefile`` into
``oracle/liboracle.so``. Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` load it; it is the checker, never the product.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

HARD_SPHERE = 0
HARD_CONVEX_POLYGON = 1
HARD_CONVEX_POLYHEDRON = 2
LENNARD_JONES = 3
HARD_CONVEX_SURFACE_MESH_2D = 4
OVERLAP_PENALTY = 5
CONVEX_POLYHEDRON_PENALTY = 6  # Anisotropic { ApproximateShapeOverlap { Convex(ConvexPolyhedron), OverlapPenalty } }
CONVEX_POLYGON_PENALTY = 7     # the same with Convex(ConvexPolygon)
ISOTROPIC = 8                  # Isotropic { W(F), r_cut }: F and W below
SURFACE_MESH_2D_PENALTY = 9    # ApproximateShapeOverlap with ConvexSurfaceMesh2d (separating axes)
UV_LENNARD_JONES, UV_WEEKS_CHANDLER_ANDERSON, UV_HARMONIC, UV_HARMONIC_REPULSION, UV_BOXCAR, UV_OVERLAP_PENALTY, \
    UV_LENNARD_JONES_GAUSS = range(7)
UVW_NONE, UVW_SHIFTED, UVW_EXPANDED, UVW_XPLOR = range(4)
TRANSLATE = 0
ROTATE = 1

_dp = C.POINTER(C.c_double)
_u64p = C.POINTER(C.c_uint64)
_u8p = C.POINTER(C.c_uint8)
_u32p = C.POINTER(C.c_uint32)


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.oracle_sfc64_outputs.argtypes = [C.c_uint64] * 6 + [_u64p]
        L.oracle_sfc64_seed_from_u64.argtypes = [C.c_uint64] * 3 + [_u64p]
        L.oracle_counter_outputs.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64, _u64p]
        L.oracle_counter_uniforms.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64, _dp]
        L.oracle_counter_normals.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64, _dp]
        L.oracle_counter_ball.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32,
                                          C.c_double, C.c_uint64, _dp]
        L.oracle_counter_choose.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32]
        L.oracle_counter_choose.restype = C.c_uint32
        L.oracle_cbrt.argtypes = [C.c_double]
        L.oracle_cbrt.restype = C.c_double
        L.oracle_sincos_half.argtypes = [C.c_double, _dp, _dp]
        L.oracle_ziggurat_tables.argtypes = [_dp, _dp]
        L.oracle_wrap.argtypes = [C.c_uint32, _dp, _dp]
        L.oracle_generate_ghosts.argtypes = [C.c_uint32, _dp, C.c_double, _dp, _dp]
        L.oracle_generate_ghosts.restype = C.c_uint32
        L.oracle_checkerboard_dimensions.argtypes = [C.c_uint32, _dp, C.c_double, C.c_int, _dp, _u64p]
        L.oracle_checkerboard_dimensions.restype = C.c_int
        L.oracle_point_to_space_index.argtypes = [C.c_uint32, _dp, _dp, _u64p, C.c_int, _dp]
        L.oracle_point_to_space_index.restype = C.c_int64
        L.oracle_space_indices_by_color.argtypes = [C.c_uint32, _u64p, _u64p]
        L.oracle_checkerboard_for_counter.argtypes = [C.c_uint32, _dp, C.c_double, C.c_uint64, C.c_uint32,
                                                      C.c_uint32, _dp, _dp, _u64p]
        L.oracle_checkerboard_for_counter.restype = C.c_int
        L.oracle_convex_intersects_at_3d.argtypes = [_dp, C.c_uint32, _dp, C.c_uint32, _dp, _dp]
        L.oracle_convex_intersects_at_2d.argtypes = [_dp, C.c_uint32, _dp, C.c_uint32, _dp, C.c_double]
        L.oracle_surface_mesh_intersects_at_2d.argtypes = [_dp, C.c_uint32, _dp, C.c_uint32, _dp, C.c_double]
        L.oracle_cr_sincos.argtypes = [C.c_double, _dp, _dp]
        L.oracle_cr_sincos.restype = C.c_int
        L.oracle_convex_intersects_at_global_3d.argtypes = [_dp, C.c_uint32, _dp, _dp, _dp, _dp]
        L.oracle_versor_from_axis_angle.argtypes = [_dp, C.c_double, _dp]
        L.oracle_versor_combine.argtypes = [_dp, _dp, _dp]
        L.oracle_versor_rotate.argtypes = [_dp, _dp, _dp]
        L.oracle_lj_energy.argtypes = [C.c_double] * 3
        L.oracle_lj_energy.restype = C.c_double
        L.oracle_shifted_lj_pair.argtypes = [C.c_double] * 5
        L.oracle_shifted_lj_pair.restype = C.c_double
        L.oracle_system_create.argtypes = [C.c_uint32, _dp, C.c_uint64, _dp, _dp, C.c_uint64, C.c_uint32,
                                           C.c_uint32, C.c_uint32, C.c_double, _dp, C.c_uint32, C.c_double,
                                           C.c_double, C.c_double, C.c_double, C.c_double]
        L.oracle_system_create.restype = C.c_void_p
        L.oracle_system_destroy.argtypes = [C.c_void_p]
        L.oracle_get_state.argtypes = [C.c_void_p, _dp, _dp, _u64p, _u32p]
        L.oracle_set_counter.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32]
        L.oracle_gsd_frame.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_set_penalty.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double]
        L.oracle_set_shape_overlap.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.oracle_set_isotropic.argtypes = [C.c_void_p, C.c_uint32, _dp, C.c_uint32, _dp, C.c_double]
        L.oracle_univariate_energy.argtypes = [C.c_uint32, _dp, C.c_uint32, _dp, C.c_double]
        L.oracle_univariate_energy.restype = C.c_double
        L.oracle_approximate_separation.argtypes = [C.c_uint32, _dp, C.c_uint32, _dp, _dp, C.c_double, C.c_uint32]
        L.oracle_approximate_separation.restype = C.c_double
        L.oracle_n_bodies.argtypes = [C.c_void_p]
        L.oracle_n_bodies.restype = C.c_uint64
        L.oracle_get_box.argtypes = [C.c_void_p, _dp]
        L.oracle_set_box.argtypes = [C.c_void_p, _dp]
        L.oracle_set_box.restype = C.c_int
        L.oracle_quick_insert.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, _u64p, _u32p, _u64p, _u64p]
        L.oracle_quick_compress.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, _u32p, _u32p, _dp]
        L.oracle_quick_compress.restype = C.c_int
        L.oracle_grand_canonical.argtypes = [C.c_void_p, C.c_double, C.c_double, _u64p]
        L.oracle_increment_step.argtypes = [C.c_void_p]
        L.oracle_parallel_sweep.argtypes = [C.c_void_p, C.c_uint32, C.c_double, C.c_double, C.c_double,
                                            _u64p, _u64p]
        L.oracle_parallel_sweep.restype = C.c_int
        L.oracle_parallel_sweep_threads.argtypes = [C.c_void_p, C.c_uint32, C.c_double, C.c_double, C.c_double,
                                                    C.c_uint32, _u64p, _u64p]
        L.oracle_parallel_sweep_threads.restype = C.c_int
        L.oracle_serial_sweep_filter.argtypes = [C.c_void_p, C.c_uint32, C.c_double, C.c_double, _u8p, _u64p,
                                                 _u64p]
        L.oracle_serial_sweep_filter.restype = C.c_int
        L.oracle_serial_sweep.argtypes = [C.c_void_p, C.c_uint32, C.c_double, C.c_double, _u64p, _u64p]
        L.oracle_serial_sweep.restype = C.c_int
        L.oracle_tune.argtypes = [C.c_void_p, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_uint32, C.c_uint32]
        L.oracle_tune.restype = C.c_double
        L.oracle_tune_stream.argtypes = [C.c_void_p, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_uint32,
                                         C.c_uint32]
        L.oracle_tune_stream.restype = C.c_double
        L.oracle_sample_moves.argtypes = [C.c_uint32, C.c_uint32, C.c_double, C.c_uint64, C.c_uint32, C.c_uint32,
                                          C.c_uint64, C.POINTER(C.c_double)]
        L.oracle_sample_moves.restype = None
        L.oracle_sdf.argtypes = [C.c_void_p, C.c_double, C.c_uint32, _u64p]
        L.oracle_gr.argtypes = [C.c_void_p, C.c_double, C.c_uint32, _u64p]
        L.oracle_overlap_count.argtypes = [C.c_void_p]
        L.oracle_overlap_count.restype = C.c_uint64
        L.oracle_total_energy.argtypes = [C.c_void_p]
        L.oracle_total_energy.restype = C.c_double
        L.oracle_delta_energy_one.argtypes = [C.c_void_p, C.c_uint64, _dp, _dp]
        L.oracle_delta_energy_one.restype = C.c_double
        L.oracle_eval_moves.argtypes = [C.c_void_p, C.c_uint64, _u64p, _dp, _dp, _dp, C.c_double, _u8p, _dp]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a if shape is None else a.reshape(shape)


# ---- random numbers ---------------------------------------------------------------
def sfc64_seed_from_u64(state: int, n: int, skip: int = 0) -> np.ndarray:
    out = np.zeros(n, dtype=np.uint64)
    lib().oracle_sfc64_seed_from_u64(state, skip, n, out.ctypes.data_as(_u64p))
    return out


def counter_outputs(step, substep, seed, index, n):
    out = np.zeros(n, dtype=np.uint64)
    lib().oracle_counter_outputs(step, substep, seed, index, n, out.ctypes.data_as(_u64p))
    return out


def counter_uniforms(step, substep, seed, index, n):
    out = np.zeros(n)
    lib().oracle_counter_uniforms(step, substep, seed, index, n, _d(out))
    return out


def counter_normals(step, substep, seed, index, n):
    out = np.zeros(n)
    lib().oracle_counter_normals(step, substep, seed, index, n, _d(out))
    return out


def counter_ball(step, substep, seed, index, dim, radius, n):
    out = np.zeros((n, dim))
    lib().oracle_counter_ball(step, substep, seed, index, dim, radius, n, _d(out))
    return out


def sample_moves(dim, kind, maximum, n, step=0, substep=0, seed=0) -> np.ndarray:
    """The samplers for a body at the origin, sample i from Counter(step, substep, seed).index(i)
    (kind 0 translate, 1 rotate, 2 standard normal), shaped like Context.sample_moves."""
    per = 1 if kind == 2 else (dim if kind == 0 else (4 if dim == 3 else 1))
    out = np.empty(n * per)
    lib().oracle_sample_moves(dim, kind, maximum, step, substep, seed, n, _d(out))
    return out.reshape(n, per) if per > 1 else out


def cbrt(x: float) -> float:
    return lib().oracle_cbrt(x)


def ziggurat_tables():
    x = np.zeros(257)
    f = np.zeros(257)
    lib().oracle_ziggurat_tables(_d(x), _d(f))
    return x, f


# ---- boundary / checkerboard ------------------------------------------------------
def wrap(point, edge_lengths):
    p = _f64(point).copy()
    L = _f64(edge_lengths)
    lib().oracle_wrap(len(L), _d(L), _d(p))
    return p


def generate_ghosts(point, edge_lengths, rng):
    L = _f64(edge_lengths)
    p = _f64(point)
    out = np.zeros(7 * len(L))
    n = lib().oracle_generate_ghosts(len(L), _d(L), rng, _d(p), _d(out))
    return out[: n * len(L)].reshape(n, len(L))


def checkerboard_dimensions(edge_lengths, rng, periodic):
    L = _f64(edge_lengths)
    w = np.zeros(len(L))
    s = np.zeros(len(L), dtype=np.uint64)
    rc = lib().oracle_checkerboard_dimensions(len(L), _d(L), rng, int(periodic), _d(w), s.ctypes.data_as(_u64p))
    if rc:
        raise ValueError("interaction range too large for the boundary")
    return w, s


def point_to_space_index(origin, width, shape, periodic, point):
    o = _f64(origin)
    w = _f64(width)
    s = np.ascontiguousarray(shape, dtype=np.uint64)
    p = _f64(point)
    r = lib().oracle_point_to_space_index(len(o), _d(o), _d(w), s.ctypes.data_as(_u64p), int(periodic), _d(p))
    return None if r < 0 else int(r)


def space_indices_by_color(shape):
    s = np.ascontiguousarray(shape, dtype=np.uint64)
    total = int(np.prod(s))
    out = np.zeros(total, dtype=np.uint64)
    lib().oracle_space_indices_by_color(len(s), s.ctypes.data_as(_u64p), out.ctypes.data_as(_u64p))
    return out.reshape(2 ** len(s), -1)


def checkerboard_for_counter(edge_lengths, rng, step, substep, seed):
    L = _f64(edge_lengths)
    o = np.zeros(len(L))
    w = np.zeros(len(L))
    s = np.zeros(len(L), dtype=np.uint64)
    rc = lib().oracle_checkerboard_for_counter(len(L), _d(L), rng, step, substep, seed, _d(o), _d(w),
                                               s.ctypes.data_as(_u64p))
    if rc:
        raise ValueError("interaction range too large for the boundary")
    return o, w, s


# ---- geometry / potentials --------------------------------------------------------
def convex_intersects_at_3d(verts_a, verts_b, v_ij, q_ij) -> bool:
    a = _f64(verts_a)
    b = _f64(verts_b)
    v = _f64(v_ij)
    q = _f64(q_ij)
    return bool(lib().oracle_convex_intersects_at_3d(_d(a), len(a) // 3 if a.ndim == 1 else a.shape[0], _d(b),
                                                     len(b) // 3 if b.ndim == 1 else b.shape[0], _d(v), _d(q)))


def convex_intersects_at_2d(verts_a, verts_b, v_ij, theta) -> bool:
    a = _f64(verts_a)
    b = _f64(verts_b)
    v = _f64(v_ij)
    return bool(lib().oracle_convex_intersects_at_2d(_d(a), a.shape[0], _d(b), b.shape[0], _d(v), theta))


def surface_mesh_intersects_at_2d(verts_a, verts_b, v_ij, theta) -> bool:
    a = _f64(verts_a, (-1, 2))
    b = _f64(verts_b, (-1, 2))
    v = _f64(v_ij)
    return bool(lib().oracle_surface_mesh_intersects_at_2d(_d(a), a.shape[0], _d(b), b.shape[0], _d(v), theta))


def approximate_separation(vertices, v_ij, o_ij, resolution, sat=False) -> float:
    """IntersectsAt::approximate_separation_distance of two equal convex polytopes; o_ij is a versor
    (s, x, y, z) in 3-D or an angle in 2-D; sat: ConvexSurfaceMesh2d polygons."""
    verts = _f64(vertices)
    dim = verts.shape[1]
    return float(lib().oracle_approximate_separation(dim, _d(verts), verts.shape[0], _d(_f64(v_ij)),
                                                     _d(_f64(np.atleast_1d(o_ij))), resolution, int(sat)))


def _params(p, n):
    a = np.zeros(n)
    a[:len(p)] = p
    return a


def univariate_energy(kind, params, r, wrap=UVW_NONE, wrap_params=()) -> float:
    """W(F).energy(r) for a univariate F (UV_*) with parameters `params` and a wrapper W (UVW_*)."""
    return float(lib().oracle_univariate_energy(kind, _d(_params(params, 4)), wrap, _d(_params(wrap_params, 2)), r))


def cr_sincos(x: float):
    """Correctly rounded (sin x, cos x); raises for |x| >= 2^20."""
    s = C.c_double()
    c = C.c_double()
    if lib().oracle_cr_sincos(x, C.byref(s), C.byref(c)):
        raise ValueError("|x| >= 2^20")
    return s.value, c.value


def versor_from_axis_angle(axis, angle):
    a = _f64(axis)
    q = np.zeros(4)
    lib().oracle_versor_from_axis_angle(_d(a), angle, _d(q))
    return q


def versor_combine(a, b):
    a = _f64(a)
    b = _f64(b)
    o = np.zeros(4)
    lib().oracle_versor_combine(_d(a), _d(b), _d(o))
    return o


def versor_rotate(q, v):
    q = _f64(q)
    v = _f64(v)
    o = np.zeros(3)
    lib().oracle_versor_rotate(_d(q), _d(v), _d(o))
    return o


def lj_energy(epsilon, sigma, r):
    return lib().oracle_lj_energy(epsilon, sigma, r)


def shifted_lj_pair(epsilon, sigma, r_cut, r_shift, r_squared):
    return lib().oracle_shifted_lj_pair(epsilon, sigma, r_cut, r_shift, r_squared)


# ---- systems -------------------------------------------------------------------
class System:
    """An oracle microstate: bodies in a periodic box with one pair interaction."""

    def __init__(self, dim, edge_lengths, positions, orientations=None, *, step=0, substep=0, seed=0,
                 interaction=HARD_SPHERE, diameter=1.0, vertices=None, lj_epsilon=1.0, lj_sigma=1.0,
                 lj_r_cut=2.5, lj_r_shift=2.5, boundary_range=None, penalty=(10000.0, 0.2, 100.0),
                 resolution=0.01, r_cut=None, isotropic=None):
        self.dim = dim
        self.L = _f64(edge_lengths)
        self.seed = seed
        pos = _f64(positions, (-1,))
        self.n = pos.size // dim
        self.interaction = interaction
        ori = None if orientations is None else _f64(orientations, (-1,))
        verts = None if vertices is None else _f64(vertices, (-1,))
        nv = 0 if verts is None else verts.size // dim
        if boundary_range is None and interaction == ISOTROPIC:
            boundary_range = isotropic["r_cut"]
        if boundary_range is None:
            if interaction in (HARD_SPHERE, OVERLAP_PENALTY):
                boundary_range = diameter
            elif interaction == LENNARD_JONES:
                boundary_range = lj_r_cut
            else:
                boundary_range = 2.0 * float(np.sqrt(np.max(np.sum(verts.reshape(nv, dim) ** 2, axis=1))))
        self.boundary_range = boundary_range
        self._h = lib().oracle_system_create(dim, _d(self.L), self.n, _d(pos), _d(ori), step, substep, seed,
                                             interaction, diameter, _d(verts), nv, lj_epsilon, lj_sigma,
                                             lj_r_cut, lj_r_shift, boundary_range)
        self.ori_len = 0 if interaction in (HARD_SPHERE, LENNARD_JONES, OVERLAP_PENALTY, ISOTROPIC) else \
            (4 if dim == 3 else 1)
        if interaction == ISOTROPIC:
            # isotropic = {"kind", "params", "wrap", "wrap_params", "r_cut"}
            lib().oracle_set_isotropic(self._h, isotropic["kind"], _d(_params(isotropic["params"], 4)),
                                       isotropic.get("wrap", UVW_NONE), _d(_params(isotropic.get("wrap_params", ()), 2)),
                                       isotropic["r_cut"])
        if interaction in (OVERLAP_PENALTY, CONVEX_POLYHEDRON_PENALTY, CONVEX_POLYGON_PENALTY, SURFACE_MESH_2D_PENALTY):
            lib().oracle_set_penalty(self._h, *penalty)
        if interaction in (CONVEX_POLYHEDRON_PENALTY, CONVEX_POLYGON_PENALTY, SURFACE_MESH_2D_PENALTY):
            lib().oracle_set_shape_overlap(self._h, resolution, boundary_range if r_cut is None else r_cut)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().oracle_system_destroy(h)
            self._h = None

    def state(self):
        pos = np.zeros((self.n, self.dim))
        ori = np.zeros((self.n, self.ori_len)) if self.ori_len else None
        step = C.c_uint64()
        sub = C.c_uint32()
        lib().oracle_get_state(self._h, _d(pos), _d(ori), C.byref(step), C.byref(sub))
        return pos, ori, step.value, sub.value

    def set_counter(self, step, substep):
        lib().oracle_set_counter(self._h, step, substep)

    @property
    def n_bodies(self) -> int:
        return int(lib().oracle_n_bodies(self._h))

    def box(self):
        L = np.zeros(self.dim)
        lib().oracle_get_box(self._h, _d(L))
        return L

    def set_box(self, edge_lengths):
        L = _f64(edge_lengths)
        if lib().oracle_set_box(self._h, _d(L)) != 0:
            raise ValueError("a body is outside the box")
        self.L = L

    def quick_insert(self, state: dict):
        """QuickInsert::apply; state holds target, allowed_overlaps, inserted, complete."""
        ins, comp = C.c_uint64(state["inserted"]), C.c_uint32(state["complete"])
        a, r = C.c_uint64(), C.c_uint64()
        lib().oracle_quick_insert(self._h, state["target"], state["allowed_overlaps"], C.byref(ins), C.byref(comp),
                                  C.byref(a), C.byref(r))
        state["inserted"], state["complete"] = ins.value, comp.value
        self.n = self.n_bodies
        return a.value, r.value

    def grand_canonical(self, temperature, fugacity, n_trials=1):
        """GrandCanonical::apply n_trials times: (insert accepted, insert rejected, remove
        accepted, remove rejected)."""
        c = np.zeros(4, dtype=np.uint64)
        for _ in range(n_trials):
            lib().oracle_grand_canonical(self._h, temperature, fugacity, c.ctypes.data_as(_u64p))
        self.n = self.n_bodies
        return tuple(int(x) for x in c)

    def quick_compress(self, state: dict):
        """QuickCompress::apply; state holds target_volume, maximum_energy_per_site, maximum_delta,
        state, is_final, boundary."""
        st, fin = C.c_uint32(state["state"]), C.c_uint32(state["is_final"])
        b = np.array(list(state["boundary"]) + [0.0] * (3 - len(state["boundary"])), dtype=np.float64)
        rc = lib().oracle_quick_compress(self._h, state["target_volume"], state["maximum_energy_per_site"],
                                         state["maximum_delta"], C.byref(st), C.byref(fin), _d(b))
        if rc != 0:
            raise ValueError("a body is outside the box")
        state["state"], state["is_final"], state["boundary"] = st.value, fin.value, b.tolist()
        self.L = self.box()

    def gsd_frame(self):
        """FP32 site positions (n, 3) and versors (n, 4) or None, as a GSD frame holds them."""
        pos = np.zeros((self.n, 3), dtype=np.float32)
        ori = np.zeros((self.n, 4), dtype=np.float32) if self.ori_len else None
        lib().oracle_gsd_frame(self._h, pos.ctypes.data, None if ori is None else ori.ctypes.data)
        return pos, ori

    def increment_step(self):
        lib().oracle_increment_step(self._h)

    def parallel_sweep(self, move, maximum, kt, body_interaction_range, threads=1):
        a = C.c_uint64()
        r = C.c_uint64()
        rc = lib().oracle_parallel_sweep_threads(self._h, move, maximum, kt, body_interaction_range, threads,
                                                 C.byref(a), C.byref(r))
        if rc:
            raise RuntimeError(f"oracle parallel sweep failed ({rc})")
        return a.value, r.value

    def serial_sweep(self, move, maximum, kt, mask=None):
        a = C.c_uint64()
        r = C.c_uint64()
        m = None if mask is None else np.ascontiguousarray(np.asarray(mask, dtype=bool).astype(np.uint8))
        lib().oracle_serial_sweep_filter(self._h, move, maximum, kt, None if m is None else m.ctypes.data_as(_u8p),
                                         C.byref(a), C.byref(r))
        return a.value, r.value

    def tune(self, move, maximum, kt, target, samples, steps) -> float:
        """The per-sample-stream tuner (each sample its own Counter index)."""
        return float(lib().oracle_tune(self._h, move, maximum, kt, target, samples, steps))

    def tune_stream(self, move, maximum, kt, target, samples, steps) -> float:
        """tune_local_trial with the reference's one sequential stream."""
        return float(lib().oracle_tune_stream(self._h, move, maximum, kt, target, samples, steps))

    def sdf(self, x_max, n_bins) -> np.ndarray:
        out = np.zeros(n_bins, dtype=np.uint64)
        lib().oracle_sdf(self._h, x_max, n_bins, out.ctypes.data_as(_u64p))
        return out

    def gr(self, r_max, n_bins) -> np.ndarray:
        out = np.zeros(n_bins, dtype=np.uint64)
        lib().oracle_gr(self._h, r_max, n_bins, out.ctypes.data_as(_u64p))
        return out

    def overlap_count(self) -> int:
        return int(lib().oracle_overlap_count(self._h))

    def total_energy(self) -> float:
        return float(lib().oracle_total_energy(self._h))

    def delta_energy_one(self, body, position, orientation=None):
        p = _f64(position)
        o = None if orientation is None else _f64(orientation)
        return lib().oracle_delta_energy_one(self._h, body, _d(p), _d(o))

    def eval_moves(self, bodies, positions, orientations, u, kt):
        b = np.ascontiguousarray(bodies, dtype=np.uint64)
        n = b.size
        p = _f64(positions, (-1,))
        o = None if orientations is None else _f64(orientations, (-1,))
        uu = _f64(u)
        dec = np.zeros(n, dtype=np.uint8)
        dh = np.zeros(n)
        lib().oracle_eval_moves(self._h, n, b.ctypes.data_as(_u64p), _d(p), _d(o), _d(uu), kt,
                                dec.ctypes.data_as(_u8p), _d(dh))
        return dec.astype(bool), dh
