// Hard convex polygons: PairwiseCutoff<HardShape<Convex<ConvexPolygon>>> (XenoCollide) and
// PairwiseCutoff<HardShape<ConvexSurfaceMesh2d>> (separating axes), with
// Translate<Cartesian<2>> and Rotate<Angle> trial moves.
//
// The pair test is IntersectsAtGlobal (hoomd-geometry/src/convex.rs:101-121 and
// shape/convex_surface_mesh_2d.rs:514-536): a circumcircle rejection, pair_system_to_local
// (hoomd-vector/src/lib.rs:878-888) with Angle rotations (hoomd-vector/src/angle.rs:120-230),
// then XenoCollide in 2-D (hoomd-geometry/src/xenocollide.rs:92-154, :361-414) or the
// separating-axis test (convex_surface_mesh_2d.rs:578-640). Every product, sum and fused
// multiply-add follows the reference's expression order; sin and cos are correctly rounded
// (cr_sincos), so the FP64 decision is the reference's on a correctly rounded libm.
//
// The colour pass gives a warp four trials, as for polyhedra (k_sweep_poly2); injected moves
// take one warp per move and the stencil's candidates 32 at a time, with an early exit by
// vote. FP32 + recheck: candidates whose FP32 centre distance clears the circumcircles by more
// than the FP32 error bound are skipped; every other candidate runs the FP64 test.
#include <cuda_runtime.h>

#include "hmc_serial.cuh"

namespace hmc {
namespace {

// Resident blocks per SM the colour pass is compiled for: 8 caps it at 64 registers. On 2^18
// hard squares at area fraction 0.60 this measured 6.4e8 (FP32 prefilter) and 6.7e8 (FP64)
// trial moves/s, against 6.1e8 and 6.5e8 at 80 registers, 4.3e8 and 4.2e8 uncapped (180
// registers) and 1.5e8 and 1.6e8 with one warp per trial.
#ifndef HMC_POLY2_MIN_BLOCKS
#define HMC_POLY2_MIN_BLOCKS 8
#endif

struct V2 {
    double x, y;
};
struct M2 {
    V2 r[2];
};
__device__ __forceinline__ double dot2(const V2& a, const V2& b) {  // mul_add fold from 0.0
    return dfma(a.y, b.y, dfma(a.x, b.x, 0.0));
}
__device__ __forceinline__ V2 sub2(const V2& a, const V2& b) { return {dsub(a.x, b.x), dsub(a.y, b.y)}; }
__device__ __forceinline__ V2 perp2(const V2& a) { return {-a.y, a.x}; }  // cartesian.rs:755
__device__ __forceinline__ V2 mat2_rotate(const M2& m, const V2& v) { return {dot2(m.r[0], v), dot2(m.r[1], v)}; }
__device__ __forceinline__ M2 transpose2(const M2& m) { return {{{m.r[0].x, m.r[1].x}, {m.r[0].y, m.r[1].y}}}; }

// RotationMatrix::from(Angle) (angle.rs:120-131); false when |theta| >= 2^20.
__device__ __forceinline__ bool mat2_from_angle(double theta, M2* m) {
    double s, c;
    if (!cr_sincos(theta, &s, &c)) return false;
    *m = {{{c, -s}, {s, c}}};
    return true;
}

// ConvexPolytope::support_mapping in 2-D: argmax of v0 n0 + v1 n1, first maximum wins.
__device__ __forceinline__ V2 support2(const double4* __restrict__ verts, uint32_t nv, const V2& n) {
    uint32_t arg = 0;
    double best = -INFINITY;
#pragma unroll 4  // vertex loads of several iterations in flight; comparisons stay in order
    for (uint32_t i = 0; i < nv; ++i) {
        const double4 v = ldg4(verts + i);
        const double x = dadd(dmul(v.x, n.x), dmul(v.y, n.y));
        if (x > best) {
            best = x;
            arg = i;
        }
    }
    const double4 v = ldg4(verts + arg);
    return {v.x, v.y};
}

constexpr int kXenoMaxIter2 = 1024;  // xenocollide.rs:38

// collide for N = 2 (xenocollide.rs:92-154, :361-414); the iteration cap returns overlap.
__device__ __noinline__ bool collide2d(const double4* verts, uint32_t nv, const V2& vij, const M2& q) {
    const M2 qinv = transpose2(q);
    // composite_support_mapping (xenocollide.rs:318-328)
    auto s = [&](const V2& n) -> V2 {
        const V2 sb = support2(verts, nv, mat2_rotate(qinv, n));
        V2 r = mat2_rotate(q, sb);
        r = {dadd(r.x, vij.x), dadd(r.y, vij.y)};
        const V2 sa = support2(verts, nv, V2{-n.x, -n.y});
        return sub2(r, sa);
    };
    const double TOL = 1e-16;
    const V2 v0 = vij;
    const V2 v1 = s(V2{-v0.x, -v0.y});
    V2 vp = perp2(sub2(v1, v0));
    if (dot2(v1, vp) > 0.0) vp = {-vp.x, -vp.y};
    const V2 v2 = s(vp);
    V2 p0 = v1, p1 = v2;
    for (int count = 1;; ++count) {
        V2 nn = perp2(sub2(p1, p0));
        if (dot2(sub2(p0, v0), nn) < 0.0) nn = {-nn.x, -nn.y};
        if (dot2(p0, nn) >= 0.0) return true;
        const V2 vnew = s(nn);
        if (dot2(vnew, nn) < 0.0) return false;
        // tolerance_check (:127-138): d = w - project(w, e), w = vnew - p0, e = p1 - p0
        const V2 w = sub2(vnew, p0);
        const V2 e = sub2(p1, p0);
        const double kk = dot2(w, e);
        const double nb = dot2(e, e);
        const V2 pr{ddiv(dmul(e.x, kk), nb), ddiv(dmul(e.y, kk), nb)};
        const V2 d = sub2(w, pr);
        if (dot2(d, d) < dmul(TOL, dot2(vnew, vnew))) return true;
        // narrow_portal (:141-154)
        V2 vpp = perp2(sub2(vnew, v0));
        if (dot2(sub2(p0, vnew), vpp) < 0.0) vpp = {-vpp.x, -vpp.y};
        if (dot2(vnew, vpp) < 0.0)
            p1 = vnew;
        else
            p0 = vnew;
        if (count >= kXenoMaxIter2) return true;
    }
}

// is_separating (convex_surface_mesh_2d.rs:625-640): every vertex of a strictly outside.
__device__ __forceinline__ bool is_separating(const double4* verts, uint32_t nv, const V2& p, const V2& n) {
    const double n_dot_p = dot2(n, p);
    for (uint32_t i = 0; i < nv; ++i) {
        const double4 v = ldg4(verts + i);
        if (dsub(dot2(n, V2{v.x, v.y}), n_dot_p) <= 0.0) return false;
    }
    return true;
}
// b_edge_separates (:597-623) with a = b = the shape.
__device__ __forceinline__ bool b_edge_separates(const double4* verts, uint32_t nv, const V2& v_ab, const M2& o_b) {
    uint32_t previous = nv - 1;
    for (uint32_t current = 0; current < nv; ++current) {
        const double4 pc = ldg4(verts + current), pp = ldg4(verts + previous);
        const V2 p{pc.x, pc.y};
        const V2 edge = sub2(p, V2{pp.x, pp.y});
        const V2 n{edge.y, -edge.x};  // -edge.perpendicular()
        V2 pa = mat2_rotate(o_b, p);
        pa = {dadd(pa.x, v_ab.x), dadd(pa.y, v_ab.y)};
        const V2 na = mat2_rotate(o_b, n);
        if (is_separating(verts, nv, pa, na)) return true;
        previous = current;
    }
    return false;
}
// ConvexSurfaceMesh2d::intersects_at (:578-593).
__device__ __noinline__ bool sat_intersects(const double4* verts, uint32_t nv, const V2& v_ij, const M2& o_j) {
    if (b_edge_separates(verts, nv, v_ij, o_j)) return false;
    const M2 inv = transpose2(o_j);
    const V2 v_ji = mat2_rotate(inv, V2{-v_ij.x, -v_ij.y});
    return !b_edge_separates(verts, nv, v_ji, inv);
}

struct PolyShape2 {
    const double4* verts;
    uint32_t nv;
    double rcut2;      // (R_a + R_b)^2
    float rcut2_hi32;  // FP32 threshold: at or above this, outside the circumcircles for certain
};

// Trial site t with angle ti against slot q's site sj (image rule) and angle: the pair test of
// HardShape::site_pair_energy. *range_error is set when an angle is beyond the supported
// range of cr_sincos; the pair then counts as overlapping (the move is rejected).
template <bool SAT>
__device__ __forceinline__ bool poly2_overlap64(const Geometry& g, const Arrays& A, const PolyShape2& sh,
                                                const double* t, double ti, const double* sj, uint32_t q,
                                                bool* range_error) {
    double d[3];
    const double d2 = ref_disp<2>(g, t, sj, d);
    if (d2 >= sh.rcut2) return false;  // r_self.distance_squared(r_other) >= r_cut^2
    const V2 rab{-d[0], -d[1]};  // image - t
    const double tj = __ldg(&A.sorted_q[q].x);
    const double inv = -ti;  // Angle::inverted
    double sn, cs;
    M2 m;
    if (!cr_sincos(inv, &sn, &cs) || !mat2_from_angle(dadd(inv, tj), &m)) {
        *range_error = true;
        return true;
    }
    const V2 vij{dsub(dmul(rab.x, cs), dmul(rab.y, sn)), dadd(dmul(rab.x, sn), dmul(rab.y, cs))};  // Angle::rotate
    return SAT ? sat_intersects(sh.verts, sh.nv, vij, m) : collide2d(sh.verts, sh.nv, vij, m);
}

__device__ __forceinline__ bool warp_any2(bool v) { return __any_sync(0xffffffffu, v); }

// Overlap of the trial (t, ti) with any candidate of the stencil fs (the 3 rows around the
// trial's space), skipping slot self: the warp takes the candidates 32 at a time across the
// rows, with a vote after each step.
template <bool FP32, bool SAT>
__device__ __forceinline__ bool poly2_overlaps(const Geometry& g, const Arrays& A, const PolyShape2& sh,
                                               const double* t, double ti, float4 t32, int mf, const FlatStencil& fs,
                                               uint32_t self, uint32_t lane, PairStats& st, bool* range_error) {
    const uint32_t sf = g.shape[1];
#pragma unroll 1
    for (uint32_t j0 = 0; j0 < fs.total; j0 += 32) {
        const uint32_t j = j0 + lane;
        uint32_t part;
        const uint32_t q = flat_slot(fs, j, part);
        const float s0 = __shfl_sync(0xffffffffu, fs.s0, part);
        bool hit = false;
        if (j < fs.total && q != self) {
            bool test = true;
            if (FP32) {
                const float4 o = __ldg(A.sorted_off + q);
                int dm = __float_as_int(o.w) - mf;
                if (sf >= 4) {  // the wrapped space of a row at a fast-axis end
                    if (dm > 1)
                        dm -= (int)sf;
                    else if (dm < -1)
                        dm += (int)sf;
                }
                st.checks++;
                test = fp32_dist2<2>(g, t32, o, s0, 0.f, dm) < sh.rcut2_hi32;
                if (test) st.rechecks++;
            }
            if (test) {
                // shapes keep S in both precision modes (the FP32 pass only prefilters)
                const double4 s4 = ldg4(A.sorted_s + q);
                const double sj[3] = {s4.x, s4.y, 0.0};
                if (!FP32) st.checks++;
                hit = poly2_overlap64<SAT>(g, A, sh, t, ti, sj, q, range_error);
            }
        }
        if (warp_any2(hit)) return true;
    }
    return false;
}

// ---- the colour pass, four trials per warp ---------------------------------------------------
// As for polyhedra (hmc_poly.cu): each group of 8 lanes computes its trial and prefilters its
// candidates by circumcircle, the candidates that need the full FP64 test are compacted over
// the warp into a shared-memory list, and the warp runs those tests 32 pairs at a time, ORing
// overlaps into a per-trial mask (a trial known to overlap lists no further candidates). The
// decision of each trial is the OR of the same pair tests as with one warp per trial.
constexpr int kPoly2TrialsPerWarp = 4;
constexpr uint32_t kPair2Cap = 128;  // listed pairs per warp before the warp drains the list

struct Poly2Trial {
    double t[2];
    double angle;
};

template <bool SAT>
__device__ __forceinline__ void drain_pairs2(const Geometry& g, const Arrays& A, const PolyShape2& sh,
                                             const Poly2Trial* trials, const uint32_t* pair_q, const uint8_t* pair_g,
                                             uint32_t n_pairs, uint32_t lane, uint32_t& mask, bool* range_error) {
    __syncwarp();
    for (uint32_t p0 = 0; p0 < n_pairs; p0 += 32) {
        const uint32_t p = p0 + lane;
        uint32_t bit = 0;
        if (p < n_pairs) {
            const uint32_t gg = pair_g[p];
            if (!((mask >> gg) & 1u)) {
                const uint32_t q = pair_q[p];
                const Poly2Trial& tr = trials[gg];
                const double t[3] = {tr.t[0], tr.t[1], 0.0};
                const double4 s4 = ldg4(A.sorted_s + q);
                const double sj[3] = {s4.x, s4.y, 0.0};
                if (poly2_overlap64<SAT>(g, A, sh, t, tr.angle, sj, q, range_error)) bit = 1u << gg;
            }
        }
        mask |= __reduce_or_sync(0xffffffffu, bit);
    }
    __syncwarp();
}

template <bool FP32, bool SAT>
__global__ void __launch_bounds__(128, HMC_POLY2_MIN_BLOCKS)
    k_sweep_poly2(Geometry g, Arrays A, PolyShape2 sh, Launch L, uint32_t rotate) {
    constexpr uint32_t G = kPoly2TrialsPerWarp, S = 32 / G;  // trials per warp, lanes per trial
    if (L.early_wait) grid_dependency_wait();  // first pass: the rebuild's arrays are read at once
    __shared__ Poly2Trial s_trial[4][G];
    __shared__ uint32_t s_pair_q[4][kPair2Cap];
    __shared__ uint8_t s_pair_g[4][kPair2Cap];
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const uint32_t grp = lane / S, sub = lane % S;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
    uint32_t n_accepted = 0;
    PairStats st;
    bool range_error = false;
    const uint32_t sf = g.shape[1];
    const uint32_t n_active = active_count(A, L.color, L.round);
    for (uint32_t w0 = warp * G; w0 < n_active; w0 += n_warps * G) {  // warp-uniform
        const uint32_t w = w0 + grp;
        uint32_t m[3] = {0, 0, 0};
        uint32_t k = 0;
        bool valid = false;
        double t[3] = {0.0, 0.0, 0.0};
        double ti = 0.0;
        float4 t32 = make_float4(0.f, 0.f, 0.f, 0.f);
        if (w < n_active) {  // the group's trial from k_propose_poly2
            const size_t e = (size_t)L.color * g.color_stride + w;
            k = __ldg(A.trial_k + e);
            valid = k != kNoTrial;
            if (valid) {
                unpack_m<2>(__ldg(A.color_cells + e), m);
                const double4 t4 = ldg4(A.trial_t + e);
                t[0] = t4.x;
                t[1] = t4.y;
                ti = t4.w;
                if (FP32) t32 = __ldg(A.trial_o + e);
            }
        }
        if (sub == 0) {
            Poly2Trial& tr = s_trial[wib][grp];
            tr.t[0] = t[0];
            tr.t[1] = t[1];
            tr.angle = ti;
        }
        grid_dependency_wait();  // the previous colour's moves are visible from here on
        allow_dependent_launch();
        uint32_t mask = 0, n_pairs = 0;  // warp-uniform
#pragma unroll 1
        for (int part = 0; part < 2 * kRows<2>; ++part) {
            uint32_t lo = 0, len = 0;
            float s0 = 0.f, s1 = 0.f;
            if (valid) stencil_part<2>(g, A.cell_start, m, part >> 1, (part & 1) != 0, lo, len, s0, s1);
            const uint32_t iters = __reduce_max_sync(0xffffffffu, (len + S - 1) / S);
            for (uint32_t it = 0; it < iters; ++it) {
                const uint32_t j = it * S + sub;
                const uint32_t q = lo + j;
                bool need = false;
                if (j < len && q != k && !((mask >> grp) & 1u)) {
                    st.checks++;
                    if (FP32) {
                        const float4 o = __ldg(A.sorted_off + q);
                        int dm = __float_as_int(o.w) - (int)m[1];
                        if (sf >= 4) {  // the wrapped space of a row at a fast-axis end
                            if (dm > 1)
                                dm -= (int)sf;
                            else if (dm < -1)
                                dm += (int)sf;
                        }
                        need = fp32_dist2<2>(g, t32, o, s0, 0.f, dm) < sh.rcut2_hi32;
                        if (need) st.rechecks++;
                    } else {
                        // the circumcircle test that opens poly2_overlap64
                        const double4 s4 = ldg4(A.sorted_s + q);
                        const double sj[3] = {s4.x, s4.y, 0.0};
                        double d[3];
                        need = ref_disp<2>(g, t, sj, d) < sh.rcut2;
                    }
                }
                const unsigned b = __ballot_sync(0xffffffffu, need);
                if (need) {
                    const uint32_t pos = n_pairs + __popc(b & ((1u << lane) - 1u));
                    s_pair_q[wib][pos] = q;
                    s_pair_g[wib][pos] = (uint8_t)grp;
                }
                n_pairs += __popc(b);
                if (n_pairs > kPair2Cap - 32) {
                    drain_pairs2<SAT>(g, A, sh, s_trial[wib], s_pair_q[wib], s_pair_g[wib], n_pairs, lane, mask,
                                      &range_error);
                    n_pairs = 0;
                }
            }
        }
        drain_pairs2<SAT>(g, A, sh, s_trial[wib], s_pair_q[wib], s_pair_g[wib], n_pairs, lane, mask, &range_error);
        if (sub == 0 && valid && !((mask >> grp) & 1u)) {
            n_accepted++;
            double sv[3] = {t[0], t[1], 0.0};
            wrap_inv<2>(g.L, g.invL, sv);
            const uint32_t body = A.sorted_body[k];
            A.sorted_b[k] = make_double4(t[0], t[1], 0.0, 0.0);
            A.sorted_s[k] = make_double4(sv[0], sv[1], 0.0, 0.0);
            A.sorted_off[k] = cell_offsets<2>(g, sv, m);
            A.sorted_q[k] = make_double4(ti, 0.0, 0.0, 0.0);
            A.body_pos[body] = make_double4(t[0], t[1], 0.0, 0.0);
            A.body_ori[body] = make_double4(ti, 0.0, 0.0, 0.0);
        }
        __syncwarp();
    }
    grid_dependency_wait();
    allow_dependent_launch();
    if (range_error) atomicOr(&A.stats->error_flags, kErrAngleRange);
    flush_stats(A.stats, st, n_accepted);
}

// ---- the insertion hamiltonian: approximate shape overlap -----------------------------------
// Anisotropic::site_pair_energy (anisotropic.rs:120-135) of ApproximateShapeOverlap
// (approximate_shape_overlap.rs:122-131) for the site t with angle ti against the site sj (image
// rule) with angle tj: 0 at a centre distance >= r_cut, else pair_system_to_local (Angle::rotate
// by -ti, o_ij = -ti + tj) and IntersectsAt::approximate_separation_distance (hoomd-geometry/src/
// lib.rs:307-325): the direction v / |v| (the last axis for v = 0) and d grown by `resolution`
// while Convex::intersects_at (convex.rs:87-99: the bounding circles, |w|^2 <= (R + R)^2, then
// XenoCollide) holds at w = v + direction * d; the energy is OverlapPenalty(-d). An angle beyond
// cr_sincos's range sets *range_error and counts as infinite.
// SAT: ConvexSurfaceMesh2d, whose intersects_at (convex_surface_mesh_2d.rs:538-595) is the
// separating-axis test alone, without the bounding circles.
template <bool SAT>
__device__ __forceinline__ double shape_overlap2(const Geometry& g, const PolyShape2& sh, const ShapeOverlap& so,
                                                 const double* t, double ti, const double* sj, double tj,
                                                 uint32_t& capped, bool* range_error) {
    double d[3];
    const double d2 = ref_disp<2>(g, t, sj, d);
    if (dsqrt(d2) >= so.rcut) return 0.0;
    const V2 rab{-d[0], -d[1]};  // image - t
    const double inv = -ti;
    double sn, cs;
    M2 m;
    if (!cr_sincos(inv, &sn, &cs) || !mat2_from_angle(dadd(inv, tj), &m)) {
        *range_error = true;
        return __longlong_as_double(0x7ff0000000000000ll);
    }
    const V2 v{dsub(dmul(rab.x, cs), dmul(rab.y, sn)), dadd(dmul(rab.x, sn), dmul(rab.y, cs))};
    const double norm = dsqrt(dot2(v, v));
    const V2 dir = norm == 0.0 ? V2{0.0, 1.0} : V2{ddiv(v.x, norm), ddiv(v.y, norm)};
    double sep = 0.0;
    for (uint32_t step = 0;; ++step) {
        const V2 w{dadd(v.x, dmul(dir.x, sep)), dadd(v.y, dmul(dir.y, sep))};
        if (SAT ? !sat_intersects(sh.verts, sh.nv, w, m) : (!(dot2(w, w) <= so.rr) || !collide2d(sh.verts, sh.nv, w, m)))
            break;
        if (step >= so.max_steps) {
            capped = 1;
            break;
        }
        sep = dadd(sep, so.resolution);
    }
    return separation_penalty(so, sep);
}

// ParallelSweep colour pass of convex polygons under the approximate shape overlap (FP64), one
// warp per trial from k_propose_poly2 (soft: the uniform in trial_t.z, the angle in .w); the
// sums and the Metropolis test as in k_sweep_poly3_soft.
template <bool SAT>
__global__ void __launch_bounds__(128) k_sweep_poly2_soft(Geometry g, Arrays A, PolyShape2 sh, ShapeOverlap so,
                                                          Launch L) {
    if (L.early_wait) grid_dependency_wait();  // first pass: the rebuild's arrays are read at once
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
    uint32_t n_accepted = 0, capped = 0;
    bool range_error = false;
    PairStats pst;
    const uint32_t n_active = active_count(A, L.color, L.round);
    for (uint32_t w = warp; w < n_active; w += n_warps) {
        const size_t e = (size_t)L.color * g.color_stride + w;
        const uint32_t k = __ldg(A.trial_k + e);
        if (k == kNoTrial) continue;  // warp-uniform: the move left its space
        uint32_t m[3] = {0, 0, 0};
        unpack_m<2>(__ldg(A.color_cells + e), m);
        const double4 t4 = ldg4(A.trial_t + e);
        const double t[3] = {t4.x, t4.y, 0.0};
        const double u = t4.z, tt = t4.w;
        const FlatStencil fs = flat_stencil<2>(g, A.cell_start, m, lane);
        grid_dependency_wait();  // the previous colour's moves are visible from here on
        allow_dependent_launch();
        const double4 s4 = ldg4(A.sorted_s + k);
        const double si[3] = {s4.x, s4.y, 0.0};
        const double tk = __ldg(&A.sorted_q[k].x);
        double a = 0.0, b = 0.0, mag = 0.0;
#pragma unroll 1
        for (uint32_t j0 = 0; j0 < fs.total; j0 += 32) {
            const uint32_t j = j0 + lane;
            uint32_t part;
            const uint32_t q = flat_slot(fs, j, part);
            if (j < fs.total && q != k) {
                const double4 c4 = ldg4(A.sorted_s + q);
                const double sj[3] = {c4.x, c4.y, 0.0};
                const double tj = __ldg(&A.sorted_q[q].x);
                const double x = shape_overlap2<SAT>(g, sh, so, t, tt, sj, tj, capped, &range_error);
                const double y = shape_overlap2<SAT>(g, sh, so, si, tk, sj, tj, capped, &range_error);
                a = dadd(a, x);
                b = dadd(b, y);
                mag += fabs(x) + fabs(y);
                pst.checks += 2;
            }
        }
        const double e_new = warp_sum64(a), e_old = warp_sum64(b);
        mag = warp_sum64(mag);
        const double du = dsub(e_new, e_old);
        const double e0 = exp(ddiv(-du, L.kt));
        if (lane == 0 && order_ambiguous(du, mag, fs.total, u, L.kt, e0)) pst.ambiguous++;
        if ((du <= 0.0 || u < e0) && lane == 0) {
            n_accepted++;
            double sv[3] = {t[0], t[1], 0.0};
            wrap_inv<2>(g.L, g.invL, sv);
            const uint32_t body = A.sorted_body[k];
            A.sorted_b[k] = make_double4(t[0], t[1], 0.0, 0.0);
            A.sorted_s[k] = make_double4(sv[0], sv[1], 0.0, 0.0);
            A.sorted_off[k] = cell_offsets<2>(g, sv, m);
            A.sorted_q[k] = make_double4(tt, 0.0, 0.0, 0.0);
            A.body_pos[body] = make_double4(t[0], t[1], 0.0, 0.0);
            A.body_ori[body] = make_double4(tt, 0.0, 0.0, 0.0);
        }
        __syncwarp();
    }
    if (__any_sync(0xffffffffu, capped != 0u) && lane == 0) atomicOr(&A.stats->error_flags, kErrIterationCap);
    if (range_error) atomicOr(&A.stats->error_flags, kErrAngleRange);
    grid_dependency_wait();
    allow_dependent_launch();
    flush_stats(A.stats, pst, n_accepted);
}

// PairwiseCutoff::total_energy under the approximate shape overlap for polygons (as
// k_energy_poly3_soft).
template <bool SAT>
__global__ void k_energy_poly2_soft(Geometry g, Arrays A, PolyShape2 sh, ShapeOverlap so, uint32_t n, double* out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t capped = 0;
    bool range_error = false;
    if (k < n) {
        const uint32_t bi = A.sorted_body[k];
        const double4 s4 = A.sorted_s[k];
        const double t[3] = {s4.x, s4.y, 0.0};
        const double ti = A.sorted_q[k].x;
        uint32_t m[3] = {0, 0, 0};
        uint32_t c = A.body_cell[bi];
        for (int a = 1; a >= 0; --a) {
            m[a] = c % g.shape[a];
            c /= g.shape[a];
        }
        double e = 0.0;
        for_each_neighbor<2>(g, A.cell_start, m, [&](uint32_t q, const float*) -> bool {
            if (A.sorted_body[q] <= bi) return false;
            const double4 c4 = A.sorted_s[q];
            const double sj[3] = {c4.x, c4.y, 0.0};
            e = dadd(e, shape_overlap2<SAT>(g, sh, so, t, ti, sj, A.sorted_q[q].x, capped, &range_error));
            return false;
        });
        atomicAdd(out, e);
    }
    if (capped) atomicOr(&A.stats->error_flags, kErrIterationCap);
    if (range_error) atomicOr(&A.stats->error_flags, kErrAngleRange);
}

// QuickInsert's insertion loop for convex polygons under the approximate shape overlap, one warp
// (k_quick_insert_poly3 with the angle drawn from Uniform::new(0, 2 pi), angle.rs:268-285).
template <bool SAT>
__global__ void __launch_bounds__(32) k_quick_insert_poly2(Geometry g, Arrays A, SerialGrid G, PolyShape2 sh,
                                                           ShapeOverlap so, Launch L, QuickInsertArgs q, BodyTags T,
                                                           unsigned long long* out) {
    const uint32_t lane = threadIdx.x;
    if (A.stats->error_flags) return;
    Sfc64 rng = make_rng(L.step, L.substep, L.seed, 0);
    uint32_t n = q.n0, capped = 0;
    bool range_error = false;
    uint64_t inserted = 0, overlapping = 0, rejected = 0;
    const double two_pi = dmul(2.0, 3.141592653589793);
    for (uint64_t attempt = 0; attempt < q.attempts; ++attempt) {
        double x[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            const double u = dsub(as_double(0x3FF0000000000000ULL | (rng.next_u64() >> 12)), 1.0);
            x[a] = dadd(dmul(u, q.scale[a]), q.low[a]);
        }
        const double ua = dsub(as_double(0x3FF0000000000000ULL | (rng.next_u64() >> 12)), 1.0);
        const double o = dadd(dmul(ua, dsub(two_pi, 0.0)), 0.0);
        double t[3] = {x[0], x[1], 0.0};
        wrap_inv<2>(g.L, g.invL, t);
        uint32_t m[3] = {0, 0, 0}, cell;
        serial_cell<2>(g, G, t, m);
        bool inf = false, pos = false;
        if (lane_cell<2>(G, m, lane, &cell)) {
            const uint32_t cnt = G.size[cell];
            for (uint32_t kk = 0; kk < cnt && !inf; ++kk) {
                const uint32_t j = G.items[(size_t)cell * G.cap + kk];
                const double4 s4 = G.site[j];
                const double sv[3] = {s4.x, s4.y, 0.0};
                const double e = shape_overlap2<SAT>(g, sh, so, t, o, sv, A.body_ori[j].x, capped, &range_error);
                inf = e == __longlong_as_double(0x7ff0000000000000ll);
                pos = pos || e > 0.0;
            }
        }
        inf = __any_sync(0xffffffffu, inf);
        pos = __any_sync(0xffffffffu, pos);
        if (inf) {
            rejected++;
            continue;
        }
        if (n >= q.capacity) {
            if (lane == 0) atomicOr(&A.stats->error_flags, kErrCellOverflow);
            break;
        }
        if (lane == 0) {
            grid_append<2>(g, A, G, T, n, x);
            A.body_ori[n] = make_double4(o, 0.0, 0.0, 0.0);
        }
        __syncwarp();
        n++;
        inserted++;
        if (pos) overlapping++;
        if (inserted == q.to_insert || overlapping >= q.allowed) break;
        if (A.stats->error_flags) break;
    }
    if (__any_sync(0xffffffffu, capped != 0u) && lane == 0) atomicOr(&A.stats->error_flags, kErrIterationCap);
    if (__any_sync(0xffffffffu, range_error) && lane == 0) atomicOr(&A.stats->error_flags, kErrAngleRange);
    if (lane == 0) {
        out[0] = inserted;
        out[1] = overlapping;
        out[2] = rejected;
        out[3] = n;
    }
}

// Injected moves (position and angle): warp per move.
template <bool FP32, bool SAT>
__global__ void __launch_bounds__(128) k_eval_poly2(Geometry g, Arrays A, PolyShape2 sh, const uint64_t* bodies,
                                                    const double4* trial, const double4* trial_q, uint32_t n,
                                                    uint8_t* decisions) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    PairStats st;
    bool range_error = false;
    if (i < n) {
        const uint32_t k = A.slot_of_body[bodies[i]];
        const double4 w4 = trial[i];
        double t[3] = {w4.x, w4.y, 0.0};
        wrap_inv<2>(g.L, g.invL, t);
        const double ti = trial_q[i].x;
        uint32_t m[3] = {0, 0, 0};
        uint8_t dec = 0;
        if (point_to_space<2>(g, t, m)) {
            const float4 t32 = FP32 ? cell_offsets<2>(g, t, m) : make_float4(0.f, 0.f, 0.f, 0.f);
            const FlatStencil fs = flat_stencil<2>(g, A.cell_start, m, lane);
            dec = poly2_overlaps<FP32, SAT>(g, A, sh, t, ti, t32, (int)m[1], fs, k, lane, st, &range_error) ? 0 : 1;
        } else if (lane == 0) {
            atomicOr(&A.stats->error_flags, kErrOutsideCheckerboard);
        }
        if (lane == 0) decisions[i] = dec;
    }
    if (range_error) atomicOr(&A.stats->error_flags, kErrAngleRange);
    flush_stats(A.stats, st, 0u);
}

// The sequential-stream tuner for hard convex polygons (tune_stream_run): Translate or
// Rotate<Angle> (theta += Uniform(-a, a): 52 random bits in [1, 2) minus one, times the range,
// plus the low end; rotate/angle.rs:46-55) proposals, the trial accepted when no candidate of the
// stencil around its site's space overlaps it (FP64 XenoCollide or separating axes).
template <bool SAT>
__global__ void __launch_bounds__(32) k_tune_stream_poly2(TuneJob* jobs, uint32_t n_jobs, PolyShape2 sh) {
    if (blockIdx.x >= n_jobs) return;
    TuneJob& J = jobs[blockIdx.x];
    const Geometry& g = J.g;
    const Arrays& A = J.a;
    const uint32_t lane = threadIdx.x & 31u;
    PairStats st;
    bool range_error = false;
    tune_stream_run(
        J,
        [&](Sfc64& rng, double m, uint32_t b, double* x, double* q) {
            q[0] = A.body_ori[b].x;
            if (J.rotate) {
                const double4 b4 = A.body_pos[b];
                x[0] = b4.x;
                x[1] = b4.y;
                const double u = dsub(as_double(0x3FF0000000000000ULL | (rng.next_u64() >> 12)), 1.0);
                q[0] = dadd(q[0], dadd(dmul(u, dsub(m, -m)), -m));
                wrap_inv<2>(g.L, g.invL, x);
            } else {
                tune_translate<2>(rng, g, A, m, b, x);
            }
        },
        [&](Sfc64&, uint32_t b, const double* x, const double* q) -> bool {
            double t[3] = {x[0], x[1], 0.0};
            wrap_inv<2>(g.L, g.invL, t);
            uint32_t m[3] = {0, 0, 0};
            if (!point_to_space<2>(g, t, m)) {
                if (lane == 0) atomicOr(&A.stats->error_flags, kErrOutsideCheckerboard);
                return false;
            }
            const FlatStencil fs = flat_stencil<2>(g, A.cell_start, m, lane);
            return !poly2_overlaps<false, SAT>(g, A, sh, t, q[0], make_float4(0.f, 0.f, 0.f, 0.f), (int)m[1], fs,
                                               A.slot_of_body[b], lane, st, &range_error);
        });
    if (range_error) atomicOr(&J.a.stats->error_flags, kErrAngleRange);
}

// A round's trial moves of convex polygons for every colour list, one thread per trial: the
// chosen body, Translate (Ball::sample) or Rotate<Angle> (theta += Uniform(-a, a), rotate/angle.rs:
// 46-55), W1 = wrap(propose(..)), the space check, T = wrap(W1) with the angle in .w, and T's FP32
// offsets; the packed pass reads them instead of computing each move on the 8 lanes of its group.
template <bool FP32>
__global__ void __launch_bounds__(128) k_propose_poly2(Geometry g, Arrays A, Launch L, uint32_t rotate,
                                                       uint32_t soft) {
    const DeviceStats* st = A.stats;
    if (st->error_flags != 0u || L.round >= st->rounds) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 4u * g.color_stride; i += gridDim.x * blockDim.x) {
        const uint32_t c = i / g.color_stride, w = i - c * g.color_stride;
        if (w >= st->color_count[c]) continue;
        uint32_t m[3] = {0, 0, 0};
        unpack_m<2>(__ldg(A.color_cells + i), m);
        const uint32_t cell = cell_index<2>(g, m);
        const uint32_t start = __ldg(A.cell_start + cell);
        const uint32_t count = __ldg(A.cell_start + cell + 1) - start;
        Sfc64 rng = make_rng(L.step, L.substep, L.seed, (uint64_t)cell);
        const uint32_t k = start + canon_range_u32(rng, count);
        const double4 b4 = A.sorted_b[k];
        double x[3] = {b4.x, b4.y, 0.0};
        double ti = A.sorted_q[k].x;
        if (rotate) {
            const double u = dsub(as_double(0x3FF0000000000000ULL | (rng.next_u64() >> 12)), 1.0);
            ti = dadd(ti, dadd(dmul(u, dsub(L.max_move, -L.max_move)), -L.max_move));
        } else {
            double dv[3];
            ball_sample<2>(rng, L.max_move, A.zig_x, A.zig_f, dv);
            x[0] = dadd(x[0], dv[0]);
            x[1] = dadd(x[1], dv[1]);
        }
        // soft: the Metropolis uniform, the stream's next draw after the move
        const double u = soft ? uniform01(rng) : 0.0;
        wrap_inv<2>(g.L, g.invL, x);  // W1 = wrap(propose(..))
        uint32_t mt[3];
        if (!(point_to_space<2>(g, x, mt) && cell_index<2>(g, mt) == cell)) {
            A.trial_k[i] = kNoTrial;
            continue;
        }
        double t[3] = {x[0], x[1], 0.0};
        wrap_inv<2>(g.L, g.invL, t);
        A.trial_t[i] = make_double4(t[0], t[1], u, ti);
        if (FP32) A.trial_o[i] = cell_offsets<2>(g, t, m);
        A.trial_k[i] = k;
    }
}

// Sweep::apply_with_filter (hoomd-mc/src/sweep.rs:159-224) for hard convex polygons: one trial per
// body in index order from one stream, Translate or Rotate<Angle>, accepted when no site of the
// serial grid's stencil overlaps it (no uniform is drawn); one warp, a lane per stencil cell. The
// pair tests read each body's angle by body index.
template <bool SAT>
__global__ void __launch_bounds__(32) k_serial_poly2(Geometry g, Arrays A, SerialGrid G, PolyShape2 sh, Launch L,
                                                     uint32_t rotate, const uint8_t* __restrict__ mask) {
    const uint32_t lane = threadIdx.x;
    if (A.stats->error_flags) return;
    Arrays Ab = A;
    Ab.sorted_q = A.body_ori;
    bool range_error = false;
    Sfc64 rng = make_rng(L.step, L.substep, L.seed, 0);
    uint64_t accepted = 0;
    for (uint32_t b = 0; b < L.n_bodies; ++b) {
        if (mask && !mask[b]) continue;
        const double4 b4 = A.body_pos[b];
        double x[3] = {b4.x, b4.y, 0.0};
        double ti = A.body_ori[b].x;
        if (rotate) {
            // Rotate<Angle>::propose (rotate/angle.rs:46-55): theta += Uniform(-a, a)
            const double u = dsub(as_double(0x3FF0000000000000ULL | (rng.next_u64() >> 12)), 1.0);
            ti = dadd(ti, dadd(dmul(u, dsub(L.max_move, -L.max_move)), -L.max_move));
        } else {
            double dv[3];
            ball_sample<2>(rng, L.max_move, A.zig_x, A.zig_f, dv);
            x[0] = dadd(x[0], dv[0]);
            x[1] = dadd(x[1], dv[1]);
        }
        wrap_inv<2>(g.L, g.invL, x);  // W1 = wrap(propose(..))
        double t[3] = {x[0], x[1], 0.0};
        wrap_inv<2>(g.L, g.invL, t);  // the trial site T = wrap(W1)
        uint32_t m[3] = {0, 0, 0}, cell;
        serial_cell<2>(g, G, t, m);
        bool overlap = false;
        if (lane_cell<2>(G, m, lane, &cell)) {
            const uint32_t cnt = G.size[cell];
            for (uint32_t k = 0; k < cnt && !overlap; ++k) {
                const uint32_t j = G.items[(size_t)cell * G.cap + k];
                if (j == b) continue;
                const double4 s4 = G.site[j];
                const double sv[3] = {s4.x, s4.y, 0.0};
                overlap = poly2_overlap64<SAT>(g, Ab, sh, t, ti, sv, j, &range_error);
            }
        }
        if (__any_sync(0xffffffffu, overlap)) continue;
        accepted++;
        if (lane == 0) {
            double sv[3] = {t[0], t[1], 0.0};
            wrap_inv<2>(g.L, g.invL, sv);
            A.body_pos[b] = make_double4(t[0], t[1], 0.0, 0.0);
            A.body_ori[b].x = ti;
            G.site[b] = make_double4(sv[0], sv[1], 0.0, 0.0);
            serial_move<2>(g, G, A, b, sv);
        }
        __syncwarp();
        if (A.stats->error_flags) break;
    }
    if (range_error) atomicOr(&A.stats->error_flags, kErrAngleRange);
    if (lane == 0) {
        A.stats->accepted = accepted;
        A.stats->rechecks = 0;
    }
}

// Overlapping pairs (i < j), FP64 (the overlap check of total_energy).
template <bool SAT>
__global__ void k_overlap_poly2(Geometry g, Arrays A, PolyShape2 sh, uint32_t n) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t found = 0;
    bool range_error = false;
    if (k < n) {
        const uint32_t bi = A.sorted_body[k];
        const double4 s4 = A.sorted_s[k];
        const double t[3] = {s4.x, s4.y, 0.0};
        const double ti = A.sorted_q[k].x;
        uint32_t m[3] = {0, 0, 0};
        uint32_t c = A.body_cell[bi];
        m[1] = c % g.shape[1];
        m[0] = c / g.shape[1];
        for_each_neighbor<2>(g, A.cell_start, m, [&](uint32_t q, const float*) -> bool {
            if (A.sorted_body[q] <= bi) return false;
            const double4 o4 = A.sorted_s[q];
            const double sj[3] = {o4.x, o4.y, 0.0};
            if (poly2_overlap64<SAT>(g, A, sh, t, ti, sj, q, &range_error)) found++;
            return false;
        });
    }
    if (range_error) atomicOr(&A.stats->error_flags, kErrAngleRange);
    const unsigned tot = __reduce_add_sync(0xffffffffu, found);
    if ((threadIdx.x & 31) == 0 && tot) atomicAdd(&A.stats->overlaps, (unsigned long long)tot);
}

// cr_sincos over an array (the exact values the rotation path uses).
__global__ void k_sincos(const double* x, uint64_t n, double* s, double* c, uint32_t* bad) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double sv = 0.0, cv = 0.0;
    if (!cr_sincos(x[i], &sv, &cv)) {
        atomicOr(bad, 1u);
        sv = cv = NAN;
    }
    s[i] = sv;
    c[i] = cv;
}

}  // namespace

cudaError_t launch_sweep_poly2(bool fp32, bool sat, const Geometry& g, const Arrays& a, const double4* verts,
                               uint32_t nv, double rcut2, float rcut2_hi32, const Launch& l, bool rotate,
                               cudaStream_t s) {
    if (l.n_active == 0) return cudaSuccess;
    static int max_blocks = 0;
    if (max_blocks == 0) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        max_blocks = sms * 16;
    }
    PolyShape2 sh{verts, nv, rcut2, rcut2_hi32};
    const uint32_t per_block = 4u * kPoly2TrialsPerWarp;  // four warps per block
    uint32_t blocks = (l.n_active + per_block - 1) / per_block;
    if (blocks > (uint32_t)max_blocks) blocks = (uint32_t)max_blocks;
    const uint32_t rot = rotate ? 1u : 0u;
    PassLaunch pl(blocks, l.overlap_previous != 0 || l.early_wait != 0, s);
    if (fp32)
        return sat ? cudaLaunchKernelEx(&pl.cfg, k_sweep_poly2<true, true>, g, a, sh, l, rot)
                   : cudaLaunchKernelEx(&pl.cfg, k_sweep_poly2<true, false>, g, a, sh, l, rot);
    return sat ? cudaLaunchKernelEx(&pl.cfg, k_sweep_poly2<false, true>, g, a, sh, l, rot)
               : cudaLaunchKernelEx(&pl.cfg, k_sweep_poly2<false, false>, g, a, sh, l, rot);
}

cudaError_t launch_propose_poly2(bool fp32, const Geometry& g, const Arrays& a, const Launch& l, bool rotate,
                                 bool soft, cudaStream_t s) {
    const uint64_t n = (uint64_t)g.color_stride << 2;
    if (n == 0) return cudaSuccess;
    const int wave = resident_wave((const void*)(fp32 ? k_propose_poly2<true> : k_propose_poly2<false>));
    uint32_t blocks = (uint32_t)((n + 127) / 128);
    if (blocks > (uint32_t)wave) blocks = (uint32_t)wave;
    if (fp32)
        k_propose_poly2<true><<<blocks, 128, 0, s>>>(g, a, l, rotate ? 1u : 0u, soft ? 1u : 0u);
    else
        k_propose_poly2<false><<<blocks, 128, 0, s>>>(g, a, l, rotate ? 1u : 0u, soft ? 1u : 0u);
    return cudaGetLastError();
}

cudaError_t launch_sweep_poly2_soft(bool sat, const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                                    const ShapeOverlap& so, const Launch& l, cudaStream_t s) {
    if (l.n_active == 0) return cudaSuccess;
    PolyShape2 sh{verts, nv, so.rr, 0.f};
    using SoftKernel = void (*)(Geometry, Arrays, PolyShape2, ShapeOverlap, Launch);
    const SoftKernel k = sat ? k_sweep_poly2_soft<true> : k_sweep_poly2_soft<false>;
    const int wave = resident_wave((const void*)k);
    uint32_t blocks = (l.n_active + 3) / 4;  // four warps (trials) per block
    if (blocks > (uint32_t)wave) blocks = (uint32_t)wave;
    PassLaunch pl(blocks, l.overlap_previous != 0 || l.early_wait != 0, s);
    return cudaLaunchKernelEx(&pl.cfg, k, g, a, sh, so, l);
}

cudaError_t launch_energy_poly2_soft(bool sat, const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                                     const ShapeOverlap& so, uint32_t n, double* out, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    PolyShape2 sh{verts, nv, so.rr, 0.f};
    if (sat)
        k_energy_poly2_soft<true><<<(n + 127) / 128, 128, 0, s>>>(g, a, sh, so, n, out);
    else
        k_energy_poly2_soft<false><<<(n + 127) / 128, 128, 0, s>>>(g, a, sh, so, n, out);
    return cudaGetLastError();
}

cudaError_t launch_quick_insert_poly2(bool sat, const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                                      const ShapeOverlap& so, const Launch& l, const QuickInsertArgs& q,
                                      const BodyTags& tags, const uint32_t* nc, const double* w, uint32_t cap,
                                      uint32_t* size, uint32_t* items, uint32_t* cell_of, double4* site,
                                      unsigned long long* out, cudaStream_t s) {
    const SerialGrid G = make_grid(2, nc, w, cap, size, items, cell_of, site);
    cudaError_t e = build_grid(2, g, a, G, q.n0, s);
    if (e != cudaSuccess) return e;
    PolyShape2 sh{verts, nv, so.rr, 0.f};
    if (sat)
        k_quick_insert_poly2<true><<<1, 32, 0, s>>>(g, a, G, sh, so, l, q, tags, out);
    else
        k_quick_insert_poly2<false><<<1, 32, 0, s>>>(g, a, G, sh, so, l, q, tags, out);
    return cudaGetLastError();
}

cudaError_t launch_serial_poly2(bool sat, const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                                double rcut2, const Launch& l, bool rotate, const uint32_t* nc, const double* w,
                                uint32_t cap, uint32_t* size, uint32_t* items, uint32_t* cell_of, double4* site,
                                const uint8_t* mask, cudaStream_t s) {
    const SerialGrid G = make_grid(2, nc, w, cap, size, items, cell_of, site);
    cudaError_t e = build_grid(2, g, a, G, l.n_bodies, s);
    if (e != cudaSuccess || l.n_bodies == 0) return e;
    const PolyShape2 sh{verts, nv, rcut2, 0.f};
    if (sat)
        k_serial_poly2<true><<<1, 32, 0, s>>>(g, a, G, sh, l, rotate ? 1u : 0u, mask);
    else
        k_serial_poly2<false><<<1, 32, 0, s>>>(g, a, G, sh, l, rotate ? 1u : 0u, mask);
    return cudaGetLastError();
}

cudaError_t launch_tune_stream_poly2(bool sat, TuneJob* jobs, uint32_t n_jobs, const double4* verts, uint32_t nv,
                                     double rcut2, cudaStream_t s) {
    if (n_jobs == 0) return cudaSuccess;
    const PolyShape2 sh{verts, nv, rcut2, 0.f};
    if (sat)
        k_tune_stream_poly2<true><<<n_jobs, 32, 0, s>>>(jobs, n_jobs, sh);
    else
        k_tune_stream_poly2<false><<<n_jobs, 32, 0, s>>>(jobs, n_jobs, sh);
    return cudaGetLastError();
}

cudaError_t launch_eval_poly2(bool fp32, bool sat, const Geometry& g, const Arrays& a, const double4* verts,
                              uint32_t nv, double rcut2, float rcut2_hi32, const uint64_t* bodies,
                              const double4* trial, const double4* trial_q, uint32_t n, uint8_t* decisions,
                              cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    PolyShape2 sh{verts, nv, rcut2, rcut2_hi32};
    const uint32_t blocks = (n + 3) / 4;
    if (fp32) {
        if (sat)
            k_eval_poly2<true, true><<<blocks, 128, 0, s>>>(g, a, sh, bodies, trial, trial_q, n, decisions);
        else
            k_eval_poly2<true, false><<<blocks, 128, 0, s>>>(g, a, sh, bodies, trial, trial_q, n, decisions);
    } else {
        if (sat)
            k_eval_poly2<false, true><<<blocks, 128, 0, s>>>(g, a, sh, bodies, trial, trial_q, n, decisions);
        else
            k_eval_poly2<false, false><<<blocks, 128, 0, s>>>(g, a, sh, bodies, trial, trial_q, n, decisions);
    }
    return cudaGetLastError();
}

cudaError_t launch_overlap_poly2(bool sat, const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                                 double rcut2, uint32_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    PolyShape2 sh{verts, nv, rcut2, 0.f};
    if (sat)
        k_overlap_poly2<true><<<(n + 127) / 128, 128, 0, s>>>(g, a, sh, n);
    else
        k_overlap_poly2<false><<<(n + 127) / 128, 128, 0, s>>>(g, a, sh, n);
    return cudaGetLastError();
}

cudaError_t launch_sincos(const double* x, uint64_t n, double* sn, double* cs, uint32_t* bad, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_sincos<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(x, n, sn, cs, bad);
    return cudaGetLastError();
}

}  // namespace hmc
