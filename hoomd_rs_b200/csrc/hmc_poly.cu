// Hard convex polyhedra: PairwiseCutoff<HardShape<Convex<ConvexPolyhedron>>> with
// Translate<Cartesian<3>> and Rotate<Versor> trial moves.
//
// The pair test is Convex::intersects_at_global (hoomd-geometry/src/convex.rs:154-170): a
// circumsphere rejection, pair_system_to_local (hoomd-vector/src/lib.rs:878-888) and
// XenoCollide / Minkowski portal refinement (hoomd-geometry/src/xenocollide.rs:172-414) over
// the support function of the vertex table (shape/convex_polytope.rs:222-244). Every
// product, sum and fused multiply-add below follows the reference's expression order, so
// the FP64 decision is the reference's.
//
// The colour pass gives a warp four trials (k_sweep_poly3_packed): each group of 8 lanes
// computes its trial and prefilters its candidates by circumsphere, and the warp runs the full
// tests of all four trials' remaining candidates together. Injected moves (k_eval_poly3) take
// one warp per move and the stencil's candidates 32 at a time, with an early exit by vote.
// FP32 + recheck: a candidate whose FP32 centre distance clears the circumsphere by more
// than the FP32 error bound is skipped; every other candidate runs the FP64 test, so the
// decisions equal the FP64 pass.
#include <cuda_runtime.h>

#include "hmc_serial.cuh"

namespace hmc {
namespace {

// The colour pass takes kPolyTrialsPerWarp trials per warp and is compiled for
// HMC_POLY_MIN_BLOCKS resident blocks per SM (96 registers). On 2^18 hard cubes at packing
// fraction 0.55 (10,648 trials per colour pass) this measured 1.69e8 (FP32 prefilter) and
// 1.58e8 (FP64) trial moves/s, against 7.9e7 and 8.3e7 with one warp per trial, 1.38e8 and
// 1.26e8 with 8 trials per warp, 1.48e8 and 1.43e8 with 4 trials at 80 registers.
#ifndef HMC_POLY_MIN_BLOCKS
#define HMC_POLY_MIN_BLOCKS 5
#endif
constexpr int kPolyTrialsPerWarp = 4;

struct Q {
    double s, x, y, z;
};
struct V3 {
    double x, y, z;
};

__device__ __forceinline__ double dot3(const V3& a, const V3& b) {  // mul_add fold from 0.0
    return dfma(a.z, b.z, dfma(a.y, b.y, dfma(a.x, b.x, 0.0)));
}
__device__ __forceinline__ V3 cross3(const V3& a, const V3& b) {  // cartesian.rs:604-610
    return {dsub(dmul(a.y, b.z), dmul(a.z, b.y)), dsub(dmul(a.z, b.x), dmul(a.x, b.z)),
            dsub(dmul(a.x, b.y), dmul(a.y, b.x))};
}
__device__ __forceinline__ V3 sub3(const V3& a, const V3& b) { return {dsub(a.x, b.x), dsub(a.y, b.y), dsub(a.z, b.z)}; }
__device__ __forceinline__ V3 neg3(const V3& a) { return {-a.x, -a.y, -a.z}; }

// Quaternion::mul (quaternion.rs:408-415).
__device__ __forceinline__ Q qmul(const Q& a, const Q& b) {
    const V3 av{a.x, a.y, a.z}, bv{b.x, b.y, b.z};
    const double sc = dsub(dmul(a.s, b.s), dot3(av, bv));
    const V3 c = cross3(av, bv);
    return {sc, dadd(dadd(dmul(bv.x, a.s), dmul(av.x, b.s)), c.x), dadd(dadd(dmul(bv.y, a.s), dmul(av.y, b.s)), c.y),
            dadd(dadd(dmul(bv.z, a.s), dmul(av.z, b.s)), c.z)};
}
// Versor::rotate (quaternion.rs:740-747).
__device__ __forceinline__ V3 vrotate(const Q& q, const V3& v) {
    const V3 qv{q.x, q.y, q.z};
    const double k1 = dsub(dmul(q.s, q.s), dot3(qv, qv));
    const V3 c = cross3(qv, v);
    const double k2 = dmul(2.0, q.s);
    const double k3 = dmul(2.0, dot3(qv, v));
    return {dadd(dadd(dmul(v.x, k1), dmul(c.x, k2)), dmul(qv.x, k3)),
            dadd(dadd(dmul(v.y, k1), dmul(c.y, k2)), dmul(qv.y, k3)),
            dadd(dadd(dmul(v.z, k1), dmul(c.z, k2)), dmul(qv.z, k3))};
}

struct M3 {
    V3 r[3];
};
// RotationMatrix::from(Versor) (quaternion.rs:642-690).
__device__ __forceinline__ M3 mat_from(const Q& q) {
    const double a = q.s, b = q.x, c = q.y, d = q.z;
    M3 m;
    m.r[0] = {dsub(dsub(dadd(dmul(a, a), dmul(b, b)), dmul(c, c)), dmul(d, d)),
              dsub(dmul(dmul(2.0, b), c), dmul(dmul(2.0, a), d)), dadd(dmul(dmul(2.0, b), d), dmul(dmul(2.0, a), c))};
    m.r[1] = {dadd(dmul(dmul(2.0, b), c), dmul(dmul(2.0, a), d)),
              dsub(dadd(dsub(dmul(a, a), dmul(b, b)), dmul(c, c)), dmul(d, d)),
              dsub(dmul(dmul(2.0, c), d), dmul(dmul(2.0, a), b))};
    m.r[2] = {dsub(dmul(dmul(2.0, b), d), dmul(dmul(2.0, a), c)), dadd(dmul(dmul(2.0, c), d), dmul(dmul(2.0, a), b)),
              dadd(dsub(dsub(dmul(a, a), dmul(b, b)), dmul(c, c)), dmul(d, d))};
    return m;
}
__device__ __forceinline__ V3 mat_rotate(const M3& m, const V3& v) {
    return {dot3(m.r[0], v), dot3(m.r[1], v), dot3(m.r[2], v)};
}
__device__ __forceinline__ M3 transpose(const M3& m) {
    return {{{m.r[0].x, m.r[1].x, m.r[2].x}, {m.r[0].y, m.r[1].y, m.r[2].y}, {m.r[0].z, m.r[1].z, m.r[2].z}}};
}

// ConvexPolytope::support_mapping: argmax of ((v0 n0) + v1 n1) + v2 n2, first maximum wins.
// Unrolled by four so that the vertex loads of several iterations are in flight together (the
// comparisons stay in order). For cubes this measured the same as rolled (1.69e8 trial moves/s,
// FP32), for the 2-D squares' support2 +3 %; a shared-memory copy of the table gained nothing.
__device__ __forceinline__ V3 support(const double4* __restrict__ verts, uint32_t nv, const V3& n) {
    uint32_t arg = 0;
    double best = -INFINITY;
#pragma unroll 4
    for (uint32_t i = 0; i < nv; ++i) {
        const double4 v = ldg4(verts + i);
        const double x = dadd(dadd(dmul(v.x, n.x), dmul(v.y, n.y)), dmul(v.z, n.z));
        if (x > best) {
            best = x;
            arg = i;
        }
    }
    const double4 v = ldg4(verts + arg);
    return {v.x, v.y, v.z};
}

struct Minkowski {
    const double4* verts;
    uint32_t nv;
    V3 vij;
    M3 q, qinv;
    // composite_support_mapping (xenocollide.rs:318-328)
    __device__ __forceinline__ V3 operator()(const V3& n) const {
        const V3 sb = support(verts, nv, mat_rotate(qinv, n));
        V3 r = mat_rotate(q, sb);
        r = {dadd(r.x, vij.x), dadd(r.y, vij.y), dadd(r.z, vij.z)};
        const V3 sa = support(verts, nv, neg3(n));
        return sub3(r, sa);
    }
};

constexpr int kXenoMaxIter = 1024;  // xenocollide.rs:38

// collide for N = 3 (xenocollide.rs:172-291, :361-414). The iteration caps return overlap,
// as the reference does.
__device__ __noinline__ bool collide3d(const double4* verts, uint32_t nv, const V3& vij, const Q& oij) {
    Minkowski s;
    s.verts = verts;
    s.nv = nv;
    s.vij = vij;
    s.q = mat_from(oij);
    s.qinv = transpose(s.q);
    const double TOL = 2e-12;
    const V3 v0 = vij;
    if (fabs(v0.x) < TOL && fabs(v0.y) < TOL && fabs(v0.z) < TOL) return true;
    V3 v1 = s(neg3(v0));
    if (dot3(v1, v0) > 0.0) return false;
    V3 n = cross3(v1, v0);
    if (fabs(n.x) < TOL && fabs(n.y) < TOL && fabs(n.z) < TOL) return true;
    V3 v2 = s(n);
    if (dot3(v2, n) < 0.0) return false;
    n = cross3(sub3(v1, v0), sub3(v2, v0));
    if (dot3(n, v0) > 0.0) {
        const V3 t = v1;
        v1 = v2;
        v2 = t;
        n = neg3(n);
    }
    V3 v3;
    for (int count = 1;; ++count) {
        if (count >= kXenoMaxIter) return true;
        v3 = s(n);
        if (dot3(v3, n) <= 0.0) return false;
        if (dot3(cross3(v1, v3), v0) < 0.0) {
            v2 = v3;
            n = cross3(sub3(v1, v0), sub3(v2, v0));
            continue;
        }
        if (dot3(cross3(v3, v2), v0) < 0.0) {
            v1 = v3;
            n = cross3(sub3(v1, v0), sub3(v2, v0));
            continue;
        }
        break;
    }
    V3 p0 = v1, p1 = v2, p2 = v3;
    for (int count = 1;; ++count) {
        V3 nn = cross3(sub3(p1, p0), sub3(p2, p0));
        if (dot3(sub3(p0, v0), nn) < 0.0) nn = neg3(nn);
        if (dot3(p0, nn) >= 0.0) return true;
        const V3 vn = s(nn);
        if (dot3(vn, nn) < 0.0) return false;
        const double tol = dmul(TOL, dsqrt(dot3(nn, nn)));
        if (fabs(dot3(sub3(vn, p0), nn)) < tol) return false;
        if (fabs(dot3(p0, nn)) < tol) return true;
        const V3 vp = cross3(vn, v0);
        const bool t1 = dot3(vp, p0) > 0.0, t2 = dot3(vp, p1) > 0.0, t3 = dot3(vp, p2) > 0.0;
        if (t1 && t2)
            p0 = vn;
        else if (t1 && !t2)
            p2 = vn;
        else if (!t1 && t3)
            p1 = vn;
        else
            p0 = vn;
        if (count >= kXenoMaxIter) return true;
    }
}

// Trial site t (position) with versor qi against the site of slot q (position S via the image
// rule, versor sorted_q[q]): HardShape::site_pair_energy -> intersects_at_global.
__device__ __forceinline__ bool poly_overlap64(const Geometry& g, const Arrays& A, const double4* verts, uint32_t nv,
                                               double rcut2, const double* t, const Q& qi, const double* sj, uint32_t q) {
    double d[3];
    const double d2 = ref_disp<3>(g, t, sj, d);
    if (d2 >= rcut2) return false;  // r_self.distance_squared(r_other) >= r_cut^2
    const V3 rab{-d[0], -d[1], -d[2]};  // image - t, exactly -(t - image)
    const double4 o4 = ldg4(A.sorted_q + q);
    const Q qj{o4.x, o4.y, o4.z, o4.w};
    const Q ia{qi.s, -qi.x, -qi.y, -qi.z};  // Versor::inverted = conjugate
    const V3 vij = vrotate(ia, rab);
    const Q oij = qmul(ia, qj);
    return collide3d(verts, nv, vij, oij);
}

// Rotate<Versor>::propose (rotate/versor.rs:40-71, 112-123): Gaussian rotation vector with
// standard deviation sigma, rejected beyond pi, lifted by the exponential map, composed in
// front of the current orientation.
__device__ __forceinline__ Q versor_move(Sfc64& rng, double sigma, const double* zx, const double* zf, const Q& q) {
    for (;;) {
        double s0 = dadd(0.0, dmul(sigma, standard_normal(rng, zx, zf)));
        double s1 = dadd(0.0, dmul(sigma, standard_normal(rng, zx, zf)));
        double s2 = dadd(0.0, dmul(sigma, standard_normal(rng, zx, zf)));
        const V3 sv{s0, s1, s2};
        const double theta = dsqrt(dot3(sv, sv));
        if (theta > 3.141592653589793) continue;
        double sh, ch;
        portable_sincos(dmul(0.5, theta), &sh, &ch);
        double vf = ddiv(sh, theta);
        if (!isfinite(vf)) vf = 0.5;
        const Q dq{ch, dmul(s0, vf), dmul(s1, vf), dmul(s2, vf)};
        return qmul(dq, q);
    }
}

struct PolyShape {
    const double4* verts;
    uint32_t nv;
    double rcut2;     // (R_a + R_b)^2
    float rcut2_hi32; // FP32 threshold: at or above this, outside the circumsphere for certain
};

__device__ __forceinline__ bool warp_any(bool v) { return __any_sync(0xffffffffu, v); }

// Overlap of the trial (t, qi; FP32 offsets t32) with any candidate of the stencil fs,
// skipping slot self. The warp takes the stencil's candidates 32 at a time across its rows
// (at the bench's density one step holds the whole stencil, so the lanes that need the full
// test run it together), and a vote after each step stops the warp at the first overlap.
// FP32: the circumsphere prefilter in FP32 under the bound.
template <bool FP32>
__device__ __forceinline__ bool poly_overlaps(const Geometry& g, const Arrays& A, const PolyShape& sh, const double* t,
                                              const Q& qi, float4 t32, int mf, const FlatStencil& fs, uint32_t self,
                                              uint32_t lane, PairStats& st) {
    const uint32_t sf = g.shape[2];
#pragma unroll 1
    for (uint32_t j0 = 0; j0 < fs.total; j0 += 32) {
        const uint32_t j = j0 + lane;
        uint32_t part;
        const uint32_t q = flat_slot(fs, j, part);
        const float s0 = __shfl_sync(0xffffffffu, fs.s0, part);
        const float s1 = __shfl_sync(0xffffffffu, fs.s1, part);
        bool hit = false;
        if (j < fs.total && q != self) {
            bool test = true;
            if (FP32) {
                const float4 o = __ldg(A.sorted_off + q);
                int dm = __float_as_int(o.w) - mf;
                if (sf >= 4) {
                    if (dm > 1)
                        dm -= (int)sf;
                    else if (dm < -1)
                        dm += (int)sf;
                }
                st.checks++;
                test = fp32_dist2<3>(g, t32, o, s0, s1, dm) < sh.rcut2_hi32;
                if (test) st.rechecks++;
            }
            if (test) {
                // shapes keep S in both precision modes (the FP32 pass only prefilters)
                const double4 s4 = ldg4(A.sorted_s + q);
                const double sj[3] = {s4.x, s4.y, s4.z};
                if (!FP32) st.checks++;
                hit = poly_overlap64(g, A, sh.verts, sh.nv, sh.rcut2, t, qi, sj, q);
            }
        }
        if (warp_any(hit)) return true;
    }
    return false;
}

// ---- the colour pass, G trials per warp -----------------------------------------------------
// A trial's candidates mostly clear the circumsphere; the few that do not need the full FP64
// test (XenoCollide, thousands of instructions). With one warp per trial that test runs with a
// handful of lanes active. Here a warp takes G trials (32/G lanes each): every group computes
// its trial, walks its stencil with the circumsphere test, and the candidates that need the
// full test are compacted over the whole warp into a shared-memory list; the warp then runs
// the full tests 32 pairs at a time and ORs the overlaps into a per-trial mask. Candidates of a
// trial already known to overlap are skipped. The decision of each trial is the OR of the same
// pair tests as in the warp-per-trial pass, so the trajectory is the same.
struct PolyTrial {
    double t[3];
    double q[4];  // s, x, y, z
};

constexpr uint32_t kPairCap = 128;  // listed pairs per warp before the warp drains the list

template <int G>
__device__ __forceinline__ void drain_pairs(const Geometry& g, const Arrays& A, const PolyShape& sh,
                                            const PolyTrial* trials, const uint32_t* pair_q, const uint8_t* pair_g,
                                            uint32_t n_pairs, uint32_t lane, uint32_t& mask) {
    __syncwarp();
    for (uint32_t p0 = 0; p0 < n_pairs; p0 += 32) {
        const uint32_t p = p0 + lane;
        uint32_t bit = 0;
        if (p < n_pairs) {
            const uint32_t gg = pair_g[p];
            if (!((mask >> gg) & 1u)) {
                const uint32_t q = pair_q[p];
                const PolyTrial& tr = trials[gg];
                const double t[3] = {tr.t[0], tr.t[1], tr.t[2]};
                const Q qi{tr.q[0], tr.q[1], tr.q[2], tr.q[3]};
                const double4 s4 = ldg4(A.sorted_s + q);
                const double sj[3] = {s4.x, s4.y, s4.z};
                if (poly_overlap64(g, A, sh.verts, sh.nv, sh.rcut2, t, qi, sj, q)) bit = 1u << gg;
            }
        }
        mask |= __reduce_or_sync(0xffffffffu, bit);
    }
    __syncwarp();
}

// A round's trial moves of convex polyhedra for every colour list (generate_trial_moves,
// parallel_sweep.rs:231-278, up to delta_energy_one), one thread per trial: the chosen body,
// Translate (Ball::sample) or Rotate<Versor>, W1 = wrap(propose(..)), the space check, the trial
// site T = wrap(W1) and its FP32 offsets; the packed pass reads them instead of computing each
// move on the 8 lanes of its group.
template <bool FP32>
__global__ void __launch_bounds__(128) k_propose_poly3(Geometry g, Arrays A, Launch L, uint32_t rotate,
                                                       uint32_t soft) {
    const DeviceStats* st = A.stats;
    if (st->error_flags != 0u || L.round >= st->rounds) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 8u * g.color_stride; i += gridDim.x * blockDim.x) {
        const uint32_t c = i / g.color_stride, w = i - c * g.color_stride;
        if (w >= st->color_count[c]) continue;
        uint32_t m[3] = {0, 0, 0};
        unpack_m<3>(__ldg(A.color_cells + i), m);
        const uint32_t cell = cell_index<3>(g, m);
        const uint32_t start = __ldg(A.cell_start + cell);
        const uint32_t count = __ldg(A.cell_start + cell + 1) - start;
        Sfc64 rng = make_rng(L.step, L.substep, L.seed, (uint64_t)cell);
        const uint32_t k = start + canon_range_u32(rng, count);
        const double4 b4 = A.sorted_b[k];
        double x[3] = {b4.x, b4.y, b4.z};
        const double4 q4 = A.sorted_q[k];
        Q qi{q4.x, q4.y, q4.z, q4.w};
        if (rotate) {
            qi = versor_move(rng, L.max_move, A.zig_x, A.zig_f, qi);
        } else {
            double dv[3];
            ball_sample<3>(rng, L.max_move, A.zig_x, A.zig_f, dv);
            for (int a = 0; a < 3; ++a) x[a] = dadd(x[a], dv[a]);
        }
        // soft: the Metropolis uniform, the stream's next draw after the move
        const double u = soft ? uniform01(rng) : 0.0;
        wrap_inv<3>(g.L, g.invL, x);  // W1 = wrap(propose(..))
        uint32_t mt[3];
        if (!(point_to_space<3>(g, x, mt) && cell_index<3>(g, mt) == cell)) {
            A.trial_k[i] = kNoTrial;
            continue;
        }
        double t[3] = {x[0], x[1], x[2]};
        wrap_inv<3>(g.L, g.invL, t);
        A.trial_t[i] = make_double4(t[0], t[1], t[2], u);
        A.trial_q[i] = make_double4(qi.s, qi.x, qi.y, qi.z);
        if (FP32) A.trial_o[i] = cell_offsets<3>(g, t, m);
        A.trial_k[i] = k;
    }
}

// INJ: the probe mode (Injected): group trial w is injected trial w, walked around the space of
// its W1, and its decision is written instead of committed.
template <bool FP32, int G, bool INJ = false>
__global__ void __launch_bounds__(128, HMC_POLY_MIN_BLOCKS)
    k_sweep_poly3_packed(Geometry g, Arrays A, PolyShape sh, Launch L, uint32_t rotate, Injected J) {
    static_assert(G == 2 || G == 4 || G == 8, "G trials per warp");
    constexpr uint32_t S = 32 / G;  // lanes per trial
    if (L.early_wait) grid_dependency_wait();  // first pass: the rebuild's arrays are read at once
    __shared__ PolyTrial s_trial[4][G];
    __shared__ uint32_t s_pair_q[4][kPairCap];
    __shared__ uint8_t s_pair_g[4][kPairCap];
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const uint32_t grp = lane / S, sub = lane % S;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
    uint32_t n_accepted = 0;
    PairStats st;
    const uint32_t sf = g.shape[2];
    const uint32_t n_active = INJ ? J.n : active_count(A, L.color, L.round);
    for (uint32_t w0 = warp * G; w0 < n_active; w0 += n_warps * G) {  // warp-uniform
        const uint32_t w = w0 + grp;
        uint32_t m[3] = {0, 0, 0};
        uint32_t k = 0;
        bool valid = false;
        double t[3] = {0.0, 0.0, 0.0};
        Q qi{1.0, 0.0, 0.0, 0.0};
        uint8_t flag = 0;
        float4 t32p = make_float4(0.f, 0.f, 0.f, 0.f);
        if (INJ && w < n_active) {  // the injected trial (W1, versor), by the group's S lanes alike
            const uint64_t body = J.bodies[w];
            k = A.slot_of_body[body];
            const double4 w4 = J.trial[w];
            const double x[3] = {w4.x, w4.y, w4.z};
            const double4 q4 = J.trial_q[w];
            qi = Q{q4.x, q4.y, q4.z, q4.w};
            valid = point_to_space<3>(g, x, m);
            if (!valid)
                atomicOr(&A.stats->error_flags, kErrOutsideCheckerboard);
            else if (cell_index<3>(g, m) != A.body_cell[body])
                flag |= kTrialOutsideSpace;
            t[0] = x[0];
            t[1] = x[1];
            t[2] = x[2];
            wrap_inv<3>(g.L, g.invL, t);
        } else if (w < n_active) {  // the group's trial from k_propose_poly3
            const size_t e = (size_t)L.color * g.color_stride + w;
            k = __ldg(A.trial_k + e);
            valid = k != kNoTrial;
            if (valid) {
                unpack_m<3>(__ldg(A.color_cells + e), m);
                const double4 t4 = ldg4(A.trial_t + e);
                t[0] = t4.x;
                t[1] = t4.y;
                t[2] = t4.z;
                const double4 q4 = ldg4(A.trial_q + e);
                qi = Q{q4.x, q4.y, q4.z, q4.w};
                if (FP32) t32p = __ldg(A.trial_o + e);
            }
        }
        const float4 t32 = FP32 && valid ? (INJ ? cell_offsets<3>(g, t, m) : t32p) : make_float4(0.f, 0.f, 0.f, 0.f);
        if (sub == 0) {
            PolyTrial& tr = s_trial[wib][grp];
            tr.t[0] = t[0];
            tr.t[1] = t[1];
            tr.t[2] = t[2];
            tr.q[0] = qi.s;
            tr.q[1] = qi.x;
            tr.q[2] = qi.y;
            tr.q[3] = qi.z;
        }
        grid_dependency_wait();  // the previous colour's moves are visible from here on
        allow_dependent_launch();
        uint32_t mask = 0, n_pairs = 0;  // warp-uniform
#pragma unroll 1
        for (int part = 0; part < 2 * kRows<3>; ++part) {
            uint32_t lo = 0, len = 0;
            float s0 = 0.f, s1 = 0.f;
            if (valid) stencil_part<3>(g, A.cell_start, m, part >> 1, (part & 1) != 0, lo, len, s0, s1);
            const uint32_t iters = __reduce_max_sync(0xffffffffu, (len + S - 1) / S);
            for (uint32_t it = 0; it < iters; ++it) {
                const uint32_t j = it * S + sub;
                const uint32_t q = lo + j;
                bool need = false;
                if (j < len && q != k && !((mask >> grp) & 1u)) {
                    st.checks++;
                    if (FP32) {
                        const float4 o = __ldg(A.sorted_off + q);
                        int dm = __float_as_int(o.w) - (int)m[2];
                        if (sf >= 4) {
                            if (dm > 1)
                                dm -= (int)sf;
                            else if (dm < -1)
                                dm += (int)sf;
                        }
                        need = fp32_dist2<3>(g, t32, o, s0, s1, dm) < sh.rcut2_hi32;
                        if (need) st.rechecks++;
                    } else {
                        // the circumsphere test that opens poly_overlap64
                        const double4 s4 = ldg4(A.sorted_s + q);
                        const double sj[3] = {s4.x, s4.y, s4.z};
                        double d[3];
                        need = ref_disp<3>(g, t, sj, d) < sh.rcut2;
                    }
                }
                const unsigned b = __ballot_sync(0xffffffffu, need);
                if (need) {
                    const uint32_t pos = n_pairs + __popc(b & ((1u << lane) - 1u));
                    s_pair_q[wib][pos] = q;
                    s_pair_g[wib][pos] = (uint8_t)grp;
                }
                n_pairs += __popc(b);
                if (n_pairs > kPairCap - 32) {
                    drain_pairs<G>(g, A, sh, s_trial[wib], s_pair_q[wib], s_pair_g[wib], n_pairs, lane, mask);
                    n_pairs = 0;
                }
            }
        }
        drain_pairs<G>(g, A, sh, s_trial[wib], s_pair_q[wib], s_pair_g[wib], n_pairs, lane, mask);
        if constexpr (INJ) {
            if (sub == 0 && w < n_active) {
                J.decisions[w] = valid && !((mask >> grp) & 1u);
                J.flags[w] = flag;
            }
        } else if (sub == 0 && valid && !((mask >> grp) & 1u)) {
            n_accepted++;
            double sv[3] = {t[0], t[1], t[2]};
            wrap_inv<3>(g.L, g.invL, sv);
            const uint32_t body = A.sorted_body[k];
            A.sorted_b[k] = make_double4(t[0], t[1], t[2], 0.0);
            A.sorted_s[k] = make_double4(sv[0], sv[1], sv[2], 0.0);
            A.sorted_off[k] = cell_offsets<3>(g, sv, m);
            A.sorted_q[k] = make_double4(qi.s, qi.x, qi.y, qi.z);
            A.body_pos[body] = make_double4(t[0], t[1], t[2], 0.0);
            A.body_ori[body] = make_double4(qi.s, qi.x, qi.y, qi.z);
        }
        __syncwarp();
    }
    grid_dependency_wait();
    allow_dependent_launch();
    flush_stats(A.stats, st, n_accepted);
}

// ---- the insertion hamiltonian: approximate shape overlap -----------------------------------
// Anisotropic::site_pair_energy (anisotropic.rs:120-135) of ApproximateShapeOverlap
// (approximate_shape_overlap.rs:122-131) for the site t with versor qi against the site sj (image
// rule) with versor qj: 0 at a centre distance >= r_cut, else pair_system_to_local and
// IntersectsAt::approximate_separation_distance (hoomd-geometry/src/lib.rs:307-325): the
// direction v / |v| (lib.rs:632-639; the last axis for v = 0, cartesian.rs:313-318) and d grown
// by `resolution` while Convex::intersects_at (convex.rs:130-143: the bounding spheres,
// |w|^2 <= (R + R)^2, then XenoCollide) holds at w = v + direction * d; the energy is
// OverlapPenalty(-d).
__device__ __forceinline__ double shape_overlap3(const Geometry& g, const PolyShape& sh, const ShapeOverlap& so,
                                                 const double* t, const Q& qi, const double* sj, const Q& qj,
                                                 uint32_t& capped) {
    double d[3];
    const double d2 = ref_disp<3>(g, t, sj, d);
    if (dsqrt(d2) >= so.rcut) return 0.0;
    const V3 rab{-d[0], -d[1], -d[2]};  // image - t
    const Q ia{qi.s, -qi.x, -qi.y, -qi.z};
    const V3 v = vrotate(ia, rab);
    const Q oij = qmul(ia, qj);
    const double norm = dsqrt(dot3(v, v));
    const V3 dir = norm == 0.0 ? V3{0.0, 0.0, 1.0} : V3{ddiv(v.x, norm), ddiv(v.y, norm), ddiv(v.z, norm)};
    double sep = 0.0;
    for (uint32_t step = 0;; ++step) {
        const V3 w{dadd(v.x, dmul(dir.x, sep)), dadd(v.y, dmul(dir.y, sep)), dadd(v.z, dmul(dir.z, sep))};
        if (!(dot3(w, w) <= so.rr) || !collide3d(sh.verts, sh.nv, w, oij)) break;
        if (step >= so.max_steps) {
            capped = 1;
            break;
        }
        sep = dadd(sep, so.resolution);
    }
    return separation_penalty(so, sep);
}

// ParallelSweep colour pass under the approximate shape overlap (FP64 in both precision modes):
// one warp per trial from k_propose_poly3 (soft), the stencil's candidates 32 at a time. Each lane
// adds the pair energies of the trial (T, q) and of the body's current site (S, q_k) against its
// candidates; butterfly sums give E_final and E_initial (delta_energy_one, pairwise_cutoff.rs:
// 919-941: an infinite pair makes E_final infinite and the move is rejected) and the Metropolis
// test (parallel_sweep.rs:267-268) uses the uniform drawn after the move.
__global__ void __launch_bounds__(128) k_sweep_poly3_soft(Geometry g, Arrays A, PolyShape sh, ShapeOverlap so,
                                                          Launch L) {
    if (L.early_wait) grid_dependency_wait();  // first pass: the rebuild's arrays are read at once
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
    uint32_t n_accepted = 0, capped = 0;
    PairStats pst;
    const uint32_t n_active = active_count(A, L.color, L.round);
    for (uint32_t w = warp; w < n_active; w += n_warps) {
        const size_t e = (size_t)L.color * g.color_stride + w;
        const uint32_t k = __ldg(A.trial_k + e);
        if (k == kNoTrial) continue;  // warp-uniform: the move left its space
        uint32_t m[3] = {0, 0, 0};
        unpack_m<3>(__ldg(A.color_cells + e), m);
        const double4 t4 = ldg4(A.trial_t + e);
        const double t[3] = {t4.x, t4.y, t4.z};
        const double u = t4.w;
        const double4 q4 = ldg4(A.trial_q + e);
        const Q qt{q4.x, q4.y, q4.z, q4.w};
        const FlatStencil fs = flat_stencil<3>(g, A.cell_start, m, lane);
        grid_dependency_wait();  // the previous colour's moves are visible from here on
        allow_dependent_launch();
        const double4 s4 = ldg4(A.sorted_s + k);
        const double si[3] = {s4.x, s4.y, s4.z};
        const double4 o4 = ldg4(A.sorted_q + k);
        const Q qk{o4.x, o4.y, o4.z, o4.w};
        double a = 0.0, b = 0.0, mag = 0.0;
#pragma unroll 1
        for (uint32_t j0 = 0; j0 < fs.total; j0 += 32) {
            const uint32_t j = j0 + lane;
            uint32_t part;
            const uint32_t q = flat_slot(fs, j, part);
            if (j < fs.total && q != k) {
                const double4 c4 = ldg4(A.sorted_s + q);
                const double sj[3] = {c4.x, c4.y, c4.z};
                const double4 cq = ldg4(A.sorted_q + q);
                const Q qj{cq.x, cq.y, cq.z, cq.w};
                const double x = shape_overlap3(g, sh, so, t, qt, sj, qj, capped);
                const double y = shape_overlap3(g, sh, so, si, qk, sj, qj, capped);
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
            double sv[3] = {t[0], t[1], t[2]};
            wrap_inv<3>(g.L, g.invL, sv);
            const uint32_t body = A.sorted_body[k];
            A.sorted_b[k] = make_double4(t[0], t[1], t[2], 0.0);
            A.sorted_s[k] = make_double4(sv[0], sv[1], sv[2], 0.0);
            A.sorted_off[k] = cell_offsets<3>(g, sv, m);
            A.sorted_q[k] = make_double4(qt.s, qt.x, qt.y, qt.z);
            A.body_pos[body] = make_double4(t[0], t[1], t[2], 0.0);
            A.body_ori[body] = make_double4(qt.s, qt.x, qt.y, qt.z);
        }
        __syncwarp();
    }
    if (__any_sync(0xffffffffu, capped != 0u) && lane == 0) atomicOr(&A.stats->error_flags, kErrIterationCap);
    grid_dependency_wait();
    allow_dependent_launch();
    flush_stats(A.stats, pst, n_accepted);
}

// PairwiseCutoff::total_energy (pairwise_cutoff.rs:720-745) under the approximate shape overlap:
// one thread per body i adds the pairs with the bodies j > i of its stencil in i's frame (the
// reference's site_tag_i < site_tag_j; tags are body indices here), summed with atomics.
__global__ void k_energy_poly3_soft(Geometry g, Arrays A, PolyShape sh, ShapeOverlap so, uint32_t n, double* out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t capped = 0;
    if (k < n) {
        const uint32_t bi = A.sorted_body[k];
        const double4 s4 = A.sorted_s[k];
        const double t[3] = {s4.x, s4.y, s4.z};
        const double4 o4 = A.sorted_q[k];
        const Q qi{o4.x, o4.y, o4.z, o4.w};
        uint32_t m[3];
        uint32_t c = A.body_cell[bi];
        for (int a = 2; a >= 0; --a) {
            m[a] = c % g.shape[a];
            c /= g.shape[a];
        }
        double e = 0.0;
        for_each_neighbor<3>(g, A.cell_start, m, [&](uint32_t q, const float*) -> bool {
            if (A.sorted_body[q] <= bi) return false;
            const double4 c4 = A.sorted_s[q];
            const double sj[3] = {c4.x, c4.y, c4.z};
            const double4 cq = A.sorted_q[q];
            e = dadd(e, shape_overlap3(g, sh, so, t, qi, sj, Q{cq.x, cq.y, cq.z, cq.w}, capped));
            return false;
        });
        atomicAdd(out, e);
    }
    if (capped) atomicOr(&A.stats->error_flags, kErrIterationCap);
}

// QuickInsert's insertion loop (k_quick_insert in hmc_serial.cu) for convex polyhedra under the
// approximate shape overlap, one warp: a UniformIn body draws its position per axis, then a
// uniform random versor (StandardUniform for Versor, quaternion.rs:863-885: four standard normals,
// scalar first, divided by sqrt(|v|^2 + s^2)); only whether the insertion energy is infinite or
// positive matters, and single pairs decide both.
__global__ void __launch_bounds__(32) k_quick_insert_poly3(Geometry g, Arrays A, SerialGrid G, PolyShape sh,
                                                           ShapeOverlap so, Launch L, QuickInsertArgs q, BodyTags T,
                                                           unsigned long long* out) {
    const uint32_t lane = threadIdx.x;
    if (A.stats->error_flags) return;
    Sfc64 rng = make_rng(L.step, L.substep, L.seed, 0);
    uint32_t n = q.n0, capped = 0;
    uint64_t inserted = 0, overlapping = 0, rejected = 0;
    for (uint64_t attempt = 0; attempt < q.attempts; ++attempt) {
        double x[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double u = dsub(as_double(0x3FF0000000000000ULL | (rng.next_u64() >> 12)), 1.0);
            x[a] = dadd(dmul(u, q.scale[a]), q.low[a]);
        }
        const double sc = standard_normal(rng, A.zig_x, A.zig_f);
        V3 vv;
        vv.x = standard_normal(rng, A.zig_x, A.zig_f);
        vv.y = standard_normal(rng, A.zig_x, A.zig_f);
        vv.z = standard_normal(rng, A.zig_x, A.zig_f);
        const double norm = dsqrt(dadd(dot3(vv, vv), dmul(sc, sc)));
        const Q o{ddiv(sc, norm), ddiv(vv.x, norm), ddiv(vv.y, norm), ddiv(vv.z, norm)};
        double t[3] = {x[0], x[1], x[2]};
        wrap_inv<3>(g.L, g.invL, t);
        uint32_t m[3] = {0, 0, 0}, cell;
        serial_cell<3>(g, G, t, m);
        bool inf = false, pos = false;
        if (lane_cell<3>(G, m, lane, &cell)) {
            const uint32_t cnt = G.size[cell];
            for (uint32_t kk = 0; kk < cnt && !inf; ++kk) {
                const uint32_t j = G.items[(size_t)cell * G.cap + kk];
                const double4 s4 = G.site[j];
                const double sv[3] = {s4.x, s4.y, s4.z};
                const double4 oj = A.body_ori[j];
                const double e = shape_overlap3(g, sh, so, t, o, sv, Q{oj.x, oj.y, oj.z, oj.w}, capped);
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
            grid_append<3>(g, A, G, T, n, x);
            A.body_ori[n] = make_double4(o.s, o.x, o.y, o.z);
        }
        __syncwarp();
        n++;
        inserted++;
        if (pos) overlapping++;
        if (inserted == q.to_insert || overlapping >= q.allowed) break;
        if (A.stats->error_flags) break;
    }
    if (__any_sync(0xffffffffu, capped != 0u) && lane == 0) atomicOr(&A.stats->error_flags, kErrIterationCap);
    if (lane == 0) {
        out[0] = inserted;
        out[1] = overlapping;
        out[2] = rejected;
        out[3] = n;
    }
}

// Injected moves (position and versor): warp per move, decision in the requested mode.
template <bool FP32>
__global__ void __launch_bounds__(128) k_eval_poly3(Geometry g, Arrays A, PolyShape sh, const uint64_t* bodies,
                                                    const double4* trial, const double4* trial_q, uint32_t n,
                                                    uint8_t* decisions) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    PairStats st;
    if (i < n) {
        const uint32_t k = A.slot_of_body[bodies[i]];
        const double4 w4 = trial[i];
        double t[3] = {w4.x, w4.y, w4.z};
        wrap_inv<3>(g.L, g.invL, t);
        const double4 q4 = trial_q[i];
        const Q qi{q4.x, q4.y, q4.z, q4.w};
        uint32_t m[3];
        uint8_t dec = 0;
        if (point_to_space<3>(g, t, m)) {
            const float4 t32 = FP32 ? cell_offsets<3>(g, t, m) : make_float4(0.f, 0.f, 0.f, 0.f);
            const FlatStencil fs = flat_stencil<3>(g, A.cell_start, m, lane);
            dec = poly_overlaps<FP32>(g, A, sh, t, qi, t32, (int)m[2], fs, k, lane, st) ? 0 : 1;
        } else if (lane == 0) {
            atomicOr(&A.stats->error_flags, kErrOutsideCheckerboard);
        }
        if (lane == 0) decisions[i] = dec;
    }
    flush_stats(A.stats, st, 0u);
}

// Overlapping pairs (i < j), FP64 (the overlap check of total_energy).
__global__ void k_overlap_poly3(Geometry g, Arrays A, PolyShape sh, uint32_t n) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t found = 0;
    if (k < n) {
        const uint32_t bi = A.sorted_body[k];
        const double4 s4 = A.sorted_s[k];
        const double t[3] = {s4.x, s4.y, s4.z};
        const double4 q4 = A.sorted_q[k];
        const Q qi{q4.x, q4.y, q4.z, q4.w};
        uint32_t m[3];
        uint32_t c = A.body_cell[bi];
        for (int a = 2; a >= 0; --a) {
            m[a] = c % g.shape[a];
            c /= g.shape[a];
        }
        for_each_neighbor<3>(g, A.cell_start, m, [&](uint32_t q, const float*) -> bool {
            if (A.sorted_body[q] <= bi) return false;
            const double4 o4 = A.sorted_s[q];
            const double sj[3] = {o4.x, o4.y, o4.z};
            if (poly_overlap64(g, A, sh.verts, sh.nv, sh.rcut2, t, qi, sj, q)) found++;
            return false;
        });
    }
    const unsigned tot = __reduce_add_sync(0xffffffffu, found);
    if ((threadIdx.x & 31) == 0 && tot) atomicAdd(&A.stats->overlaps, (unsigned long long)tot);
}

// Trial moves for the move-size tuner (tune_local.rs:21-89): sample j draws a uniformly random
// body, proposes a move of it and its Metropolis uniform from its own counter stream
// Counter(step, substep, seed).index(2^63 | tune_step << 32 | j). The reference draws all samples
// from one sequential stream; per-sample streams make the samples independent of each other
// and of the sweep's streams, with the same distribution.
template <int DIM>
__global__ void k_tune_moves(Geometry g, Arrays A, Launch L, uint32_t tune_step, uint32_t samples, uint32_t rotate,
                             uint64_t* bodies, double4* trial, double4* trial_q, double* uu) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= samples) return;
    Sfc64 rng = make_rng(L.step, L.substep, L.seed, (1ull << 63) | ((uint64_t)tune_step << 32) | (uint64_t)j);
    const uint32_t b = canon_range_u32(rng, L.n_bodies);
    const double4 b4 = A.body_pos[b];
    double x[3] = {b4.x, b4.y, b4.z};
    Q q{1.0, 0.0, 0.0, 0.0};
    if (A.body_ori) {
        const double4 q4 = A.body_ori[b];
        q = Q{q4.x, q4.y, q4.z, q4.w};
    }
    if (rotate && DIM == 2) {
        // Rotate<Angle>::propose (rotate/angle.rs:46-55): theta += Uniform(-a, a); q.s holds theta
        const double u = dsub(as_double(0x3FF0000000000000ULL | (rng.next_u64() >> 12)), 1.0);
        q.s = dadd(q.s, dadd(dmul(u, dsub(L.max_move, -L.max_move)), -L.max_move));
    } else if (rotate) {
        q = versor_move(rng, L.max_move, A.zig_x, A.zig_f, q);
    } else {
        double dv[3];
        ball_sample<DIM>(rng, L.max_move, A.zig_x, A.zig_f, dv);
        for (int a = 0; a < DIM; ++a) x[a] = dadd(x[a], dv[a]);
    }
    wrap_inv<DIM>(g.L, g.invL, x);
    bodies[j] = b;
    trial[j] = make_double4(x[0], x[1], DIM == 3 ? x[2] : 0.0, 0.0);
    trial_q[j] = make_double4(q.s, q.x, q.y, q.z);
    uu[j] = uniform01(rng);
}

// The sequential-stream tuner for hard convex polyhedra (tune_stream_run): Translate or
// Rotate<Versor> proposals, the trial accepted when XenoCollide finds no overlap with any
// candidate of the stencil around its site's space (FP64, the warp 32 candidates at a time).
__global__ void __launch_bounds__(32) k_tune_stream_poly3(TuneJob* jobs, uint32_t n_jobs, PolyShape sh) {
    if (blockIdx.x >= n_jobs) return;
    TuneJob& J = jobs[blockIdx.x];
    const Geometry& g = J.g;
    const Arrays& A = J.a;
    const uint32_t lane = threadIdx.x & 31u;
    PairStats st;
    tune_stream_run(
        J,
        [&](Sfc64& rng, double m, uint32_t b, double* x, double* q) {
            const double4 q4 = A.body_ori[b];
            Q qi{q4.x, q4.y, q4.z, q4.w};
            if (J.rotate) {
                const double4 b4 = A.body_pos[b];
                x[0] = b4.x;
                x[1] = b4.y;
                x[2] = b4.z;
                qi = versor_move(rng, m, A.zig_x, A.zig_f, qi);
                wrap_inv<3>(g.L, g.invL, x);
            } else {
                tune_translate<3>(rng, g, A, m, b, x);
            }
            q[0] = qi.s;
            q[1] = qi.x;
            q[2] = qi.y;
            q[3] = qi.z;
        },
        [&](Sfc64&, uint32_t b, const double* x, const double* q) -> bool {
            double t[3] = {x[0], x[1], x[2]};
            wrap_inv<3>(g.L, g.invL, t);
            uint32_t m[3] = {0, 0, 0};
            if (!point_to_space<3>(g, t, m)) {
                if (lane == 0) atomicOr(&A.stats->error_flags, kErrOutsideCheckerboard);
                return false;
            }
            const FlatStencil fs = flat_stencil<3>(g, A.cell_start, m, lane);
            const Q qi{q[0], q[1], q[2], q[3]};
            return !poly_overlaps<false>(g, A, sh, t, qi, make_float4(0.f, 0.f, 0.f, 0.f), (int)m[2], fs,
                                         A.slot_of_body[b], lane, st);
        });
}

// Sweep::apply_with_filter (hoomd-mc/src/sweep.rs:159-224) for hard convex polyhedra: one trial
// per body in index order from the one stream Counter(step, substep, seed).make_rng(), Translate
// or Rotate<Versor>, accepted when no site of the serial grid's stencil overlaps it (dH is 0 or
// infinite: no uniform is drawn); one warp, a lane per stencil cell, as for spheres. The pair
// tests read each body's versor by body index.
__global__ void __launch_bounds__(32) k_serial_poly3(Geometry g, Arrays A, SerialGrid G, PolyShape sh, Launch L,
                                                     uint32_t rotate, const uint8_t* __restrict__ mask) {
    const uint32_t lane = threadIdx.x;
    if (A.stats->error_flags) return;
    Arrays Ab = A;
    Ab.sorted_q = A.body_ori;
    Sfc64 rng = make_rng(L.step, L.substep, L.seed, 0);
    uint64_t accepted = 0;
    for (uint32_t b = 0; b < L.n_bodies; ++b) {
        if (mask && !mask[b]) continue;
        const double4 b4 = A.body_pos[b];
        double x[3] = {b4.x, b4.y, b4.z};
        const double4 q4 = A.body_ori[b];
        Q qi{q4.x, q4.y, q4.z, q4.w};
        if (rotate) {
            qi = versor_move(rng, L.max_move, A.zig_x, A.zig_f, qi);
        } else {
            double dv[3];
            ball_sample<3>(rng, L.max_move, A.zig_x, A.zig_f, dv);
            for (int a = 0; a < 3; ++a) x[a] = dadd(x[a], dv[a]);
        }
        wrap_inv<3>(g.L, g.invL, x);  // W1 = wrap(propose(..))
        double t[3] = {x[0], x[1], x[2]};
        wrap_inv<3>(g.L, g.invL, t);  // the trial site T = wrap(W1)
        uint32_t m[3] = {0, 0, 0}, cell;
        serial_cell<3>(g, G, t, m);
        bool overlap = false;
        if (lane_cell<3>(G, m, lane, &cell)) {
            const uint32_t cnt = G.size[cell];
            for (uint32_t k = 0; k < cnt && !overlap; ++k) {
                const uint32_t j = G.items[(size_t)cell * G.cap + k];
                if (j == b) continue;
                const double4 s4 = G.site[j];
                const double sv[3] = {s4.x, s4.y, s4.z};
                overlap = poly_overlap64(g, Ab, sh.verts, sh.nv, sh.rcut2, t, qi, sv, j);
            }
        }
        if (__any_sync(0xffffffffu, overlap)) continue;
        accepted++;
        if (lane == 0) {
            // update_body_properties: body = wrap(W1) = T, site = wrap(body), versor as proposed
            double sv[3] = {t[0], t[1], t[2]};
            wrap_inv<3>(g.L, g.invL, sv);
            A.body_pos[b] = make_double4(t[0], t[1], t[2], 0.0);
            A.body_ori[b] = make_double4(qi.s, qi.x, qi.y, qi.z);
            G.site[b] = make_double4(sv[0], sv[1], sv[2], 0.0);
            serial_move<3>(g, G, A, b, sv);
        }
        __syncwarp();
        if (A.stats->error_flags) break;
    }
    if (lane == 0) {
        A.stats->accepted = accepted;
        A.stats->rechecks = 0;
    }
}

// Proposals for a body at the origin with the identity orientation, proposal i from
// Counter(step, substep, seed).index(i): kind 0 Translate (the displacement), kind 1 Rotate
// (3-D: the versor; 2-D: the angle), kind 2 one StandardNormal draw.
template <int DIM>
__global__ void k_sample_moves(Launch L, uint32_t kind, uint64_t n, const double* zx, const double* zf, double* out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Sfc64 rng = make_rng(L.step, L.substep, L.seed, i);
    if (kind == 2) {
        out[i] = standard_normal(rng, zx, zf);
    } else if (kind == 0) {
        double dv[3];
        ball_sample<DIM>(rng, L.max_move, zx, zf, dv);
        for (int a = 0; a < DIM; ++a) out[i * DIM + a] = dv[a];
    } else if (DIM == 3) {
        const Q q = versor_move(rng, L.max_move, zx, zf, Q{1.0, 0.0, 0.0, 0.0});
        out[i * 4 + 0] = q.s;
        out[i * 4 + 1] = q.x;
        out[i * 4 + 2] = q.y;
        out[i * 4 + 3] = q.z;
    } else {
        const double u = dsub(as_double(0x3FF0000000000000ULL | (rng.next_u64() >> 12)), 1.0);
        out[i] = dadd(0.0, dadd(dmul(u, dsub(L.max_move, -L.max_move)), -L.max_move));
    }
}

}  // namespace

cudaError_t launch_sample_moves(int dim, uint32_t kind, double maximum, uint64_t step, uint32_t substep,
                                uint32_t seed, uint64_t n, const double* zig, double* out, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    Launch l{};
    l.step = step;
    l.substep = substep;
    l.seed = seed;
    l.max_move = maximum;
    const uint32_t blocks = (uint32_t)((n + 127) / 128);
    if (dim == 2)
        k_sample_moves<2><<<blocks, 128, 0, s>>>(l, kind, n, zig, zig + kZigLayers + 1, out);
    else
        k_sample_moves<3><<<blocks, 128, 0, s>>>(l, kind, n, zig, zig + kZigLayers + 1, out);
    return cudaGetLastError();
}

cudaError_t launch_serial_poly(const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv, double rcut2,
                               const Launch& l, bool rotate, const uint32_t* nc, const double* w, uint32_t cap,
                               uint32_t* size, uint32_t* items, uint32_t* cell_of, double4* site, const uint8_t* mask,
                               cudaStream_t s) {
    const SerialGrid G = make_grid(3, nc, w, cap, size, items, cell_of, site);
    cudaError_t e = build_grid(3, g, a, G, l.n_bodies, s);
    if (e != cudaSuccess || l.n_bodies == 0) return e;
    k_serial_poly3<<<1, 32, 0, s>>>(g, a, G, PolyShape{verts, nv, rcut2, 0.f}, l, rotate ? 1u : 0u, mask);
    return cudaGetLastError();
}

cudaError_t launch_propose_poly(bool fp32, const Geometry& g, const Arrays& a, const Launch& l, bool rotate,
                                bool soft, cudaStream_t s) {
    const uint64_t n = (uint64_t)g.color_stride << 3;
    if (n == 0) return cudaSuccess;
    const int wave = resident_wave((const void*)(fp32 ? k_propose_poly3<true> : k_propose_poly3<false>));
    uint32_t blocks = (uint32_t)((n + 127) / 128);
    if (blocks > (uint32_t)wave) blocks = (uint32_t)wave;
    if (fp32)
        k_propose_poly3<true><<<blocks, 128, 0, s>>>(g, a, l, rotate ? 1u : 0u, soft ? 1u : 0u);
    else
        k_propose_poly3<false><<<blocks, 128, 0, s>>>(g, a, l, rotate ? 1u : 0u, soft ? 1u : 0u);
    return cudaGetLastError();
}

cudaError_t launch_sweep_poly3_soft(const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                                    const ShapeOverlap& so, const Launch& l, cudaStream_t s) {
    if (l.n_active == 0) return cudaSuccess;
    PolyShape sh{verts, nv, so.rr, 0.f};
    const int wave = resident_wave((const void*)k_sweep_poly3_soft);
    uint32_t blocks = (l.n_active + 3) / 4;  // four warps (trials) per block
    if (blocks > (uint32_t)wave) blocks = (uint32_t)wave;
    PassLaunch pl(blocks, l.overlap_previous != 0 || l.early_wait != 0, s);
    return cudaLaunchKernelEx(&pl.cfg, k_sweep_poly3_soft, g, a, sh, so, l);
}

cudaError_t launch_energy_poly3_soft(const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                                     const ShapeOverlap& so, uint32_t n, double* out, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    PolyShape sh{verts, nv, so.rr, 0.f};
    k_energy_poly3_soft<<<(n + 127) / 128, 128, 0, s>>>(g, a, sh, so, n, out);
    return cudaGetLastError();
}

cudaError_t launch_quick_insert_poly3(const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                                      const ShapeOverlap& so, const Launch& l, const QuickInsertArgs& q,
                                      const BodyTags& tags, const uint32_t* nc, const double* w, uint32_t cap,
                                      uint32_t* size, uint32_t* items, uint32_t* cell_of, double4* site,
                                      unsigned long long* out, cudaStream_t s) {
    const SerialGrid G = make_grid(3, nc, w, cap, size, items, cell_of, site);
    cudaError_t e = build_grid(3, g, a, G, q.n0, s);
    if (e != cudaSuccess) return e;
    PolyShape sh{verts, nv, so.rr, 0.f};
    k_quick_insert_poly3<<<1, 32, 0, s>>>(g, a, G, sh, so, l, q, tags, out);
    return cudaGetLastError();
}

cudaError_t launch_tune_stream_poly(TuneJob* jobs, uint32_t n_jobs, const double4* verts, uint32_t nv, double rcut2,
                                    cudaStream_t s) {
    if (n_jobs == 0) return cudaSuccess;
    k_tune_stream_poly3<<<n_jobs, 32, 0, s>>>(jobs, n_jobs, PolyShape{verts, nv, rcut2, 0.f});
    return cudaGetLastError();
}

cudaError_t launch_sweep_poly(bool fp32, const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                              double rcut2, float rcut2_hi32, const Launch& l, bool rotate, cudaStream_t s,
                              uint32_t variant) {
    if (l.n_active == 0) return cudaSuccess;
    static int max_blocks = 0;
    if (max_blocks == 0) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        max_blocks = sms * 16;
    }
    PolyShape sh{verts, nv, rcut2, rcut2_hi32};
    const uint32_t per_block = 4u * kPolyShapes[variant < 3 ? variant : 0].trials_per_warp;  // four warps per block
    uint32_t blocks = (l.n_active + per_block - 1) / per_block;
    if (blocks > (uint32_t)max_blocks) blocks = (uint32_t)max_blocks;
    PassLaunch pl(blocks, l.overlap_previous != 0 || l.early_wait != 0, s);
    const uint32_t rot = rotate ? 1u : 0u;
    using PolyKernel = void (*)(Geometry, Arrays, PolyShape, Launch, uint32_t, Injected);
    // the compiled launch variants, in the order of kPolyShapes (trials per warp 4, 2, 8)
    static const PolyKernel kernels[2][3] = {
        {k_sweep_poly3_packed<false, 4>, k_sweep_poly3_packed<false, 2>, k_sweep_poly3_packed<false, 8>},
        {k_sweep_poly3_packed<true, 4>, k_sweep_poly3_packed<true, 2>, k_sweep_poly3_packed<true, 8>}};
    static_assert(n_shapes(kPolyShapes) == 3, "one compiled kernel per polyhedron variant");
    const uint32_t v = variant < 3 ? variant : 0;
    return cudaLaunchKernelEx(&pl.cfg, kernels[fp32][v], g, a, sh, l, rot, Injected{});
}

cudaError_t launch_trials_poly(bool fp32, const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                               double rcut2, float rcut2_hi32, const Injected& j, cudaStream_t s) {
    if (j.n == 0) return cudaSuccess;
    PolyShape sh{verts, nv, rcut2, rcut2_hi32};
    const Launch l{};
    const uint32_t per_block = 4u * kPolyTrialsPerWarp;  // four warps per block
    const uint32_t blocks = (j.n + per_block - 1) / per_block;
    if (fp32)
        k_sweep_poly3_packed<true, kPolyTrialsPerWarp, true><<<blocks, 128, 0, s>>>(g, a, sh, l, 0u, j);
    else
        k_sweep_poly3_packed<false, kPolyTrialsPerWarp, true><<<blocks, 128, 0, s>>>(g, a, sh, l, 0u, j);
    return cudaGetLastError();
}

cudaError_t launch_eval_poly(bool fp32, const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                             double rcut2, float rcut2_hi32, const uint64_t* bodies, const double4* trial,
                             const double4* trial_q, uint32_t n, uint8_t* decisions, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    PolyShape sh{verts, nv, rcut2, rcut2_hi32};
    const uint32_t blocks = (n + 3) / 4;
    if (fp32)
        k_eval_poly3<true><<<blocks, 128, 0, s>>>(g, a, sh, bodies, trial, trial_q, n, decisions);
    else
        k_eval_poly3<false><<<blocks, 128, 0, s>>>(g, a, sh, bodies, trial, trial_q, n, decisions);
    return cudaGetLastError();
}

cudaError_t launch_overlap_poly(const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv, double rcut2,
                                uint32_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    PolyShape sh{verts, nv, rcut2, 0.f};
    k_overlap_poly3<<<(n + 127) / 128, 128, 0, s>>>(g, a, sh, n);
    return cudaGetLastError();
}

}  // namespace hmc

namespace hmc {
cudaError_t launch_tune_moves(int dim, const Geometry& g, const Arrays& a, const Launch& l, uint32_t tune_step,
                              uint32_t samples, bool rotate, uint64_t* bodies, double4* trial, double4* trial_q,
                              double* u, cudaStream_t s) {
    if (samples == 0) return cudaSuccess;
    const uint32_t blocks = (samples + 127) / 128;
    if (dim == 2)
        k_tune_moves<2><<<blocks, 128, 0, s>>>(g, a, l, tune_step, samples, rotate ? 1u : 0u, bodies, trial, trial_q, u);
    else
        k_tune_moves<3><<<blocks, 128, 0, s>>>(g, a, l, tune_step, samples, rotate ? 1u : 0u, bodies, trial, trial_q, u);
    return cudaGetLastError();
}
}  // namespace hmc
