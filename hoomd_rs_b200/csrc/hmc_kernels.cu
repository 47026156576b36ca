// Device kernels of the checkerboard Monte Carlo sweep (sm_100a).
//
// Data layout in HBM (one system):
//   body order : body_pos[n] double4 (B), body_ori[n] double4
//   cell order : sorted_b[n] double4 (B), sorted_s[n] double4 (S = wrap(B)),
//                sorted_off[n] float4 (S - cell corner in FP32, .w = fast-axis cell index),
//                sorted_body[n] u32, cell_start[cells + 1] u32 (CSR over checkerboard spaces)
// The checkerboard spaces of hoomd-mc's HypercuboidCheckerboard are the cells: every
// space is at least one interaction range wide, so a trial body interacts only with
// bodies in the 3^d spaces around its own. Bodies never leave their space during a
// sweep (parallel_sweep.rs:253-258 rejects such moves), so one counting sort per sweep
// keeps the cell order valid for every colour pass of that sweep.
//
// The last axis is the fastest-varying cell index (multi_index_to_index,
// hypercuboid.rs:152-162), so the three spaces of a stencil row along it are adjacent in
// memory and their bodies form one contiguous range of the cell-ordered arrays.
#include <cuda_runtime.h>

#include <mutex>
#include <type_traits>
#include <unordered_map>

#include "hmc_device.cuh"

namespace hmc {
namespace {

// Resident blocks per SM the direct pass is compiled for: 6 caps it at 80 registers,
// which measured fastest on B200 (more resident warps beat the few spilled values).
#ifndef HMC_SWEEP_MIN_BLOCKS
#define HMC_SWEEP_MIN_BLOCKS 6
#endif
// The replica batch pass reads its geometry from the replica table and spilled 320 bytes at
// 80 registers; at 4 blocks per SM (128 registers) it spills nothing: 2.31e9 against 2.28e9
// trial moves/s on 256 boxes (5 blocks: 2.24e9).
#ifndef HMC_BATCH_MIN_BLOCKS
#define HMC_BATCH_MIN_BLOCKS 4
#endif

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// FP64 recheck of a pair whose FP32 d^2 lies inside the bound.
// S of the candidate is wrap(B), recomputed from its body position.
template <int DIM>
__device__ __forceinline__ bool recheck_fp64(const Geometry& g, const Arrays& A, const Pair& P, const double* t,
                                          float dd, uint32_t q, PairStats& st) {
    st.rechecks++;
    double4 b4 = ldg4(A.sorted_b + q);
    double sv[3] = {b4.x, b4.y, b4.z};
    wrap_inv<DIM>(g.L, g.invL, sv);
    double r2 = ref_dist2<DIM>(g, t, sv);
    double e = fabs((double)dd - r2);
    st.max_err = e > st.max_err ? e : st.max_err;
    return r2 < P.sigma2;
}

// FP32 pair decision: certain overlap below sig2_lo32, certain clearance at or above
// sig2_hi32, the reference FP64 test in between.
template <int DIM>
__device__ __forceinline__ bool fp32_pair_overlaps(const Geometry& g, const Arrays& A, const Pair& P,
                                                   const double* t, float dd, uint32_t q, PairStats& st) {
    st.checks++;
    if (dd < P.sig2_lo32) return true;
    if (dd >= P.sig2_hi32) return false;
    return recheck_fp64<DIM>(g, A, P, t, dd, q, st);
}

// Hard-sphere overlap of the trial site t against the stencil of space m, any position of
// m (generic walk). FP32: bounded FP32 test plus FP64 recheck; else the reference FP64 test
// on sorted S.
template <int DIM, bool FP32>
__device__ __forceinline__ bool sphere_overlaps_generic(const Geometry& g, const Arrays& A, const Pair& P,
                                                        const uint32_t* __restrict__ cs, const double* t, float4 t32,
                                                        const uint32_t* m, uint32_t self, PairStats& st) {
    const uint32_t sf = g.shape[DIM - 1];
    const int mf = (int)m[DIM - 1];
    return for_each_neighbor<DIM>(g, cs, m, [&](uint32_t q, const float* slow_shift) -> bool {
        if (q == self) return false;
        if (FP32) {
            float4 o = __ldg(A.sorted_off + q);
            int dm = __float_as_int(o.w) - mf;
            if (sf >= 4) {
                if (dm > 1)
                    dm -= (int)sf;
                else if (dm < -1)
                    dm += (int)sf;
            }
            float dd = fp32_dist2<DIM>(g, t32, o, slow_shift[0], slow_shift[1], dm);
            return fp32_pair_overlaps<DIM>(g, A, P, t, dd, q, st);
        } else {
            double4 s4 = ldg4(A.sorted_s + q);
            double sv[3] = {s4.x, s4.y, s4.z};
            st.checks++;
            return ref_dist2<DIM>(g, t, sv) < P.sigma2;
        }
    });
}

// The same test for a space away from the fast-axis ends, over preloaded row ranges.
// Candidates are taken one per row per step, so the loads of all rows of a step are
// independent and in flight together. Returns kClear, kOverlap, or (FP32 only) kUncertain
// when no pair overlaps for certain but some pair lies inside the FP32 bound; the caller
// then settles the trial in FP64 (sphere_warp_recheck in the colour passes).

template <int DIM, bool FP32>
__device__ __forceinline__ int sphere_overlaps_rows(const Geometry& g, const Arrays& A, const Pair& P,
                                                    const double* t, float4 t32, int mf, uint32_t self,
                                                    const uint32_t* a0, const uint32_t* a1, PairStats& st) {
    constexpr int R = kRows<DIM>;
    bool uncertain = false;
    for (uint32_t k = 0;; ++k) {
        bool any = false;
        if (FP32) {
            float4 v[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                uint32_t q = a0[r] + k;
                bool ok = q < a1[r];
                any |= ok;
                v[r] = ok ? __ldg(A.sorted_off + q) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
            if (!any) return uncertain ? kUncertain : kClear;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                uint32_t q = a0[r] + k;
                if (q < a1[r] && q != self) {
                    int i0 = DIM == 3 ? r / 3 - 1 : 0;
                    int i1 = DIM == 3 ? r % 3 - 1 : r - 1;
                    float s0 = DIM == 3 ? (float)i0 * g.w32[0] : (float)i1 * g.w32[0];
                    float s1 = DIM == 3 ? (float)i1 * g.w32[1] : 0.f;
                    int dm = __float_as_int(v[r].w) - mf;
                    float dd = fp32_dist2<DIM>(g, t32, v[r], s0, s1, dm);
                    st.checks++;
                    if (dd < P.sig2_lo32) return kOverlap;
                    uncertain |= dd < P.sig2_hi32;
                }
            }
        } else {
            double4 v[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                uint32_t q = a0[r] + k;
                bool ok = q < a1[r];
                any |= ok;
                v[r] = ok ? ldg4(A.sorted_s + q) : make_double4(0.0, 0.0, 0.0, 0.0);
            }
            if (!any) return kClear;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                uint32_t q = a0[r] + k;
                if (q < a1[r] && q != self) {
                    double sv[3] = {v[r].x, v[r].y, v[r].z};
                    st.checks++;
                    if (ref_dist2<DIM>(g, t, sv) < P.sigma2) return kOverlap;
                }
            }
        }
    }
}

// The proposal half of a trial (no neighbour data): the stencil's row ranges, the chosen body,
// the trial site and its FP32 offsets.
template <int DIM>
struct SphereProposal {
    uint32_t a0[kRows<DIM>], a1[kRows<DIM>];
    uint32_t k;
    double t[3];
    float4 t32;
};

template <int DIM, bool FP32>
__device__ __forceinline__ bool sphere_propose(const Geometry& g, const Arrays& A, const uint32_t* __restrict__ cs,
                                               const uint32_t* m, uint64_t step, uint32_t substep, uint32_t seed,
                                               double max_move, SphereProposal<DIM>& pr) {
    const uint32_t cell = cell_index<DIM>(g, m);
    const uint32_t sf = g.shape[DIM - 1], mf = m[DIM - 1];
    // The stencil depends only on the space: start its loads before the proposal math.
    uint32_t lo, hi;
    row_span(sf, mf, &lo, &hi);
    load_rows<DIM>(g, cs, m, lo, hi, pr.a0, pr.a1);
    const uint32_t start = __ldg(cs + cell);
    const uint32_t count = __ldg(cs + cell + 1) - start;
    Sfc64 rng = make_rng(step, substep, seed, (uint64_t)cell);
    pr.k = start + canon_range_u32(rng, count);
    double4 b4 = A.sorted_b[pr.k];
    double x[3] = {b4.x, b4.y, b4.z};
    double dv[3];
    ball_sample<DIM>(rng, max_move, A.zig_x, A.zig_f, dv);
#pragma unroll
    for (int a = 0; a < DIM; ++a) x[a] = dadd(x[a], dv[a]);
    wrap_inv<DIM>(g.L, g.invL, x);  // W1 = wrap(propose(..))
    uint32_t mt[3];
    if (!(point_to_space<DIM>(g, x, mt) && cell_index<DIM>(g, mt) == cell)) return false;
    pr.t[0] = x[0];
    pr.t[1] = x[1];
    pr.t[2] = DIM == 3 ? x[2] : 0.0;
    wrap_inv<DIM>(g.L, g.invL, pr.t);  // delta_energy_one wraps the site again: T = wrap(W1)
    pr.t32 = FP32 ? cell_offsets<DIM>(g, pr.t, m) : make_float4(0.f, 0.f, 0.f, 0.f);
    return true;
}

// The proposal half of injected trial i (the colour passes' probe mode): the given W1 in
// place of the drawn one, the walk around W1's own space (the stencil of its body's space when
// W1 stays in it, as in the sweep), self = the body's slot. A W1 outside the body's space is
// flagged (the sweep rejects it before any pair test) and its pair decision still computed.
template <int DIM, bool FP32>
__device__ __forceinline__ bool sphere_inject(const Geometry& g, const Arrays& A, const uint32_t* __restrict__ cs,
                                              const Injected& J, uint32_t i, uint32_t* m, SphereProposal<DIM>& pr,
                                              uint8_t& flag) {
    const uint64_t body = J.bodies[i];
    pr.k = A.slot_of_body[body];
    const double4 w = J.trial[i];
    double x[3] = {w.x, w.y, DIM == 3 ? w.z : 0.0};
    if (!point_to_space<DIM>(g, x, m)) {
        atomicOr(&A.stats->error_flags, kErrOutsideCheckerboard);
        return false;
    }
    if (cell_index<DIM>(g, m) != A.body_cell[body]) flag |= kTrialOutsideSpace;
    uint32_t lo, hi;
    row_span(g.shape[DIM - 1], m[DIM - 1], &lo, &hi);
    load_rows<DIM>(g, cs, m, lo, hi, pr.a0, pr.a1);
    pr.t[0] = x[0];
    pr.t[1] = x[1];
    pr.t[2] = x[2];
    wrap_inv<DIM>(g.L, g.invL, pr.t);  // T = wrap(W1), as delta_energy_one wraps the site
    pr.t32 = FP32 ? cell_offsets<DIM>(g, pr.t, m) : make_float4(0.f, 0.f, 0.f, 0.f);
    return true;
}

// update_body_properties for an accepted move: body = wrap(W1) = T, site = wrap(body).
template <int DIM, bool FP32>
__device__ __forceinline__ void sphere_commit(const Geometry& g, const Arrays& A, const uint32_t* m, uint32_t k,
                                              const double* t) {
    double sv[3] = {t[0], t[1], t[2]};
    wrap_inv<DIM>(g.L, g.invL, sv);
    A.sorted_b[k] = make_double4(t[0], t[1], t[2], 0.0);
    if (!FP32) A.sorted_s[k] = make_double4(sv[0], sv[1], sv[2], 0.0);
    A.sorted_off[k] = cell_offsets<DIM>(g, sv, m);
    A.body_pos[A.sorted_body[k]] = make_double4(t[0], t[1], t[2], 0.0);
}

// The decision half: the candidate walk against the current sites, then update_body_properties.
// Returns kOverlap (rejected) or kClear (accepted and committed); with DEFER_UNCERTAIN it returns
// the walk's result (kUncertain included) and commits nothing; NO_COMMIT settles the trial and
// commits nothing (the probe mode). COMPACT (the replica batch pass,
// whose larger code misses in the instruction cache): one copy of the row walk for both
// segments.
template <int DIM, bool FP32, bool COMPACT = false, bool DEFER_UNCERTAIN = false, bool DEFER_EDGE = false,
          bool NO_COMMIT = false>
__device__ __forceinline__ int sphere_decide_res(const Geometry& g, const Arrays& A, const Pair& P,
                                                 const uint32_t* __restrict__ cs, const uint32_t* m,
                                                 SphereProposal<DIM>& pr, PairStats& st) {
    const uint32_t sf = g.shape[DIM - 1], mf = m[DIM - 1];
    const bool edge = sf > 2 && (mf == 0 || mf + 1 == sf);
    const uint32_t k = pr.k;
    const double* t = pr.t;
    // At a fast-axis end, the wrapped space of each row follows; its stored fast-axis index is
    // sf-1 (mf = 0) or 0 (mf = sf-1), so a virtual mf of sf or -1 gives the cell shift -1 or +1.
    int res;
    if constexpr (COMPACT) {
        // one copy of the row walk for both segments (smaller code)
        res = kClear;
        int mfx = (int)mf;
#pragma unroll 1
        for (int seg = 0; seg < (edge && !DEFER_EDGE ? 2 : 1); ++seg) {
            if (seg == 1) {
                const uint32_t wlo = mf == 0 ? sf - 1u : 0u;
                load_rows<DIM>(g, cs, m, wlo, wlo + 1u, pr.a0, pr.a1);
                mfx = mf == 0 ? (int)sf : -1;
            }
            const int r2 = sphere_overlaps_rows<DIM, FP32>(g, A, P, t, pr.t32, mfx, k, pr.a0, pr.a1, st);
            res = r2 == kOverlap ? kOverlap : (res == kUncertain || r2 == kUncertain ? kUncertain : kClear);
            if (res == kOverlap) break;
        }
    } else {
        res = sphere_overlaps_rows<DIM, FP32>(g, A, P, t, pr.t32, (int)mf, k, pr.a0, pr.a1, st);
        if (!DEFER_EDGE && edge && res != kOverlap) {  // DEFER_EDGE: the caller walks the wrapped rows
            const uint32_t wlo = mf == 0 ? sf - 1u : 0u;
            load_rows<DIM>(g, cs, m, wlo, wlo + 1u, pr.a0, pr.a1);
            int r2 = sphere_overlaps_rows<DIM, FP32>(g, A, P, t, pr.t32, mf == 0 ? (int)sf : -1, k, pr.a0, pr.a1, st);
            res = r2 == kOverlap ? kOverlap : (res == kUncertain || r2 == kUncertain ? kUncertain : kClear);
        }
    }
    if (DEFER_UNCERTAIN) return res;  // the caller settles kUncertain and commits
    if (res == kUncertain) {
        PairStats st2;  // the fast path already counted its pair checks
        const bool ov = sphere_overlaps_generic<DIM, FP32>(g, A, P, cs, t, pr.t32, m, k, st2);
        res = ov ? kOverlap : kClear;
        st.rechecks += st2.rechecks;
        st.max_err = st2.max_err > st.max_err ? st2.max_err : st.max_err;
    }
    if (res == kOverlap) return kOverlap;
    if (!NO_COMMIT) sphere_commit<DIM, FP32>(g, A, m, k, t);
    return kClear;
}

template <int DIM, bool FP32, bool COMPACT = false>
__device__ __forceinline__ bool sphere_decide(const Geometry& g, const Arrays& A, const Pair& P,
                                              const uint32_t* __restrict__ cs, const uint32_t* m,
                                              SphereProposal<DIM>& pr, PairStats& st) {
    return sphere_decide_res<DIM, FP32, COMPACT>(g, A, P, cs, m, pr, st) == kClear;
}

// The FP32 trial of lane src that its own walk left undecided (no certain overlap, some pair
// inside the bound), settled by the whole warp: the lanes take its stencil's candidates 32 at
// a time (FlatStencil) and decide pairs inside the bound in FP64, the same tests as the
// per-lane generic walk but with 32 loads in flight instead of a chain of ~27. Call with every
// lane of the warp; returns whether the trial overlaps.
// WRAPPED_ONLY: only the wrapped rows of a trial at a fast-axis end whose own walk covered the
// rest (the pair checks are counted here).
template <int DIM, bool WRAPPED_ONLY = false>
__device__ __forceinline__ bool sphere_warp_recheck(const Geometry& g, const Arrays& A, const Pair& P,
                                                    const uint32_t* __restrict__ cs, const uint32_t* m,
                                                    const SphereProposal<DIM>& pr, int src, uint32_t lane,
                                                    PairStats& st) {
    const unsigned full = 0xffffffffu;
    uint32_t ms[3];
    double ts[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        ms[a] = __shfl_sync(full, m[a], src);
        ts[a] = __shfl_sync(full, pr.t[a], src);
    }
    const float4 t32 = make_float4(__shfl_sync(full, pr.t32.x, src), __shfl_sync(full, pr.t32.y, src),
                                   __shfl_sync(full, pr.t32.z, src), __shfl_sync(full, pr.t32.w, src));
    const uint32_t self = __shfl_sync(full, pr.k, src);
    const FlatStencil fs = flat_stencil<DIM>(g, cs, ms, lane, WRAPPED_ONLY);
    const uint32_t sf = g.shape[DIM - 1];
    const int mf = (int)ms[DIM - 1];
    for (uint32_t j0 = 0; j0 < fs.total; j0 += 32) {
        const uint32_t j = j0 + lane;
        uint32_t part;
        const uint32_t q = flat_slot(fs, j, part);
        const float s0 = __shfl_sync(full, fs.s0, part), s1 = __shfl_sync(full, fs.s1, part);
        bool hit = false;
        if (j < fs.total && q != self) {
            const float4 o = __ldg(A.sorted_off + q);
            int dm = __float_as_int(o.w) - mf;
            if (sf >= 4) {  // the wrapped space of a row at a fast-axis end
                if (dm > 1)
                    dm -= (int)sf;
                else if (dm < -1)
                    dm += (int)sf;
            }
            const float dd = fp32_dist2<DIM>(g, t32, o, s0, s1, dm);
            if (WRAPPED_ONLY) st.checks++;
            hit = dd < P.sig2_lo32 || (dd < P.sig2_hi32 && recheck_fp64<DIM>(g, A, P, ts, dd, q, st));
        }
        if (__any_sync(full, hit)) return true;
    }
    return false;
}

// ---- the colour pass ------------------------------------------------------------------------
// One thread per non-empty space of the colour: ParallelSweep::generate_trial_moves for that
// space (parallel_sweep.rs:231-278) followed by update_bodies (:283-314) for an accepted move.
// Spaces of one colour are two spaces apart, so the in-place update of an accepted body is
// invisible to every other trial of the colour, as in the reference.
// INJ: the probe mode (Injected): lane i takes injected trial i, runs the same decision code
// and writes its decision instead of committing.
// MINB: resident blocks per SM the pass is compiled for (its register cap), a launch variant
// the autotuner chooses among.
template <int DIM, bool FP32, bool INJ = false, int MINB = HMC_SWEEP_MIN_BLOCKS>
__global__ void __launch_bounds__(128, MINB)
    k_sweep_sphere(Geometry g, Arrays A, Pair P, Launch L, Injected J) {
    if (L.early_wait) grid_dependency_wait();  // first pass: the rebuild's arrays are read at once
    uint32_t n_accepted = 0;
    PairStats st;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t n_active = INJ ? J.n : active_count(A, L.color, L.round);
    if (FP32) {
        // Warp-uniform loop: a trial left undecided by its lane's walk is settled by the whole
        // warp (sphere_warp_recheck). The per-lane generic walk it replaces is a chain of ~27
        // dependent loads; a pass holds a few such trials, and every pass waited for the slowest
        // (2^20 spheres: colour passes 356 -> 333 us per sweep, 3.75e9 -> 3.95e9 trial moves/s).
        const uint32_t lane = threadIdx.x & 31u;
        for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n_active; base += stride) {
            const uint32_t tid = base + lane;
            uint32_t m[3] = {0, 0, 0};
            SphereProposal<DIM> pr;
            bool valid = false;
            uint8_t flag = 0;
            if (tid < n_active) {
                if constexpr (INJ) {
                    valid = sphere_inject<DIM, FP32>(g, A, A.cell_start, J, tid, m, pr, flag);
                } else {
                    unpack_m<DIM>(__ldg(A.color_cells + (size_t)L.color * g.color_stride + tid), m);
                    valid = sphere_propose<DIM, FP32>(g, A, A.cell_start, m, L.step, L.substep, L.seed, L.max_move, pr);
                }
            }
            grid_dependency_wait();  // the previous colour's moves are visible from here on
            allow_dependent_launch();
            int res = kOverlap;  // no trial: nothing to commit
            // 3-D: the wrapped rows of a space at a fast-axis end are walked by the whole warp below
            // (2^20 spheres: colour passes 333 -> 324 us per sweep; in 2-D, with three rows, the
            // lane's own walk is faster: disks 9.6e7 -> 8.4e7 with the warp)
            constexpr bool kWarpEdge = DIM == 3;
            if (valid) res = sphere_decide_res<DIM, FP32, false, true, kWarpEdge>(g, A, P, A.cell_start, m, pr, st);
            unsigned todo = __ballot_sync(0xffffffffu, res == kUncertain);
            while (todo) {
                const int src = __ffs(todo) - 1;
                todo &= todo - 1u;
                const uint32_t r0 = st.rechecks;
                const bool ov = sphere_warp_recheck<DIM>(g, A, P, A.cell_start, m, pr, src, lane, st);
                if constexpr (INJ)
                    if (__any_sync(0xffffffffu, st.rechecks != r0) && (int)lane == src) flag |= kTrialRechecked;
                if ((int)lane == src) res = ov ? kOverlap : kClear;
            }
            if (kWarpEdge) {
                // spaces at a fast-axis end: their wrapped rows, walked by the whole warp
                const uint32_t sf = g.shape[DIM - 1];
                const bool edge = sf > 2 && (m[DIM - 1] == 0 || m[DIM - 1] + 1 == sf);
                unsigned todo2 = __ballot_sync(0xffffffffu, res == kClear && edge);
                while (todo2) {
                    const int src = __ffs(todo2) - 1;
                    todo2 &= todo2 - 1u;
                    const uint32_t r0 = st.rechecks;
                    const bool ov = sphere_warp_recheck<DIM, true>(g, A, P, A.cell_start, m, pr, src, lane, st);
                    if constexpr (INJ)
                        if (__any_sync(0xffffffffu, st.rechecks != r0) && (int)lane == src) flag |= kTrialRechecked;
                    if ((int)lane == src && ov) res = kOverlap;
                }
            }
            if constexpr (INJ) {
                if (tid < n_active) {
                    J.decisions[tid] = valid && res == kClear;
                    J.flags[tid] = flag;
                }
            } else if (res == kClear) {
                sphere_commit<DIM, FP32>(g, A, m, pr.k, pr.t);
                n_accepted++;
            }
        }
        grid_dependency_wait();
        allow_dependent_launch();
        flush_stats(A.stats, st, n_accepted);
        return;
    }
    for (uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x; tid < n_active; tid += stride) {
        uint32_t m[3] = {0, 0, 0};
        SphereProposal<DIM> pr;
        bool valid;
        uint8_t flag = 0;
        if constexpr (INJ) {
            valid = sphere_inject<DIM, FP32>(g, A, A.cell_start, J, tid, m, pr, flag);
        } else {
            unpack_m<DIM>(__ldg(A.color_cells + (size_t)L.color * g.color_stride + tid), m);
            valid = sphere_propose<DIM, FP32>(g, A, A.cell_start, m, L.step, L.substep, L.seed, L.max_move, pr);
        }
        grid_dependency_wait();  // the previous colour's moves are visible from here on
        allow_dependent_launch();
        if constexpr (INJ) {
            const uint32_t r0 = st.rechecks;
            const bool clear =
                valid && sphere_decide_res<DIM, FP32, false, false, false, true>(g, A, P, A.cell_start, m, pr, st) ==
                             kClear;
            J.decisions[tid] = clear;
            J.flags[tid] = flag | (st.rechecks != r0 ? kTrialRechecked : 0);
        } else if (valid && sphere_decide<DIM, FP32>(g, A, P, A.cell_start, m, pr, st)) {
            n_accepted++;
        }
    }
    grid_dependency_wait();
    allow_dependent_launch();
    flush_stats(A.stats, st, n_accepted);
}

// ---- the colour pass, warp-cooperative -------------------------------------------------------
// Each lane proposes the trial of its own space and walks the first kOwnSteps candidates of
// every stencil row itself; most overlapping trials end there. The trials still undecided
// (every accepted trial among them) then have their remaining candidates tested by the
// whole warp, one trial at a time: lane l takes range l % nr at depth l / nr, so a trial's
// ~27 candidates take one or two warp steps instead of a divergent per-lane loop whose
// length is the longest row of any lane. A decision is the OR over its candidates, so the
// order of the tests cannot change it.
#ifndef HMC_COOP_OWN_STEPS
#define HMC_COOP_OWN_STEPS 2
#endif
constexpr int kOwnSteps = HMC_COOP_OWN_STEPS;
constexpr int kFlagOverlap = 1, kFlagUncertain = 2, kFlagMore = 4;

// Candidates k < k_end of every row range; returns kFlagOverlap, or kFlagUncertain and
// kFlagMore (some row has candidates at k >= k_end).
template <int DIM, bool FP32>
__device__ __forceinline__ int sphere_rows_head(const Geometry& g, const Arrays& A, const Pair& P, const double* t,
                                                float4 t32, int mf, uint32_t self, const uint32_t* a0,
                                                const uint32_t* a1, uint32_t k_end, PairStats& st) {
    constexpr int R = kRows<DIM>;
    int flags = 0;
    for (uint32_t k = 0; k < k_end; ++k) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            uint32_t q = a0[r] + k;
            if (q < a1[r] && q != self) {
                st.checks++;
                if (FP32) {
                    float4 v = __ldg(A.sorted_off + q);
                    int i0 = DIM == 3 ? r / 3 - 1 : 0;
                    int i1 = DIM == 3 ? r % 3 - 1 : r - 1;
                    float s0 = DIM == 3 ? (float)i0 * g.w32[0] : (float)i1 * g.w32[0];
                    float s1 = DIM == 3 ? (float)i1 * g.w32[1] : 0.f;
                    float dd = fp32_dist2<DIM>(g, t32, v, s0, s1, __float_as_int(v.w) - mf);
                    if (dd < P.sig2_lo32) return kFlagOverlap;
                    if (dd < P.sig2_hi32) flags |= kFlagUncertain;
                } else {
                    double4 v = ldg4(A.sorted_s + q);
                    double sv[3] = {v.x, v.y, v.z};
                    if (ref_dist2<DIM>(g, t, sv) < P.sigma2) return kFlagOverlap;
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r)
        if (a0[r] + k_end < a1[r]) flags |= kFlagMore;
    return flags;
}

// MINB (register cap) and OWN (candidates per row a lane tests itself) are launch variants.
template <int DIM, bool FP32, bool INJ = false, int MINB = HMC_SWEEP_MIN_BLOCKS, int OWN = kOwnSteps>
__global__ void __launch_bounds__(128, MINB)
    k_sweep_sphere_coop(Geometry g, Arrays A, Pair P, Launch L, Injected J) {
    constexpr int R = kRows<DIM>;
    constexpr int NR = 2 * R;  // row ranges plus, at a fast-axis end, the wrapped spaces
    using Site = typename std::conditional<FP32, float4, double4>::type;
    __shared__ Site s_site[4][32];
    __shared__ uint32_t s_lo[4][32][NR];
    __shared__ uint32_t s_hi[4][32][NR];
    __shared__ int s_mf[4][32][2];
    __shared__ uint32_t s_self[4][32];
    const unsigned full = 0xffffffffu;
    if (L.early_wait) grid_dependency_wait();  // first pass: the rebuild's arrays are read at once
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // this lane's range and depth for a trial with R or 2R ranges
    const uint32_t rA = lane % R, dA = lane / R, rB = lane % NR, dB = lane / NR;
    uint32_t n_accepted = 0;
    PairStats st;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t n_active = INJ ? J.n : active_count(A, L.color, L.round);
    for (uint32_t base = blockIdx.x * blockDim.x + warp * 32; base < n_active; base += stride) {
        const uint32_t tid = base + lane;
        uint32_t m[3] = {0, 0, 0}, cell = 0, k = 0, sf = g.shape[DIM - 1], mf = 0;
        double t[3] = {0.0, 0.0, 0.0};
        float4 t32 = make_float4(0.f, 0.f, 0.f, 0.f);
        int res = kFlagOverlap;  // lanes without a trial in the cell count as decided
        bool edge = false, trial = false;
        uint32_t a0[R], a1[R];
        uint8_t flag = 0;
        if (INJ && tid < n_active) {
            // the probe mode: the injected W1 and the walk around its space (sphere_inject)
            const uint64_t body = J.bodies[tid];
            k = A.slot_of_body[body];
            const double4 w = J.trial[tid];
            const double x[3] = {w.x, w.y, DIM == 3 ? w.z : 0.0};
            if (point_to_space<DIM>(g, x, m)) {
                cell = cell_index<DIM>(g, m);
                if (cell != A.body_cell[body]) flag |= kTrialOutsideSpace;
                mf = m[DIM - 1];
                edge = sf > 2 && (mf == 0 || mf + 1 == sf);
                uint32_t lo, hi;
                row_span(sf, mf, &lo, &hi);
                load_rows<DIM>(g, A.cell_start, m, lo, hi, a0, a1);
                trial = true;
                t[0] = x[0];
                t[1] = x[1];
                t[2] = x[2];
                wrap_inv<DIM>(g.L, g.invL, t);
                if (FP32) t32 = cell_offsets<DIM>(g, t, m);
            } else {
                atomicOr(&A.stats->error_flags, kErrOutsideCheckerboard);
            }
        } else if (tid < n_active) {
            unpack_m<DIM>(__ldg(A.color_cells + (size_t)L.color * g.color_stride + tid), m);
            cell = cell_index<DIM>(g, m);
            mf = m[DIM - 1];
            edge = sf > 2 && (mf == 0 || mf + 1 == sf);
            uint32_t lo, hi;
            row_span(sf, mf, &lo, &hi);
            load_rows<DIM>(g, A.cell_start, m, lo, hi, a0, a1);
            const uint32_t start = __ldg(A.cell_start + cell);
            const uint32_t count = __ldg(A.cell_start + cell + 1) - start;
            Sfc64 rng = make_rng(L.step, L.substep, L.seed, (uint64_t)cell);
            k = start + canon_range_u32(rng, count);
            double4 b4 = A.sorted_b[k];
            double x[3] = {b4.x, b4.y, b4.z};
            double dv[3];
            ball_sample<DIM>(rng, L.max_move, A.zig_x, A.zig_f, dv);
#pragma unroll
            for (int a = 0; a < DIM; ++a) x[a] = dadd(x[a], dv[a]);
            wrap_inv<DIM>(g.L, g.invL, x);  // W1 = wrap(propose(..))
            uint32_t mt[3];
            if (point_to_space<DIM>(g, x, mt) && cell_index<DIM>(g, mt) == cell) {
                trial = true;
                t[0] = x[0];
                t[1] = x[1];
                t[2] = DIM == 3 ? x[2] : 0.0;
                wrap_inv<DIM>(g.L, g.invL, t);  // delta_energy_one wraps the site again: T = wrap(W1)
                if (FP32) t32 = cell_offsets<DIM>(g, t, m);
            }
        }
        grid_dependency_wait();  // the previous colour's moves are visible from here on
        allow_dependent_launch();
        if (trial) {
            res = sphere_rows_head<DIM, FP32>(g, A, P, t, t32, (int)mf, k, a0, a1, (uint32_t)OWN, st);
            if (res != kFlagOverlap && (res & kFlagMore || edge)) {
                // hand the rest to the warp: remaining row ranges, then the wrapped spaces
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    s_lo[warp][lane][r] = a0[r] + (uint32_t)OWN;
                    s_hi[warp][lane][r] = a1[r];
                }
                if (edge) {
                    const uint32_t wlo = mf == 0 ? sf - 1u : 0u;
                    load_rows<DIM>(g, A.cell_start, m, wlo, wlo + 1u, a0, a1);
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        s_lo[warp][lane][R + r] = a0[r];
                        s_hi[warp][lane][R + r] = a1[r];
                    }
                    res |= kFlagMore;
                }
                if constexpr (FP32)
                    s_site[warp][lane] = t32;
                else
                    s_site[warp][lane] = make_double4(t[0], t[1], t[2], 0.0);
                s_mf[warp][lane][0] = (int)mf;
                s_mf[warp][lane][1] = mf == 0 ? (int)sf : -1;
                s_self[warp][lane] = k;
            }
        }
        const unsigned pending = __ballot_sync(full, (res & kFlagMore) != 0);
        const unsigned edges = __ballot_sync(full, edge);
        __syncwarp();
        for (unsigned todo = pending; todo; todo &= todo - 1) {
            const int src = __ffs(todo) - 1;
            const bool wide = (edges >> src) & 1u;
            const uint32_t r = wide ? rB : rA, dep = wide ? dB : dA, per = wide ? 32u / NR : 32u / R;
            const bool mine = dep < per;
            const uint32_t self = s_self[warp][src];
            const uint32_t hi = mine ? s_hi[warp][src][r] : 0u;
            uint32_t q = mine ? s_lo[warp][src][r] + dep : 0u;
            const int mfx = s_mf[warp][src][r < (uint32_t)R ? 0 : 1];
            const Site site = s_site[warp][src];
            int f = 0;
            while (__any_sync(full, q < hi)) {
                if (q < hi && q != self) {
                    st.checks++;
                    if constexpr (FP32) {
                        const float4 t4 = site;
                        float4 v = __ldg(A.sorted_off + q);
                        const int rr = (int)(r % R);
                        int i0 = DIM == 3 ? rr / 3 - 1 : 0;
                        int i1 = DIM == 3 ? rr % 3 - 1 : rr - 1;
                        float s0 = DIM == 3 ? (float)i0 * g.w32[0] : (float)i1 * g.w32[0];
                        float s1 = DIM == 3 ? (float)i1 * g.w32[1] : 0.f;
                        float dd = fp32_dist2<DIM>(g, t4, v, s0, s1, __float_as_int(v.w) - mfx);
                        if (dd < P.sig2_lo32)
                            f |= kFlagOverlap;
                        else if (dd < P.sig2_hi32)
                            f |= kFlagUncertain;
                    } else {
                        const double4 t4 = site;
                        const double tv[3] = {t4.x, t4.y, t4.z};
                        double4 v = ldg4(A.sorted_s + q);
                        double sv[3] = {v.x, v.y, v.z};
                        if (ref_dist2<DIM>(g, tv, sv) < P.sigma2) f |= kFlagOverlap;
                    }
                }
                if (__any_sync(full, f & kFlagOverlap)) break;
                q += per;
            }
            const unsigned ov = __ballot_sync(full, f & kFlagOverlap);
            const unsigned un = __ballot_sync(full, f & kFlagUncertain);
            if (lane == src) res = ov ? kFlagOverlap : ((res & kFlagUncertain) | (un ? kFlagUncertain : 0));
        }
        __syncwarp();
        bool clear = trial && res != kFlagOverlap;
        if (clear && (res & kFlagUncertain)) {
            PairStats st2;  // the fast path already counted its pair checks
            const bool ov = sphere_overlaps_generic<DIM, FP32>(g, A, P, A.cell_start, t, t32, m, k, st2);
            st.rechecks += st2.rechecks;
            st.max_err = st2.max_err > st.max_err ? st2.max_err : st.max_err;
            if (st2.rechecks) flag |= kTrialRechecked;
            if (ov) clear = false;
        }
        if constexpr (INJ) {
            if (tid < n_active) {
                J.decisions[tid] = clear;
                J.flags[tid] = flag;
            }
            continue;
        }
        if (!clear) continue;
        n_accepted++;
        // update_body_properties: body = wrap(W1) = T, site = wrap(body)
        double sv[3] = {t[0], t[1], t[2]};
        wrap_inv<DIM>(g.L, g.invL, sv);
        A.sorted_b[k] = make_double4(t[0], t[1], t[2], 0.0);
        if (!FP32) A.sorted_s[k] = make_double4(sv[0], sv[1], sv[2], 0.0);
        A.sorted_off[k] = cell_offsets<DIM>(g, sv, m);
        A.body_pos[A.sorted_body[k]] = make_double4(t[0], t[1], t[2], 0.0);
    }
    grid_dependency_wait();
    allow_dependent_launch();
    flush_stats(A.stats, st, n_accepted);
}

// ---- cell list rebuild -------------------------------------------------------------------
template <int DIM>
__global__ void k_bin(Geometry g, Arrays A, uint32_t n) {
    allow_dependent_launch();  // the scan may launch; it waits for this kernel to end
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // a pipelined call stopped by an earlier sweep: this sweep's colour passes do nothing
    if (i == 0 && A.abort_word && *A.abort_word != 0u) atomicOr(&A.stats->error_flags, kErrAborted);
    double4 b = A.body_pos[i];
    double x[3] = {b.x, b.y, b.z};
    uint32_t m[3] = {0, 0, 0};
    uint32_t cell = 0;
    bool finite = isfinite(x[0]) && isfinite(x[1]) && (DIM == 2 || isfinite(x[2]));
    if (!finite) {
        atomicOr(&A.stats->error_flags, kErrNonFinite);
    } else if (!point_to_space<DIM>(g, x, m)) {
        atomicOr(&A.stats->error_flags, kErrOutsideCheckerboard);
    } else {
        cell = cell_index<DIM>(g, m);
    }
    A.body_cell[i] = cell;
    A.body_m[i] = pack_m<DIM>(m);
    A.body_rank[i] = atomicAdd(&A.cell_count[cell], 1u);
}

// Exclusive scan over a block of kScanThreads threads (T = uint32_t or packed uint64_t).
template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T* total) {
    __shared__ T warp_sums[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        T w = lane < kScanThreads / 32 ? warp_sums[lane] : T(0);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kScanThreads / 32) warp_sums[lane] = w;
    }
    __syncthreads();
    T warp_prefix = warp > 0 ? warp_sums[warp - 1] : T(0);
    *total = warp_sums[kScanThreads / 32 - 1];
    __syncthreads();
    return warp_prefix + x - v;
}

// The colour of a space: the parity bits of its multi-index, last axis = bit 0, as
// index_to_multi_index(c, [2; N]) in hypercuboid.rs orders the colours.
template <int DIM>
__device__ __forceinline__ uint32_t color_of(const uint32_t* m) {
    uint32_t color = 0;
#pragma unroll
    for (int a = 0; a < DIM; ++a) color = (color << 1) | (m[a] & 1u);
    return color;
}


// Exclusive scan of the space counts into cell_start: per-block totals, then each block's scan
// offset by the sum of the totals before it.
__global__ void __launch_bounds__(kScanThreads) k_count_reduce(const uint32_t* __restrict__ count, uint32_t n_cells,
                                                               uint32_t* block_sums) {
    grid_dependency_wait();  // rebuild kernels run back to back: the previous one has ended here
    allow_dependent_launch();
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) sum += base + k < n_cells ? count[base + k] : 0u;
    sum = __reduce_add_sync(0xffffffffu, sum);
    __shared__ uint32_t warp_sums[kScanThreads / 32];
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
#pragma unroll
        for (int w = 0; w < kScanThreads / 32; ++w) t += warp_sums[w];
        block_sums[blockIdx.x] = t;
    }
}

// Blocks of the count scan up to which each block of k_count_apply sums the earlier blocks'
// totals itself; beyond, k_scan_block_sums scans the totals first (the per-block sums would cost
// O(blocks^2) reads).
constexpr uint32_t kScanDirectBlocks = 2048;

// Exclusive scan of the per-block totals, in place, by one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_scan_block_sums(uint32_t* block_sums, uint32_t nb) {
    grid_dependency_wait();  // rebuild kernels run back to back: the previous one has ended here
    allow_dependent_launch();
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_carry;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < nb; base += 1024) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < nb ? block_sums[i] : 0u;
        uint32_t x = v;
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_warp[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = s_warp[lane];
#pragma unroll
            for (uint32_t o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            s_warp[lane] = w;  // inclusive over the warps
        }
        __syncthreads();
        const uint32_t carry = s_carry;
        const uint32_t excl = carry + (warp > 0 ? s_warp[warp - 1] : 0u) + x - v;
        if (i < nb) block_sums[i] = excl;
        __syncthreads();  // every thread has read s_carry and s_warp
        if (threadIdx.x == 0) s_carry = carry + s_warp[31];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kScanThreads) k_count_apply(const uint32_t* __restrict__ count, uint32_t n_cells,
                                                              const uint32_t* __restrict__ block_sums,
                                                              uint32_t* cell_start, uint32_t scanned) {
    grid_dependency_wait();  // rebuild kernels run back to back: the previous one has ended here
    allow_dependent_launch();
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n_cells ? count[base + k] : 0u;
        sum += v[k];
    }
    // this block's offset: the scanned totals (scanned), else the sum of the earlier blocks'
    // totals, read by every block (at most kScanDirectBlocks values)
    __shared__ uint32_t s_prefix[kScanThreads / 32];
    uint32_t prefix = 0;
    if (scanned) {
        prefix = block_sums[blockIdx.x];
    } else {
        uint32_t part = 0;
        for (uint32_t i = threadIdx.x; i < blockIdx.x; i += kScanThreads) part += block_sums[i];
        part = __reduce_add_sync(0xffffffffu, part);
        if ((threadIdx.x & 31) == 0) s_prefix[threadIdx.x >> 5] = part;
        __syncthreads();
#pragma unroll
        for (int w = 0; w < kScanThreads / 32; ++w) prefix += s_prefix[w];
    }
    uint32_t total;
    uint32_t run = block_exclusive_scan(sum, &total) + prefix;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t c = base + k;
        if (c < n_cells) cell_start[c] = run;
        run += v[k];
        if (c + 1 == n_cells) cell_start[n_cells] = run;
    }
}

// Colour-list positions for one block: each lane with an entry gets a slot in its colour's
// list. Lanes of a warp with the same colour take consecutive slots (shared-memory counters),
// then one global atomic per colour and block reserves the block's run, so each list holds
// runs of neighbouring spaces and the global counters see few atomics. The order within a
// colour does not matter: its trials are independent. Call with every thread of the block.
__device__ __forceinline__ uint32_t append_by_color(DeviceStats* stats, bool has, uint32_t col, uint32_t* s_count,
                                                    uint32_t* s_base) {
    const unsigned full = 0xffffffffu;
    if (threadIdx.x < 8) s_count[threadIdx.x] = 0;
    __syncthreads();
    unsigned todo = __ballot_sync(full, has);
    uint32_t pos = 0;
    while (todo) {
        const int leader = __ffs(todo) - 1;
        const uint32_t cl = __shfl_sync(full, col, leader);
        const unsigned same = __ballot_sync(full, has && col == cl);
        uint32_t base = 0;
        if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(&s_count[cl], (unsigned)__popc(same));
        base = __shfl_sync(full, base, leader);
        if (has && col == cl) pos = base + __popc(same & ((1u << (threadIdx.x & 31)) - 1u));
        todo &= ~same;
    }
    __syncthreads();
    if (threadIdx.x < 8 && s_count[threadIdx.x]) s_base[threadIdx.x] = atomicAdd(&stats->color_count[threadIdx.x], s_count[threadIdx.x]);
    __syncthreads();
    return has ? s_base[col] + pos : 0u;
}

constexpr int kCellThreads = 512;  // 1024: 71.7 us per 2^20-sphere rebuild, 512: 70.7 us

// Per space: order its bodies by index (the order update_checkerboard pushes them,
// parallel_sweep.rs:194-200, which IndexedRandom::choose indexes), and list it under its
// colour when it is not empty.
template <int DIM>
__global__ void __launch_bounds__(kCellThreads) k_cells(Geometry g, Arrays A) {
    grid_dependency_wait();  // rebuild kernels run back to back: the previous one has ended here
    allow_dependent_launch();
    __shared__ uint32_t s_count[8], s_base[8], s_nonempty;
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t s = 0, e = 0;
    if (c < g.n_cells) {
        s = A.cell_start[c];
        e = A.cell_start[c + 1];
        for (uint32_t k = s + 1; k < e; ++k) {
            const uint32_t v = A.sorted_body[k];
            uint32_t j = k;
            while (j > s && A.sorted_body[j - 1] > v) {
                A.sorted_body[j] = A.sorted_body[j - 1];
                --j;
            }
            A.sorted_body[j] = v;
        }
    }
    const bool has = e > s;
    uint32_t packed = 0, col = 0;
    if (has) {
        uint32_t m[3] = {0, 0, 0};
        // the space's multi-index from its index (multi_index_to_index inverted), not from its
        // first body: no dependent gather (rebuild 74.9 -> 73.3 us for 2^20 spheres)
        uint32_t rem = c;
#pragma unroll
        for (int ax = DIM - 1; ax >= 0; --ax) {
            m[ax] = rem % g.shape[ax];
            rem /= g.shape[ax];
        }
        packed = pack_m<DIM>(m);
        col = color_of<DIM>(m);
    }
    if (threadIdx.x == 0) s_nonempty = 0;
    const uint32_t pos = append_by_color(A.stats, has, col, s_count, s_base);
    if (has) A.color_cells[(size_t)col * g.color_stride + pos] = packed;
    const unsigned n_has = __popc(__ballot_sync(0xffffffffu, has));
    if ((threadIdx.x & 31) == 0 && n_has) atomicAdd(&s_nonempty, n_has);
    __syncthreads();
    if (threadIdx.x == 0 && s_nonempty) atomicAdd(&A.stats->nonempty, s_nonempty);
}

// Per cell-order slot: gather B, S = wrap(B) (when WRITE_S), the FP32 offsets of S from its
// space corner and the orientation, and (when WRITE_SLOTS, for the injected-move and tuner
// kernels) the slot of each body; slot 0 also sets the sweep's rounds.
template <int DIM, bool WRITE_S, bool WRITE_SLOTS>
__global__ void k_gather(Geometry g, Arrays A, uint32_t n) {
    grid_dependency_wait();  // rebuild kernels run back to back: the previous one has ended here
    allow_dependent_launch();
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (k == 0) {
        const uint32_t ne = A.stats->nonempty;
        // while count.total() < N: one trial per non-empty space per colour set (:402-418)
        A.stats->rounds = ne == 0 ? 0u : (n + ne - 1) / ne;
    }
    const uint32_t i = A.sorted_body[k];
    if (WRITE_SLOTS) A.slot_of_body[i] = k;
    const double4 b = A.body_pos[i];
    A.sorted_b[k] = b;
    double sv[3] = {b.x, b.y, b.z};
    wrap_inv<DIM>(g.L, g.invL, sv);
    if (WRITE_S) A.sorted_s[k] = make_double4(sv[0], sv[1], sv[2], 0.0);
    uint32_t m[3] = {0, 0, 0};
    unpack_m<DIM>(A.body_m[i], m);
    A.sorted_off[k] = cell_offsets<DIM>(g, sv, m);
    if (A.sorted_q) A.sorted_q[k] = A.body_ori[i];
}

__global__ void k_scatter(Arrays A, uint32_t n) {
    grid_dependency_wait();  // rebuild kernels run back to back: the previous one has ended here
    allow_dependent_launch();
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    A.sorted_body[A.cell_start[A.body_cell[i]] + A.body_rank[i]] = i;
}

// ---- overlap check (PairwiseCutoff::total_energy, pairwise_cutoff.rs:720-745) -------------
template <int DIM>
__global__ void k_overlap_sphere(Geometry g, Arrays A, Pair P, uint32_t n) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t found = 0;
    if (k < n) {
        uint32_t bi = A.sorted_body[k];
        double4 s4 = A.sorted_s[k];
        double t[3] = {s4.x, s4.y, s4.z};
        uint32_t m[3];
        uint32_t c = A.body_cell[bi];
#pragma unroll
        for (int a = DIM - 1; a >= 0; --a) {
            m[a] = c % g.shape[a];
            c /= g.shape[a];
        }
        for_each_neighbor<DIM>(g, A.cell_start, m, [&](uint32_t q, const float*) -> bool {
            uint32_t bj = A.sorted_body[q];
            if (bj <= bi) return false;
            double4 o4 = A.sorted_s[q];
            double sv[3] = {o4.x, o4.y, o4.z};
            if (ref_dist2<DIM>(g, t, sv) < P.sigma2) found++;
            return false;
        });
    }
    unsigned tot = __reduce_add_sync(0xffffffffu, found);
    if ((threadIdx.x & 31) == 0 && tot) atomicAdd(&A.stats->overlaps, (unsigned long long)tot);
}

// ---- pair distributions: scale distribution function and g(r) ------------------------------
// Both histogram the pairs i < j by their minimum-image distance, d = t - s - L rint((t - s)/L)
// per axis, r^2 = sum d^2 (no hoomd-rs counterpart: equilibrium checks of the sweep, the
// pressure from the scale distribution and the radial distribution). SDF: x = 1 - sigma / r, bin floor(x * inv_dx) for x in [0, x_max),
// the scale at which the pair would overlap if the box shrank by (1 - x) (spheres only).
// g(r): bin floor(r * inv_dr) for r < r_max. The walk needs spaces at least as wide as the
// largest distance binned; the host rebuilds the cell list with such a checkerboard first.
template <int DIM>
__device__ __forceinline__ double min_image_dist2(const Geometry& g, const double* t, const double* s) {
    double p = 0.0;
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
        double d = dsub(t[a], s[a]);
        const double k = rint(ddiv(d, g.L[a]));
        d = dsub(d, dmul(k, g.L[a]));
        p = dadd(p, dmul(d, d));
    }
    return p;
}

template <int DIM, bool SDF>
__global__ void __launch_bounds__(256) k_pair_histogram(Geometry g, Arrays A, uint32_t n, double sigma, double limit,
                                                       double inv_width, uint32_t n_bins,
                                                       unsigned long long* counts) {
    extern __shared__ unsigned int s_hist[];
    for (uint32_t b = threadIdx.x; b < n_bins; b += blockDim.x) s_hist[b] = 0;
    __syncthreads();
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) {
        const uint32_t bi = A.sorted_body[k];
        const double4 s4 = A.sorted_s[k];
        const double t[3] = {s4.x, s4.y, s4.z};
        uint32_t m[3] = {0, 0, 0};
        unpack_m<DIM>(A.body_m[bi], m);
        for_each_neighbor<DIM>(g, A.cell_start, m, [&](uint32_t q, const float*) -> bool {
            if (A.sorted_body[q] <= bi) return false;
            const double4 o4 = A.sorted_s[q];
            const double sv[3] = {o4.x, o4.y, o4.z};
            const double r = dsqrt(min_image_dist2<DIM>(g, t, sv));
            double v;
            if (SDF) {
                if (!(r > sigma)) return false;  // overlapping or touching pairs have no positive scale
                v = dsub(1.0, ddiv(sigma, r));
            } else {
                v = r;
            }
            if (v < limit) {
                const double f = floor(dmul(v, inv_width));
                const uint32_t bin = f < (double)n_bins ? (uint32_t)f : n_bins - 1u;
                atomicAdd(&s_hist[bin], 1u);
            }
            return false;
        });
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < n_bins; b += blockDim.x)
        if (s_hist[b]) atomicAdd(counts + b, (unsigned long long)s_hist[b]);
}

// ---- injected moves (delta_energy_one + Metropolis for hard spheres) -----------------------
template <int DIM, bool FP32>
__global__ void k_eval_sphere(Geometry g, Arrays A, Pair P, const uint64_t* bodies, const double4* trial, uint32_t n,
                              uint8_t* decisions, uint8_t* rechecked) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    PairStats st;
    if (i < n) {
        double4 w = trial[i];
        double t[3] = {w.x, w.y, DIM == 3 ? w.z : 0.0};
        wrap_inv<DIM>(g.L, g.invL, t);
        uint32_t m[3];
        bool ok = point_to_space<DIM>(g, t, m);
        uint8_t dec = 0;
        if (ok) {
            uint32_t self = A.slot_of_body[bodies[i]];
            float4 t32 = FP32 ? cell_offsets<DIM>(g, t, m) : make_float4(0.f, 0.f, 0.f, 0.f);
            dec = sphere_overlaps_generic<DIM, FP32>(g, A, P, A.cell_start, t, t32, m, self, st) ? 0 : 1;
        } else {
            atomicOr(&A.stats->error_flags, kErrOutsideCheckerboard);
        }
        decisions[i] = dec;
        rechecked[i] = st.rechecks > 0;
    }
    flush_stats(A.stats, st, 0u);
}

// The sequential-stream tuner for hard spheres (tune_stream_run): a trial is accepted when
// its site overlaps no other site (dH = 0, no uniform drawn) and rejected otherwise (dH = inf).
// The warp takes the stencil around the trial site's space 32 candidates at a time, FP64 pair
// tests on the unchanged state, stopping at the first overlap.
template <int DIM>
__global__ void __launch_bounds__(32) k_tune_stream_sphere(TuneJob* jobs, uint32_t n_jobs) {
    if (blockIdx.x >= n_jobs) return;
    TuneJob& J = jobs[blockIdx.x];
    const Geometry& g = J.g;
    const Arrays& A = J.a;
    const double sigma2 = J.p.sigma2;
    const uint32_t lane = threadIdx.x & 31u;
    tune_stream_run(
        J, [&](Sfc64& rng, double m, uint32_t b, double* x, double*) { tune_translate<DIM>(rng, g, A, m, b, x); },
        [&](Sfc64&, uint32_t b, const double* x, const double*) -> bool {
            double t[3] = {x[0], x[1], x[2]};
            wrap_inv<DIM>(g.L, g.invL, t);  // the site of the trial body
            uint32_t m[3] = {0, 0, 0};
            if (!point_to_space<DIM>(g, t, m)) {
                if (lane == 0) atomicOr(&A.stats->error_flags, kErrOutsideCheckerboard);
                return false;
            }
            const uint32_t self = A.slot_of_body[b];
            const FlatStencil fs = flat_stencil<DIM>(g, A.cell_start, m, lane);
            for (uint32_t j0 = 0; j0 < fs.total; j0 += 32) {
                uint32_t part;
                const uint32_t q = flat_slot(fs, j0 + lane, part);
                bool hit = false;
                if (j0 + lane < fs.total && q != self) {
                    const double4 s4 = ldg4(A.sorted_s + q);
                    const double sv[3] = {s4.x, s4.y, s4.z};
                    hit = ref_dist2<DIM>(g, t, sv) < sigma2;
                }
                if (__any_sync(0xffffffffu, hit)) return false;
            }
            return true;
        });
}

template <typename T>
inline uint32_t blocks_for(T n, uint32_t threads) {
    return (uint32_t)((n + threads - 1) / threads);
}

// ---- batches of replicas -------------------------------------------------------------------
// The spaces of all replicas form one CSR (replica r's spaces start at cell_base[r]) and the
// colour lists hold every replica's non-empty spaces of a colour, tagged with the replica.
// Each replica keeps its own box, checkerboard and Counter, so every replica's trajectory is
// the one its own system would produce; one launch serves all replicas.

template <int DIM>
__global__ void k_bin_batch(Batch B, Arrays A, uint32_t n) {
    allow_dependent_launch();  // the scan may launch; it waits for this kernel to end
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Replica& R = B.rep[__ldg(B.body_rep + i)];
    const double4 b = A.body_pos[i];
    double x[3] = {b.x, b.y, b.z};
    uint32_t m[3] = {0, 0, 0};
    uint32_t cell = R.cell_base;
    const bool finite = isfinite(x[0]) && isfinite(x[1]) && (DIM == 2 || isfinite(x[2]));
    if (!finite)
        atomicOr(&A.stats->error_flags, kErrNonFinite);
    else if (!point_to_space<DIM>(R.g, x, m))
        atomicOr(&A.stats->error_flags, kErrOutsideCheckerboard);
    else
        cell += cell_index<DIM>(R.g, m);
    A.body_cell[i] = cell;
    A.body_m[i] = pack_m<DIM>(m);
    A.body_rank[i] = atomicAdd(&A.cell_count[cell], 1u);
}





template <int DIM>
__global__ void __launch_bounds__(kCellThreads) k_cells_batch(Batch B, Arrays A) {
    grid_dependency_wait();  // rebuild kernels run back to back: the previous one has ended here
    allow_dependent_launch();
    __shared__ uint32_t s_count[8], s_base[8], s_nonempty;
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t s = 0, e = 0;
    if (c < B.n_cells) {
        s = A.cell_start[c];
        e = A.cell_start[c + 1];
        for (uint32_t k = s + 1; k < e; ++k) {
            const uint32_t v = A.sorted_body[k];
            uint32_t j = k;
            while (j > s && A.sorted_body[j - 1] > v) {
                A.sorted_body[j] = A.sorted_body[j - 1];
                --j;
            }
            A.sorted_body[j] = v;
        }
    }
    const bool has = e > s;
    uint32_t packed = 0, col = 0, r = 0xffffffffu;
    if (has) {
        const uint32_t first = A.sorted_body[s];
        packed = A.body_m[first];
        r = __ldg(B.body_rep + first);
        uint32_t m[3] = {0, 0, 0};
        unpack_m<DIM>(packed, m);
        col = color_of<DIM>(m);
    }
    if (threadIdx.x == 0) s_nonempty = 0;
    const uint32_t pos = append_by_color(A.stats, has, col, s_count, s_base);
    if (has) {
        const size_t entry = (size_t)col * B.color_stride + pos;
        A.color_cells[entry] = packed;
        B.color_rep[entry] = r;
    }
    const unsigned n_has = __popc(__ballot_sync(0xffffffffu, has));
    if ((threadIdx.x & 31) == 0 && n_has) atomicAdd(&s_nonempty, n_has);
    __syncthreads();
    if (threadIdx.x == 0 && s_nonempty) atomicAdd(&A.stats->nonempty, s_nonempty);
    // non-empty spaces per replica, one atomic per replica present in the warp
    const unsigned full = 0xffffffffu;
    unsigned todo = __ballot_sync(full, has);
    while (todo) {
        const int leader = __ffs(todo) - 1;
        const uint32_t rl = __shfl_sync(full, r, leader);
        const unsigned same = __ballot_sync(full, has && r == rl);
        if ((int)(threadIdx.x & 31) == leader) atomicAdd(B.nonempty + rl, (unsigned)__popc(same));
        todo &= ~same;
    }
}

template <int DIM, bool WRITE_S>
__global__ void k_gather_batch(Batch B, Arrays A, uint32_t n) {
    grid_dependency_wait();  // rebuild kernels run back to back: the previous one has ended here
    allow_dependent_launch();
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t i = A.sorted_body[k];
    const Geometry& g = B.rep[__ldg(B.body_rep + i)].g;  // (no batch kernel reads slot_of_body)
    const double4 b = A.body_pos[i];
    A.sorted_b[k] = b;
    double sv[3] = {b.x, b.y, b.z};
    wrap_inv<DIM>(g.L, g.invL, sv);
    if (WRITE_S) A.sorted_s[k] = make_double4(sv[0], sv[1], sv[2], 0.0);
    uint32_t m[3] = {0, 0, 0};
    unpack_m<DIM>(A.body_m[i], m);
    A.sorted_off[k] = cell_offsets<DIM>(g, sv, m);
}

// Accepted moves per replica from one warp: the lanes of each replica in the warp add up.
__device__ __forceinline__ void add_per_replica(unsigned long long* acc, uint32_t r, bool accepted) {
    const unsigned full = 0xffffffffu;
    unsigned todo = full;
    while (todo) {
        const int leader = __ffs(todo) - 1;
        const uint32_t rl = __shfl_sync(full, r, leader);
        const unsigned same = __ballot_sync(full, r == rl);
        const unsigned n = __popc(__ballot_sync(full, r == rl && accepted));
        if ((threadIdx.x & 31) == (unsigned)leader && n) atomicAdd(acc + rl, (unsigned long long)n);
        todo &= ~same;
    }
}

// One colour pass over all replicas that still run round `round` of this sweep.
template <int DIM, bool FP32, int MINB = HMC_BATCH_MIN_BLOCKS>
__global__ void __launch_bounds__(128, MINB) k_sweep_batch(Batch B, Arrays A, uint32_t color,
                                                                             uint32_t round, uint32_t early_wait) {
    if (early_wait) grid_dependency_wait();  // first pass: the rebuild's arrays are read at once
    if (round == kRoundFromDevice) round = *B.round_dev;  // a captured sweep's rounds loop
    const uint32_t n_active = active_count(A, color, round);
    uint32_t n_accepted = 0;
    PairStats st;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n_active; base += stride) {
        const uint32_t tid = base + (threadIdx.x & 31u);
        bool accepted = false, valid = false;
        uint32_t r = 0xffffffffu;
        uint32_t m[3] = {0, 0, 0};
        SphereProposal<DIM> pr;
        if (tid < n_active) {
            const size_t e = (size_t)color * B.color_stride + tid;
            r = __ldg(B.color_rep + e);
            const Replica& R = B.rep[r];
            if (round < R.rounds) {
                unpack_m<DIM>(__ldg(A.color_cells + e), m);
                valid = sphere_propose<DIM, FP32>(R.g, A, A.cell_start + R.cell_base, m, R.step, R.substep + round,
                                                  R.seed, R.max_move, pr);
            }
        }
        grid_dependency_wait();  // the previous colour's moves are visible from here on
        allow_dependent_launch();
        // FP32: undecided trials settled by the whole warp (sphere_warp_recheck), then committed
        // (256 boxes: 2.29e9 -> 2.51e9 trial moves/s against the per-lane generic walk)
        int res = kOverlap;
        // 3-D FP32: wrapped rows of end spaces walked by the warp, as in the single-box pass
        // (256 boxes: 2.53e9 -> 2.56e9 trial moves/s)
        constexpr bool kWarpEdge = FP32 && DIM == 3;
        if (valid) {
            const Replica& R = B.rep[r];
            res = sphere_decide_res<DIM, FP32, true, FP32, kWarpEdge>(R.g, A, R.p, A.cell_start + R.cell_base, m, pr,
                                                                       st);
        }
        if (FP32) {
            const uint32_t lane = threadIdx.x & 31u;
            unsigned todo = __ballot_sync(0xffffffffu, res == kUncertain);
            while (todo) {
                const int src = __ffs(todo) - 1;
                todo &= todo - 1u;
                const Replica& RS = B.rep[__shfl_sync(0xffffffffu, r, src)];
                const bool ov = sphere_warp_recheck<DIM>(RS.g, A, RS.p, A.cell_start + RS.cell_base, m, pr, src, lane, st);
                if ((int)lane == src) res = ov ? kOverlap : kClear;
            }
            if (kWarpEdge) {
                // spaces at a fast-axis end: their wrapped rows, walked by the whole warp
                bool edge = false;
                if (valid) {
                    const uint32_t sf = B.rep[r].g.shape[DIM - 1];
                    edge = sf > 2 && (m[DIM - 1] == 0 || m[DIM - 1] + 1 == sf);
                }
                unsigned todo2 = __ballot_sync(0xffffffffu, res == kClear && edge);
                while (todo2) {
                    const int src = __ffs(todo2) - 1;
                    todo2 &= todo2 - 1u;
                    const Replica& RS = B.rep[__shfl_sync(0xffffffffu, r, src)];
                    const bool ov = sphere_warp_recheck<DIM, true>(RS.g, A, RS.p, A.cell_start + RS.cell_base, m, pr,
                                                                   src, lane, st);
                    if ((int)lane == src && ov) res = kOverlap;
                }
            }
            if (res == kClear) sphere_commit<DIM, FP32>(B.rep[r].g, A, m, pr.k, pr.t);
        }
        accepted = res == kClear;
        n_accepted += accepted;
        add_per_replica(B.accepted, r, accepted);
    }
    grid_dependency_wait();
    allow_dependent_launch();
    flush_stats(A.stats, st, n_accepted);
}

// update_checkerboard's origin shift (parallel_sweep.rs:176-190) for every replica from its own
// Counter's index u64::MAX stream: the host's computation, on the device.
template <int DIM>
__global__ void k_batch_origins(Batch B, Replica* rep) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= B.n_replicas) return;
    Replica& R = rep[r];
    Sfc64 rng = make_rng(R.step, R.substep, R.seed, UINT64_MAX);
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
        const double off = uniform01(rng);
        R.g.origin[a] = dsub(-R.g.L[a] / 2.0, dmul(off, R.g.width[a]));
    }
}

// The first test of a captured sweep's rounds loop: colour set 0 runs when some replica has a
// round and no earlier sweep of the call (nor this sweep's rebuild) flagged an error.
__global__ void k_batch_round_first(cudaGraphConditionalHandle h, const DeviceStats* stats, uint32_t* round_dev,
                                    const BatchSweepTotals* totals) {
    *round_dev = 0;
    cudaGraphSetConditional(h, stats->rounds > 0u && stats->error_flags == 0u && totals->error_flags == 0u);
}

// The end of one colour set of a captured sweep: the next runs while the sweep has rounds left.
__global__ void k_batch_round_next(cudaGraphConditionalHandle h, const DeviceStats* stats, uint32_t* round_dev) {
    const uint32_t next = *round_dev + 1u;
    *round_dev = next;
    cudaGraphSetConditional(h, next < stats->rounds);
}

// The host's bookkeeping after a batch sweep, on the device: per replica its trials
// (rounds x non-empty spaces) split into accepted and rejected, and its Counter
// (increment_substep per colour set, then increment_step); for the batch the sweep's statistics.
// A sweep whose rebuild flagged an error (or that follows one) ran no pass and changes nothing
// but the flags.
__global__ void k_batch_sweep_end(Batch B, Replica* rep, const DeviceStats* stats, unsigned long long* rep_counts,
                                  BatchSweepTotals* totals, uint32_t increment_step) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    // (thread 0 adds only this sweep's flags, which every thread reads itself)
    const bool failed = stats->error_flags != 0u || totals->error_flags != 0u;
    if (r == 0) {
        totals->error_flags |= stats->error_flags;
        if (!failed) {
            totals->rechecks += stats->rechecks;
            totals->pair_checks += stats->pair_checks;
            totals->ambiguous += stats->ambiguous;
            if (stats->max_err_bits > totals->max_err_bits) totals->max_err_bits = stats->max_err_bits;
            totals->sweeps += 1;
            totals->colour_sets += stats->rounds;
        }
    }
    if (failed || r >= B.n_replicas) return;
    Replica& R = rep[r];
    const unsigned long long acc = B.accepted[r];
    const unsigned long long trials = (unsigned long long)R.rounds * B.nonempty[r];
    rep_counts[2 * r] += acc;
    rep_counts[2 * r + 1] += trials - acc;
    R.substep += R.rounds;
    if (increment_step) {
        R.step += 1;
        R.substep = 0;
    }
}

// Rounds of every replica (ceil(N_r / non-empty spaces of r)) and their maximum.
__global__ void k_batch_rounds(Batch B, Replica* rep, DeviceStats* stats) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= B.n_replicas) return;
    const uint32_t n = rep[r].n_bodies, ne = B.nonempty[r];
    const uint32_t rounds = (n == 0 || ne == 0) ? 0u : (n + ne - 1) / ne;
    rep[r].rounds = rounds;
    atomicMax(&stats->rounds, rounds);
}

// Overlapping pairs (i < j) of every replica, FP64.
template <int DIM>
__global__ void k_overlap_batch(Batch B, Arrays A, uint32_t n) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t bi = A.sorted_body[k];
    const uint32_t r = __ldg(B.body_rep + bi);
    const Replica& R = B.rep[r];
    const double4 s4 = A.sorted_s[k];
    const double t[3] = {s4.x, s4.y, s4.z};
    uint32_t m[3] = {0, 0, 0};
    uint32_t c = A.body_cell[bi] - R.cell_base;
#pragma unroll
    for (int a = DIM - 1; a >= 0; --a) {
        m[a] = c % R.g.shape[a];
        c /= R.g.shape[a];
    }
    uint32_t found = 0;
    for_each_neighbor<DIM>(R.g, A.cell_start + R.cell_base, m, [&](uint32_t q, const float*) -> bool {
        if (A.sorted_body[q] <= bi) return false;
        const double4 o4 = A.sorted_s[q];
        const double sv[3] = {o4.x, o4.y, o4.z};
        if (ref_dist2<DIM>(R.g, t, sv) < R.p.sigma2) found++;
        return false;
    });
    if (found) atomicAdd(B.overlaps + r, (unsigned long long)found);
}

// ---- state transfer ------------------------------------------------------------------
__global__ void k_check_finite(const double* __restrict__ packed, uint64_t count, uint32_t dim,
                               unsigned long long* first_nonfinite) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count;
         i += (uint64_t)gridDim.x * blockDim.x) {
        if (!isfinite(packed[i])) atomicMin(first_nonfinite, (unsigned long long)(i / dim));
    }
}

template <int DIM>
__global__ void k_unpack_positions(const double* __restrict__ packed, double4* __restrict__ body_pos, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const double* p = packed + i * DIM;
        body_pos[i] = make_double4(p[0], p[1], DIM == 3 ? p[2] : 0.0, 0.0);
    }
}

template <int DIM>
__global__ void k_pack_positions(const double4* __restrict__ body_pos, double* __restrict__ packed, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        double4 b = body_pos[i];
        double* p = packed + i * DIM;
        p[0] = b.x;
        p[1] = b.y;
        if (DIM == 3) p[2] = b.z;
    }
}

__global__ void k_check_angles(const double* __restrict__ packed, uint64_t n, unsigned long long* first_bad) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const double t = packed[i];
        if (!(fabs(t) < 524288.0)) atomicMin(first_bad, (unsigned long long)i);
    }
}

__global__ void k_unpack_angles(const double* __restrict__ packed, double4* __restrict__ body_ori, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        body_ori[i] = make_double4(packed[i], 0.0, 0.0, 0.0);
}

__global__ void k_pack_angles(const double4* __restrict__ body_ori, double* __restrict__ packed, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        packed[i] = body_ori[i].x;
}

// GSD frames (hoomd-microstate/src/append.rs:46-113): FP32 site positions and orientations in
// tag (body) order. A single-site body's site is wrap(B + rotate(0)): the added vector is a zero
// of either sign, and wrap maps a zero of either sign to +0, so the site is wrap(B) bit for bit.
// The site versor is combine(q, identity) (quaternion.rs:408-415, 771-776) evaluated as written,
// which keeps the reference's signs of zero components. In 2-D the site angle is theta + 0.0
// and the written versor is from_axis_angle(z, theta) = (cos(t/2), 0 sin(t/2), 0 sin(t/2),
// sin(t/2)) (quaternion.rs:560-567), with correctly rounded sin and cos. FP32 values are the
// FP64 values rounded to nearest (Rust `as f32`).
template <int DIM, int ORI>
__global__ void k_gsd_encode(Geometry g, const double4* __restrict__ body_pos, const double4* __restrict__ body_ori,
                             uint64_t n, float* __restrict__ pos, float* __restrict__ ori) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const double4 b = body_pos[i];
        double s[3] = {b.x, b.y, b.z};
        wrap_inv<DIM>(g.L, g.invL, s);
        pos[3 * i + 0] = __double2float_rn(s[0]);
        pos[3 * i + 1] = __double2float_rn(s[1]);
        pos[3 * i + 2] = DIM == 3 ? __double2float_rn(s[2]) : 0.0f;
        if (ORI == 1) {
            const double4 q = body_ori[i];
            const double v[3] = {q.y, q.z, q.w};
            const double zero[3] = {0.0, 0.0, 0.0};
            const double sc = dsub(dmul(q.x, 1.0), dot<3>(v, zero));
            const double c[3] = {dsub(dmul(v[1], 0.0), dmul(v[2], 0.0)), dsub(dmul(v[2], 0.0), dmul(v[0], 0.0)),
                                 dsub(dmul(v[0], 0.0), dmul(v[1], 0.0))};
            ori[4 * i + 0] = __double2float_rn(sc);
#pragma unroll
            for (int a = 0; a < 3; ++a)
                ori[4 * i + 1 + a] = __double2float_rn(dadd(dadd(dmul(0.0, q.x), dmul(v[a], 1.0)), c[a]));
        } else if (ORI == 2) {
            const double half = ddiv(dadd(body_ori[i].x, 0.0), 2.0);
            double sn, cs;
            cr_sincos(half, &sn, &cs);  // |half| < 2^18: angles are checked on upload
            ori[4 * i + 0] = __double2float_rn(cs);
            ori[4 * i + 1] = __double2float_rn(dmul(0.0, sn));
            ori[4 * i + 2] = __double2float_rn(dmul(0.0, sn));
            ori[4 * i + 3] = __double2float_rn(dmul(1.0, sn));
        }
    }
}

// Microstate::clone_with_boundary (hoomd-microstate/src/microstate.rs:1529-1565) for a
// periodic hypercuboid: Hypercuboid::map_point (hoomd-geometry/src/shape/cuboid.rs:553-565)
// checks -L/2 <= x < L/2 in the old box, scales by L'/L and clamps to [-L'/2, next_down(L'/2)];
// update_body_properties then keeps B = wrap(.) in the new box.
template <int DIM>
__global__ void k_map_bodies(Geometry g, double3 old_half, double3 scale, double3 lo, double3 hi,
                             double4* __restrict__ body_pos, uint64_t n, unsigned long long* first_outside) {
    const double oh[3] = {old_half.x, old_half.y, old_half.z}, sc[3] = {scale.x, scale.y, scale.z};
    const double l[3] = {lo.x, lo.y, lo.z}, h[3] = {hi.x, hi.y, hi.z};
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const double4 b = body_pos[i];
        double x[3] = {b.x, b.y, b.z};
        bool inside = true;
#pragma unroll
        for (int a = 0; a < DIM; ++a) inside = inside && -oh[a] <= x[a] && x[a] < oh[a];
        if (!inside) {
            atomicMin(first_outside, (unsigned long long)i);
            continue;
        }
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
            double y = dmul(sc[a], x[a]);
            if (y < l[a]) y = l[a];  // f64::clamp
            if (y > h[a]) y = h[a];
            x[a] = y;
        }
        wrap_inv<DIM>(g.L, g.invL, x);
        body_pos[i] = make_double4(x[0], x[1], DIM == 3 ? x[2] : 0.0, 0.0);
    }
}

inline uint32_t stream_grid(uint64_t n) {
    uint64_t b = (n + 255) / 256;
    return (uint32_t)(b < 148ull * 16 ? (b ? b : 1) : 148ull * 16);
}

}  // namespace

cudaError_t launch_check_finite(const double* packed, uint64_t count, uint32_t dim,
                                unsigned long long* first_nonfinite, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    k_check_finite<<<stream_grid(count), 256, 0, s>>>(packed, count, dim, first_nonfinite);
    return cudaGetLastError();
}

cudaError_t launch_unpack_positions(int dim, const double* packed, double4* body_pos, uint64_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    if (dim == 2)
        k_unpack_positions<2><<<stream_grid(n), 256, 0, s>>>(packed, body_pos, n);
    else
        k_unpack_positions<3><<<stream_grid(n), 256, 0, s>>>(packed, body_pos, n);
    return cudaGetLastError();
}

cudaError_t launch_pack_positions(int dim, const double4* body_pos, double* packed, uint64_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    if (dim == 2)
        k_pack_positions<2><<<stream_grid(n), 256, 0, s>>>(body_pos, packed, n);
    else
        k_pack_positions<3><<<stream_grid(n), 256, 0, s>>>(body_pos, packed, n);
    return cudaGetLastError();
}

cudaError_t launch_check_angles(const double* packed, uint64_t n, unsigned long long* first_bad, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_check_angles<<<stream_grid(n), 256, 0, s>>>(packed, n, first_bad);
    return cudaGetLastError();
}

cudaError_t launch_unpack_angles(const double* packed, double4* body_ori, uint64_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_unpack_angles<<<stream_grid(n), 256, 0, s>>>(packed, body_ori, n);
    return cudaGetLastError();
}

cudaError_t launch_pack_angles(const double4* body_ori, double* packed, uint64_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_pack_angles<<<stream_grid(n), 256, 0, s>>>(body_ori, packed, n);
    return cudaGetLastError();
}

cudaError_t launch_map_bodies(int dim, const Geometry& g_new, const double* old_half, const double* scale,
                              const double* lo, const double* hi, double4* body_pos, uint64_t n,
                              unsigned long long* first_outside, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const double3 oh = make_double3(old_half[0], old_half[1], old_half[2]);
    const double3 sc = make_double3(scale[0], scale[1], scale[2]);
    const double3 l = make_double3(lo[0], lo[1], lo[2]), h = make_double3(hi[0], hi[1], hi[2]);
    if (dim == 2)
        k_map_bodies<2><<<stream_grid(n), 256, 0, s>>>(g_new, oh, sc, l, h, body_pos, n, first_outside);
    else
        k_map_bodies<3><<<stream_grid(n), 256, 0, s>>>(g_new, oh, sc, l, h, body_pos, n, first_outside);
    return cudaGetLastError();
}

cudaError_t launch_gsd_encode(int dim, int ori_kind, const Geometry& g, const double4* body_pos,
                              const double4* body_ori, uint64_t n, float* pos, float* ori, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const uint32_t grid = stream_grid(n);
    if (dim == 2) {
        if (ori_kind == 2)
            k_gsd_encode<2, 2><<<grid, 256, 0, s>>>(g, body_pos, body_ori, n, pos, ori);
        else
            k_gsd_encode<2, 0><<<grid, 256, 0, s>>>(g, body_pos, body_ori, n, pos, ori);
    } else {
        if (ori_kind == 1)
            k_gsd_encode<3, 1><<<grid, 256, 0, s>>>(g, body_pos, body_ori, n, pos, ori);
        else
            k_gsd_encode<3, 0><<<grid, 256, 0, s>>>(g, body_pos, body_ori, n, pos, ori);
    }
    return cudaGetLastError();
}

namespace {
// Rebuild kernels after the first launch back to back with programmatic dependent launch:
// each waits for its predecessor at its start, so only the launch latency overlaps.
template <typename... K, typename... A>
cudaError_t launch_chained(void (*kernel)(K...), uint32_t grid, uint32_t block, bool chained, cudaStream_t s,
                           A... args) {
    PassLaunch pl(grid, chained, s, block);
    return cudaLaunchKernelEx(&pl.cfg, kernel, args...);
}

cudaError_t launch_count_scan(const Arrays& a, uint32_t n_cells, cudaStream_t s, bool chained = true) {
    const uint32_t nb = blocks_for(n_cells, kScanTile);
    cudaError_t e = launch_chained(k_count_reduce, nb, kScanThreads, chained, s, (const uint32_t*)a.cell_count,
                                   n_cells, a.block_sums);
    const uint32_t scanned = nb > kScanDirectBlocks ? 1u : 0u;
    if (e == cudaSuccess && scanned) e = launch_chained(k_scan_block_sums, 1, 1024, true, s, a.block_sums, nb);
    if (e == cudaSuccess)
        e = launch_chained(k_count_apply, nb, kScanThreads, true, s, (const uint32_t*)a.cell_count, n_cells,
                           (const uint32_t*)a.block_sums, a.cell_start, scanned);
    return e;
}
}  // namespace

// Threads per block of the rebuild's per-body kernels (k_bin, k_scatter, k_gather).
#ifndef HMC_BODY_THREADS
#define HMC_BODY_THREADS 256
#endif
constexpr uint32_t kBodyThreads = HMC_BODY_THREADS;

cudaError_t launch_rebuild(int dim, const Geometry& g, const Arrays& a, uint32_t n, bool write_s, cudaStream_t s,
                           bool write_slots) {
    cudaError_t e = cudaMemsetAsync(a.cell_count, 0, sizeof(uint32_t) * g.n_cells, s);
    if (e != cudaSuccess) return e;
    if (n > 0) {
        if (dim == 2)
            k_bin<2><<<blocks_for(n, kBodyThreads), kBodyThreads, 0, s>>>(g, a, n);
        else
            k_bin<3><<<blocks_for(n, kBodyThreads), kBodyThreads, 0, s>>>(g, a, n);
    }
    if ((e = launch_count_scan(a, g.n_cells, s, n > 0)) != cudaSuccess) return e;
    if (n == 0) return cudaSuccess;
    if ((e = launch_chained(k_scatter, blocks_for(n, kBodyThreads), kBodyThreads, true, s, a, n)) != cudaSuccess) return e;
    const uint32_t cb = blocks_for(g.n_cells, kCellThreads), gb = blocks_for(n, kBodyThreads);
    if (dim == 2) {
        if ((e = launch_chained(k_cells<2>, cb, kCellThreads, true, s, g, a)) != cudaSuccess) return e;
        return launch_chained(write_slots ? (write_s ? k_gather<2, true, true> : k_gather<2, false, true>)
                                          : (write_s ? k_gather<2, true, false> : k_gather<2, false, false>),
                              gb, kBodyThreads, true, s, g, a, n);
    }
    if ((e = launch_chained(k_cells<3>, cb, kCellThreads, true, s, g, a)) != cudaSuccess) return e;
    return launch_chained(write_slots ? (write_s ? k_gather<3, true, true> : k_gather<3, false, true>)
                                      : (write_s ? k_gather<3, true, false> : k_gather<3, false, false>),
                          gb, kBodyThreads, true, s, g, a, n);
}

cudaError_t launch_rebuild_batch(int dim, const Batch& b, const Arrays& a, uint32_t n, bool write_s, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(a.cell_count, 0, sizeof(uint32_t) * b.n_cells, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.nonempty, 0, sizeof(unsigned int) * b.n_replicas, s);
    if (e != cudaSuccess) return e;
    if (n > 0) {
        if (dim == 2)
            k_bin_batch<2><<<blocks_for(n, 256), 256, 0, s>>>(b, a, n);
        else
            k_bin_batch<3><<<blocks_for(n, 256), 256, 0, s>>>(b, a, n);
    }
    if ((e = launch_count_scan(a, b.n_cells, s, n > 0)) != cudaSuccess) return e;
    if (n == 0) return cudaSuccess;
    if ((e = launch_chained(k_scatter, blocks_for(n, 256), 256, true, s, a, n)) != cudaSuccess) return e;
    const uint32_t cb = blocks_for(b.n_cells, kCellThreads), gb = blocks_for(n, 256);
    if (dim == 2) {
        if ((e = launch_chained(k_cells_batch<2>, cb, kCellThreads, true, s, b, a)) != cudaSuccess) return e;
        return launch_chained(write_s ? k_gather_batch<2, true> : k_gather_batch<2, false>, gb, 256, true, s, b, a, n);
    }
    if ((e = launch_chained(k_cells_batch<3>, cb, kCellThreads, true, s, b, a)) != cudaSuccess) return e;
    return launch_chained(write_s ? k_gather_batch<3, true> : k_gather_batch<3, false>, gb, 256, true, s, b, a, n);
}

cudaError_t launch_sweep_batch(int dim, bool fp32, const Batch& b, const Arrays& a, uint32_t color, uint32_t round,
                               uint32_t max_active, bool overlap_previous, bool early_wait, cudaStream_t s,
                               uint32_t variant) {
    if (max_active == 0) return cudaSuccess;
    using BatchKernel = void (*)(Batch, Arrays, uint32_t, uint32_t, uint32_t);
    // the compiled launch variants, in the order of kBatchShapes
    static const BatchKernel kernels[2][2][6] = {
        {{k_sweep_batch<2, false, 4>, k_sweep_batch<2, false, 3>, k_sweep_batch<2, false, 5>,
          k_sweep_batch<2, false, 6>, k_sweep_batch<2, false, 7>, k_sweep_batch<2, false, 8>},
         {k_sweep_batch<2, true, 4>, k_sweep_batch<2, true, 3>, k_sweep_batch<2, true, 5>, k_sweep_batch<2, true, 6>,
          k_sweep_batch<2, true, 7>, k_sweep_batch<2, true, 8>}},
        {{k_sweep_batch<3, false, 4>, k_sweep_batch<3, false, 3>, k_sweep_batch<3, false, 5>,
          k_sweep_batch<3, false, 6>, k_sweep_batch<3, false, 7>, k_sweep_batch<3, false, 8>},
         {k_sweep_batch<3, true, 4>, k_sweep_batch<3, true, 3>, k_sweep_batch<3, true, 5>, k_sweep_batch<3, true, 6>,
          k_sweep_batch<3, true, 7>, k_sweep_batch<3, true, 8>}}};
    static_assert(n_shapes(kBatchShapes) == 6, "one compiled kernel per batch variant");
    const BatchKernel k = kernels[dim == 3][fp32][variant < 6 ? variant : 0];
    uint32_t grid = blocks_for(max_active, 128);
    const uint32_t wave = (uint32_t)resident_wave((const void*)k);
    if (grid > wave) grid = wave;
    PassLaunch pl(grid, overlap_previous || early_wait, s);
    const uint32_t ew = early_wait ? 1u : 0u;
    return cudaLaunchKernelEx(&pl.cfg, k, b, a, color, round, ew);
}

__global__ void k_sweep_guard(const DeviceStats* stats, uint32_t enqueued, uint32_t* abort_word) {
    if (*abort_word == 0u && (stats->rounds > enqueued || (stats->error_flags & ~kErrAborted) != 0u))
        *abort_word = 1u;
}

cudaError_t launch_sweep_guard(const DeviceStats* stats, uint32_t enqueued, uint32_t* abort_word, cudaStream_t s) {
    k_sweep_guard<<<1, 1, 0, s>>>(stats, enqueued, abort_word);
    return cudaGetLastError();
}

cudaError_t launch_batch_rounds(const Batch& b, Replica* rep, DeviceStats* stats, cudaStream_t s) {
    k_batch_rounds<<<blocks_for(b.n_replicas, 128), 128, 0, s>>>(b, rep, stats);
    return cudaGetLastError();
}

cudaError_t launch_batch_origins(int dim, const Batch& b, Replica* rep, cudaStream_t s) {
    if (dim == 2)
        k_batch_origins<2><<<blocks_for(b.n_replicas, 128), 128, 0, s>>>(b, rep);
    else
        k_batch_origins<3><<<blocks_for(b.n_replicas, 128), 128, 0, s>>>(b, rep);
    return cudaGetLastError();
}

cudaError_t launch_batch_round_first(cudaGraphConditionalHandle h, const DeviceStats* stats, uint32_t* round_dev,
                                     const BatchSweepTotals* totals, cudaStream_t s) {
    k_batch_round_first<<<1, 1, 0, s>>>(h, stats, round_dev, totals);
    return cudaGetLastError();
}

cudaError_t launch_batch_round_next(cudaGraphConditionalHandle h, const DeviceStats* stats, uint32_t* round_dev,
                                    cudaStream_t s) {
    k_batch_round_next<<<1, 1, 0, s>>>(h, stats, round_dev);
    return cudaGetLastError();
}

cudaError_t launch_batch_sweep_end(const Batch& b, Replica* rep, const DeviceStats* stats,
                                   unsigned long long* rep_counts, BatchSweepTotals* totals, bool increment_step,
                                   cudaStream_t s) {
    k_batch_sweep_end<<<blocks_for(b.n_replicas, 128), 128, 0, s>>>(b, rep, stats, rep_counts, totals,
                                                                      increment_step ? 1u : 0u);
    return cudaGetLastError();
}

cudaError_t launch_overlap_batch(int dim, const Batch& b, const Arrays& a, uint32_t n, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(b.overlaps, 0, sizeof(unsigned long long) * b.n_replicas, s);
    if (e != cudaSuccess || n == 0) return e;
    if (dim == 2)
        k_overlap_batch<2><<<blocks_for(n, 128), 128, 0, s>>>(b, a, n);
    else
        k_overlap_batch<3><<<blocks_for(n, 128), 128, 0, s>>>(b, a, n);
    return cudaGetLastError();
}

namespace {
using SphereKernel = void (*)(Geometry, Arrays, Pair, Launch, Injected);

// The compiled launch variants of the sphere passes, in the order of kSphereDirectShapes /
// kSphereCoopShapes ([dim == 3][fp32][variant]).
SphereKernel direct_kernel(int dim, bool fp32, uint32_t v) {
    static const SphereKernel k[2][2][3] = {
        {{k_sweep_sphere<2, false, false, 6>, k_sweep_sphere<2, false, false, 5>, k_sweep_sphere<2, false, false, 7>},
         {k_sweep_sphere<2, true, false, 6>, k_sweep_sphere<2, true, false, 5>, k_sweep_sphere<2, true, false, 7>}},
        {{k_sweep_sphere<3, false, false, 6>, k_sweep_sphere<3, false, false, 5>, k_sweep_sphere<3, false, false, 7>},
         {k_sweep_sphere<3, true, false, 6>, k_sweep_sphere<3, true, false, 5>, k_sweep_sphere<3, true, false, 7>}}};
    static_assert(n_shapes(kSphereDirectShapes) == 3, "one compiled kernel per direct sphere variant");
    return k[dim == 3][fp32][v < 3 ? v : 0];
}
SphereKernel coop_kernel(int dim, bool fp32, uint32_t v) {
    static const SphereKernel k[2][2][5] = {
        {{k_sweep_sphere_coop<2, false, false, 6, 2>, k_sweep_sphere_coop<2, false, false, 6, 1>,
          k_sweep_sphere_coop<2, false, false, 6, 3>, k_sweep_sphere_coop<2, false, false, 5, 2>,
          k_sweep_sphere_coop<2, false, false, 7, 2>},
         {k_sweep_sphere_coop<2, true, false, 6, 2>, k_sweep_sphere_coop<2, true, false, 6, 1>,
          k_sweep_sphere_coop<2, true, false, 6, 3>, k_sweep_sphere_coop<2, true, false, 5, 2>,
          k_sweep_sphere_coop<2, true, false, 7, 2>}},
        {{k_sweep_sphere_coop<3, false, false, 6, 2>, k_sweep_sphere_coop<3, false, false, 6, 1>,
          k_sweep_sphere_coop<3, false, false, 6, 3>, k_sweep_sphere_coop<3, false, false, 5, 2>,
          k_sweep_sphere_coop<3, false, false, 7, 2>},
         {k_sweep_sphere_coop<3, true, false, 6, 2>, k_sweep_sphere_coop<3, true, false, 6, 1>,
          k_sweep_sphere_coop<3, true, false, 6, 3>, k_sweep_sphere_coop<3, true, false, 5, 2>,
          k_sweep_sphere_coop<3, true, false, 7, 2>}}};
    static_assert(n_shapes(kSphereCoopShapes) == 5, "one compiled kernel per cooperative sphere variant");
    return k[dim == 3][fp32][v < 5 ? v : 0];
}

}  // namespace

int resident_wave(const void* kernel) {
    static std::mutex mu;
    static std::unordered_map<const void*, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    const void* key = (const void*)((const char*)kernel + dev);  // one entry per kernel and device
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 128, 0) != cudaSuccess) {
        cudaGetLastError();
        per_sm = 1;
    }
    const int wave = (sms > 0 ? sms : 1) * (per_sm > 0 ? per_sm : 1);
    cache[key] = wave;
    return wave;
}

cudaError_t launch_sweep_sphere(int dim, bool fp32, const Geometry& g, const Arrays& a, const Pair& p,
                                const Launch& l, bool coop, cudaStream_t s, uint32_t variant) {
    if (l.n_active == 0) return cudaSuccess;  // no non-empty space of this colour
    // grid-stride over the colour's list with at most one resident wave of blocks
    const SphereKernel k = coop ? coop_kernel(dim, fp32, variant) : direct_kernel(dim, fp32, variant);
    uint32_t grid = blocks_for(l.n_active, 128);
    const uint32_t wave = (uint32_t)resident_wave((const void*)k);
    if (grid > wave) grid = wave;
    PassLaunch pl(grid, l.overlap_previous != 0 || l.early_wait != 0, s);
    return cudaLaunchKernelEx(&pl.cfg, k, g, a, p, l, Injected{});
}

cudaError_t launch_trials_sphere(int dim, bool fp32, bool coop, const Geometry& g, const Arrays& a, const Pair& p,
                                 const Injected& j, cudaStream_t s) {
    if (j.n == 0) return cudaSuccess;
    const Launch l{};
    const uint32_t grid = blocks_for(j.n, 128);
    if (coop) {
        if (dim == 2) {
            if (fp32)
                k_sweep_sphere_coop<2, true, true><<<grid, 128, 0, s>>>(g, a, p, l, j);
            else
                k_sweep_sphere_coop<2, false, true><<<grid, 128, 0, s>>>(g, a, p, l, j);
        } else {
            if (fp32)
                k_sweep_sphere_coop<3, true, true><<<grid, 128, 0, s>>>(g, a, p, l, j);
            else
                k_sweep_sphere_coop<3, false, true><<<grid, 128, 0, s>>>(g, a, p, l, j);
        }
    } else {
        if (dim == 2) {
            if (fp32)
                k_sweep_sphere<2, true, true><<<grid, 128, 0, s>>>(g, a, p, l, j);
            else
                k_sweep_sphere<2, false, true><<<grid, 128, 0, s>>>(g, a, p, l, j);
        } else {
            if (fp32)
                k_sweep_sphere<3, true, true><<<grid, 128, 0, s>>>(g, a, p, l, j);
            else
                k_sweep_sphere<3, false, true><<<grid, 128, 0, s>>>(g, a, p, l, j);
        }
    }
    return cudaGetLastError();
}

cudaError_t launch_tune_stream_sphere(int dim, TuneJob* jobs, uint32_t n_jobs, cudaStream_t s) {
    if (n_jobs == 0) return cudaSuccess;
    if (dim == 2)
        k_tune_stream_sphere<2><<<n_jobs, 32, 0, s>>>(jobs, n_jobs);
    else
        k_tune_stream_sphere<3><<<n_jobs, 32, 0, s>>>(jobs, n_jobs);
    return cudaGetLastError();
}

cudaError_t launch_overlap_sphere(int dim, const Geometry& g, const Arrays& a, const Pair& p, uint32_t n,
                                  cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    if (dim == 2)
        k_overlap_sphere<2><<<blocks_for(n, 128), 128, 0, s>>>(g, a, p, n);
    else
        k_overlap_sphere<3><<<blocks_for(n, 128), 128, 0, s>>>(g, a, p, n);
    return cudaGetLastError();
}

cudaError_t launch_pair_histogram(int dim, bool sdf, const Geometry& g, const Arrays& a, uint32_t n, double sigma,
                                  double limit, double inv_width, uint32_t n_bins, unsigned long long* counts,
                                  cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(unsigned long long) * n_bins, s);
    if (e != cudaSuccess || n == 0) return e;
    const size_t smem = sizeof(unsigned int) * n_bins;
    const uint32_t grid = blocks_for(n, 256);
    if (dim == 2) {
        if (sdf)
            k_pair_histogram<2, true><<<grid, 256, smem, s>>>(g, a, n, sigma, limit, inv_width, n_bins, counts);
        else
            k_pair_histogram<2, false><<<grid, 256, smem, s>>>(g, a, n, sigma, limit, inv_width, n_bins, counts);
    } else {
        if (sdf)
            k_pair_histogram<3, true><<<grid, 256, smem, s>>>(g, a, n, sigma, limit, inv_width, n_bins, counts);
        else
            k_pair_histogram<3, false><<<grid, 256, smem, s>>>(g, a, n, sigma, limit, inv_width, n_bins, counts);
    }
    return cudaGetLastError();
}

cudaError_t launch_eval_sphere(int dim, bool fp32, const Geometry& g, const Arrays& a, const Pair& p,
                               const uint64_t* bodies, const double4* trial, uint32_t n, uint8_t* decisions,
                               uint8_t* rechecked, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    uint32_t grid = blocks_for(n, 128);
    if (dim == 2) {
        if (fp32)
            k_eval_sphere<2, true><<<grid, 128, 0, s>>>(g, a, p, bodies, trial, n, decisions, rechecked);
        else
            k_eval_sphere<2, false><<<grid, 128, 0, s>>>(g, a, p, bodies, trial, n, decisions, rechecked);
    } else {
        if (fp32)
            k_eval_sphere<3, true><<<grid, 128, 0, s>>>(g, a, p, bodies, trial, n, decisions, rechecked);
        else
            k_eval_sphere<3, false><<<grid, 128, 0, s>>>(g, a, p, bodies, trial, n, decisions, rechecked);
    }
    return cudaGetLastError();
}

}  // namespace hmc
