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

#include "hmc_internal.cuh"

namespace hmc {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// ---- checkerboard maps --------------------------------------------------------------------
// point_to_space_index for a periodic checkerboard (hypercuboid.rs:85-128). Returns false
// for None. m receives the multi-index.
template <int DIM>
__device__ __forceinline__ bool point_to_space(const Geometry& g, const double* x, uint32_t* m) {
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
        double p = dsub(x[a], g.origin[a]);
        double f = floor(ddiv(p, g.width[a]));
        if (!(f >= 0.0)) return false;
        if (f > 4.0e9) return false;
        uint32_t idx = (uint32_t)f;
        if (idx == g.shape[a]) idx = 0;
        if (idx > g.shape[a]) return false;
        m[a] = idx;
    }
    return true;
}
template <int DIM>
__device__ __forceinline__ uint32_t cell_index(const Geometry& g, const uint32_t* m) {
    uint32_t idx = 0;
#pragma unroll
    for (int a = 0; a < DIM; ++a) idx = idx * g.shape[a] + m[a];
    return idx;
}

// FP32 offset of a site from the lower corner of its cell (multi-index m), periodic frame.
template <int DIM>
__device__ __forceinline__ float4 cell_offsets(const Geometry& g, const double* s, const uint32_t* m) {
    float o[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
        double off = dsub(dsub(s[a], g.origin[a]), dmul((double)m[a], g.width[a]));
        if (off > 1.5 * g.width[a])
            off = dsub(off, g.L[a]);
        else if (off < -0.5 * g.width[a])
            off = dadd(off, g.L[a]);
        o[a] = __double2float_rn(off);
    }
    return make_float4(o[0], o[1], o[2], __int_as_float((int)m[DIM - 1]));
}

// Squared distance between a trial site t and a site s exactly as the reference computes
// it against s's primary and ghost images: the ghost rule of generate_ghosts_in_range
// (boundary/periodic/cuboid.rs:109-161) gives the image translations that exist, and
// distance_squared (hoomd-vector/src/cartesian.rs:339-342) folds (t - image)^2 from 0.0.
// Each axis keeps the image with the smaller |difference|; rounding is monotone, so this
// is the minimum of the reference's d^2 over all images.
template <int DIM>
__device__ __forceinline__ double ref_dist2(const Geometry& g, const double* t, const double* s) {
    bool inside = true;
#pragma unroll
    for (int a = 0; a < DIM; ++a) inside = inside && (s[a] >= -g.half[a]) && (s[a] < g.half[a]);
    double p = 0.0;
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
        double d = dsub(t[a], s[a]);
        if (inside) {
            double tr = 0.0;
            bool has = false;
            if (s[a] > g.ghost_hi[a]) {
                tr = -g.L[a];
                has = true;
            } else if (s[a] < g.ghost_lo[a]) {
                tr = g.L[a];
                has = true;
            }
            if (has) {
                double d2 = dsub(t[a], dadd(s[a], tr));
                if (fabs(d2) < fabs(d)) d = d2;
            }
        }
        p = dadd(p, dmul(d, d));
    }
    return p;
}

// ---- trial moves --------------------------------------------------------------------------
// Ball::sample (hoomd-vector/src/distribution.rs:41-69).
template <int DIM>
__device__ __forceinline__ void ball_sample(Sfc64& r, double radius, const double* zx, const double* zf,
                                            double* out) {
    if (DIM == 2) {
        for (;;) {
            double c0 = uniform01(r);
            double c1 = uniform01(r);
            double v0 = dmul(dsub(dmul(c0, 2.0), 1.0), radius);
            double v1 = dmul(dsub(dmul(c1, 2.0), 1.0), radius);
            double n2 = dfma(v1, v1, dfma(v0, v0, 0.0));
            if (n2 < dmul(radius, radius)) {
                out[0] = v0;
                out[1] = v1;
                out[2] = 0.0;
                return;
            }
        }
    } else {
        double p[3];
        p[0] = standard_normal(r, zx, zf);
        p[1] = standard_normal(r, zx, zf);
        p[2] = standard_normal(r, zx, zf);
        double norm = dsqrt(dot<3>(p, p));
        double u = uniform01(r);
        double scale = dmul(ddiv(radius, norm), portable_cbrt(u));
        out[0] = dmul(p[0], scale);
        out[1] = dmul(p[1], scale);
        out[2] = dmul(p[2], scale);
    }
}

// ---- neighbour stencil over cell-ordered rows ----------------------------------------------
// Calls f(q, dshift) for every body slot q in the 3^DIM spaces around the space m, where
// dshift[a] (FP32) is the displacement of the candidate's cell corner from m's corner
// along each axis for the slow axes; the fast-axis shift is derived per candidate from
// its stored cell index. Stops early when f returns true. Spaces are visited once even
// when an axis has only two spaces (both neighbours are then the same space).
template <int DIM, typename F>
__device__ __forceinline__ bool for_each_neighbor(const Geometry& g, const uint32_t* __restrict__ cell_start,
                                                  const uint32_t* m, F&& f) {
    constexpr int F_AX = DIM - 1;
    const uint32_t sf = g.shape[F_AX];
    const uint32_t mf = m[F_AX];
    int lo0 = (DIM == 3) ? (g.shape[0] == 2 ? 0 : -1) : 0;
    int hi0 = (DIM == 3) ? 1 : 0;
    int lo1 = (g.shape[DIM == 3 ? 1 : 0] == 2) ? 0 : -1;
    for (int i0 = lo0; i0 <= hi0; ++i0) {
        for (int i1 = lo1; i1 <= 1; ++i1) {
            uint32_t row_base;
            float slow_shift[2];
            if (DIM == 3) {
                uint32_t c0 = (m[0] + g.shape[0] + i0) % g.shape[0];
                uint32_t c1 = (m[1] + g.shape[1] + i1) % g.shape[1];
                row_base = (c0 * g.shape[1] + c1) * sf;
                slow_shift[0] = (float)i0 * g.w32[0];
                slow_shift[1] = (float)i1 * g.w32[1];
            } else {
                uint32_t c0 = (m[0] + g.shape[0] + i1) % g.shape[0];
                row_base = c0 * sf;
                slow_shift[0] = (float)i1 * g.w32[0];
                slow_shift[1] = 0.f;
            }
            uint32_t a0, a1, b0 = 0, b1 = 0;
            if (sf == 2) {
                a0 = cell_start[row_base];
                a1 = cell_start[row_base + 2];
            } else if (mf >= 1 && mf + 1 < sf) {
                a0 = cell_start[row_base + mf - 1];
                a1 = cell_start[row_base + mf + 2];
            } else if (mf == 0) {
                a0 = cell_start[row_base];
                a1 = cell_start[row_base + 2];
                b0 = cell_start[row_base + sf - 1];
                b1 = cell_start[row_base + sf];
            } else {
                a0 = cell_start[row_base + sf - 2];
                a1 = cell_start[row_base + sf];
                b0 = cell_start[row_base];
                b1 = cell_start[row_base + 1];
            }
            for (uint32_t q = a0; q < a1; ++q)
                if (f(q, slow_shift)) return true;
            for (uint32_t q = b0; q < b1; ++q)
                if (f(q, slow_shift)) return true;
        }
    }
    return false;
}

// Read-only load of a double4 as two 16-byte loads through the non-coherent cache.
__device__ __forceinline__ double4 ldg4(const double4* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    double2 a = __ldg(q), b = __ldg(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

// Per-thread statistics of the FP32 path.
struct PairStats {
    uint32_t checks = 0;
    uint32_t rechecks = 0;
    double max_err = 0.0;
};

// Hard-sphere overlap of trial site t (FP64, FP32 offsets t32 within space m) against the
// neighbourhood of m, skipping slot `self`. FP32=true: FP32 test under the bound, FP64
// recheck in between; FP32=false: the reference FP64 test on every candidate.
template <int DIM, bool FP32>
__device__ __forceinline__ bool sphere_overlaps(const Geometry& g, const Arrays& A, const Pair& P, const double* t,
                                                float4 t32, const uint32_t* m, uint32_t self, PairStats& st) {
    const uint32_t* __restrict__ cs = A.cell_start;
    const float4* __restrict__ off = A.sorted_off;
    const double4* __restrict__ ss = A.sorted_s;
    constexpr int F_AX = DIM - 1;
    const uint32_t sf = g.shape[F_AX];
    const int mf = (int)m[F_AX];
    const float wf = g.w32[F_AX];
    const bool slow_two = (DIM == 3) ? (g.shape[0] == 2 || g.shape[1] == 2) : (g.shape[0] == 2);
    return for_each_neighbor<DIM>(g, cs, m, [&](uint32_t q, const float* slow_shift) -> bool {
        if (q == self) return false;
        if (FP32) {
            float4 o = __ldg(off + q);
            int dm = __float_as_int(o.w) - mf;
            if (sf >= 4) {
                if (dm > 1)
                    dm -= (int)sf;
                else if (dm < -1)
                    dm += (int)sf;
            }
            float tv[3] = {t32.x, t32.y, t32.z};
            float ov[3] = {o.x, o.y, o.z};
            float d[3] = {0.f, 0.f, 0.f};
            if (DIM == 3) {
                d[0] = tv[0] - (ov[0] + slow_shift[0]);
                d[1] = tv[1] - (ov[1] + slow_shift[1]);
                d[2] = tv[2] - (ov[2] + (float)dm * wf);
            } else {
                d[0] = tv[0] - (ov[0] + slow_shift[0]);
                d[1] = tv[1] - (ov[1] + (float)dm * wf);
            }
            if (slow_two || sf == 2) {
#pragma unroll
                for (int a = 0; a < DIM; ++a) {
                    if (g.shape[a] == 2) {
                        float w = g.w32[a];
                        if (d[a] > w)
                            d[a] -= 2.f * w;
                        else if (d[a] < -w)
                            d[a] += 2.f * w;
                    }
                }
            }
            float dd = d[0] * d[0] + d[1] * d[1];
            if (DIM == 3) dd += d[2] * d[2];
            st.checks++;
            if (dd < P.sig2_lo32) return true;
            if (dd >= P.sig2_hi32) return false;
            // inside the bound: the reference FP64 test decides
            st.rechecks++;
            double4 s4 = ldg4(ss + q);
            double sv[3] = {s4.x, s4.y, s4.z};
            double r2 = ref_dist2<DIM>(g, t, sv);
            double e = fabs((double)dd - r2);
            st.max_err = e > st.max_err ? e : st.max_err;
            return r2 < P.sigma2;
        } else {
            double4 s4 = ldg4(ss + q);
            double sv[3] = {s4.x, s4.y, s4.z};
            st.checks++;
            return ref_dist2<DIM>(g, t, sv) < P.sigma2;
        }
    });
}

__device__ __forceinline__ void flush_stats(DeviceStats* stats, const PairStats& st, bool accepted) {
    const unsigned full = 0xffffffffu;
    unsigned acc = __ballot_sync(full, accepted);
    unsigned checks = __reduce_add_sync(full, st.checks);
    unsigned rech = __reduce_add_sync(full, st.rechecks);
    if ((threadIdx.x & 31) == 0) {
        if (acc) atomicAdd(&stats->accepted, (unsigned long long)__popc(acc));
        if (checks) atomicAdd(&stats->pair_checks, (unsigned long long)checks);
        if (rech) atomicAdd(&stats->rechecks, (unsigned long long)rech);
    }
    if (st.max_err > 0.0) atomicMax(&stats->max_err_bits, (unsigned long long)__double_as_longlong(st.max_err));
}

// ---- the colour pass ------------------------------------------------------------------------
// One thread per space of the colour: ParallelSweep::generate_trial_moves for that space
// (parallel_sweep.rs:231-278) followed by update_bodies (:283-314) for an accepted move.
// Spaces of one colour are two spaces apart, so the in-place update of an accepted body is
// invisible to every other trial of the colour, as in the reference.
template <int DIM, bool FP32>
__global__ void __launch_bounds__(128) k_sweep_sphere(Geometry g, Arrays A, Pair P, Launch L) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    bool accepted = false;
    PairStats st;
    if (tid < L.n_active) {
        uint32_t m[3];
        uint32_t rem = tid;
#pragma unroll
        for (int a = DIM - 1; a >= 0; --a) {
            uint32_t h = rem % g.half_shape[a];
            rem /= g.half_shape[a];
            m[a] = 2u * h + ((L.color >> (DIM - 1 - a)) & 1u);
        }
        const uint32_t cell = cell_index<DIM>(g, m);
        const uint32_t start = A.cell_start[cell];
        const uint32_t count = A.cell_start[cell + 1] - start;
        if (count > 0) {
            Sfc64 rng = make_rng(L.step, L.substep, L.seed, (uint64_t)cell);
            const uint32_t k = start + canon_range_u32(rng, count);
            double4 b4 = A.sorted_b[k];
            double x[3] = {b4.x, b4.y, b4.z};
            double dv[3];
            ball_sample<DIM>(rng, L.max_move, A.zig_x, A.zig_f, dv);
#pragma unroll
            for (int a = 0; a < DIM; ++a) x[a] = dadd(x[a], dv[a]);
            wrap<DIM>(g.L, x);  // W1 = wrap(propose(..))
            uint32_t mt[3];
            bool same = point_to_space<DIM>(g, x, mt) && cell_index<DIM>(g, mt) == cell;
            if (same) {
                double t[3] = {x[0], x[1], DIM == 3 ? x[2] : 0.0};
                wrap<DIM>(g.L, t);  // delta_energy_one wraps the site again: T = wrap(W1)
                float4 t32 = FP32 ? cell_offsets<DIM>(g, t, m) : make_float4(0.f, 0.f, 0.f, 0.f);
                bool overlap = sphere_overlaps<DIM, FP32>(g, A, P, t, t32, m, k, st);
                if (!overlap) {
                    accepted = true;
                    // update_body_properties: body = wrap(W1) = T, site = wrap(body)
                    double s[3] = {t[0], t[1], t[2]};
                    wrap<DIM>(g.L, s);
                    A.sorted_b[k] = make_double4(t[0], t[1], t[2], 0.0);
                    A.sorted_s[k] = make_double4(s[0], s[1], s[2], 0.0);
                    A.sorted_off[k] = cell_offsets<DIM>(g, s, m);
                    A.body_pos[A.sorted_body[k]] = make_double4(t[0], t[1], t[2], 0.0);
                }
            }
        }
    }
    flush_stats(A.stats, st, accepted);
}

// ---- cell list rebuild -------------------------------------------------------------------
template <int DIM>
__global__ void k_bin(Geometry g, Arrays A, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
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
    A.body_rank[i] = atomicAdd(&A.cell_count[cell], 1u);
}

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warp_sums[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kScanThreads / 32 ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kScanThreads / 32) warp_sums[lane] = w;
    }
    __syncthreads();
    uint32_t warp_prefix = warp > 0 ? warp_sums[warp - 1] : 0;
    *total = warp_sums[kScanThreads / 32 - 1];
    __syncthreads();
    return warp_prefix + x - v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(Arrays A, uint32_t n_cells) {
    uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t sum = 0, nonempty = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        uint32_t c = base + k;
        uint32_t v = c < n_cells ? A.cell_count[c] : 0;
        sum += v;
        nonempty += v > 0;
    }
    uint32_t total;
    block_exclusive_scan(sum, &total);
    uint32_t ne = __reduce_add_sync(0xffffffffu, nonempty);
    if ((threadIdx.x & 31) == 0 && ne) atomicAdd(&A.stats->nonempty, ne);
    if (threadIdx.x == 0) A.block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_scan_block_sums(Arrays A, uint32_t n_blocks) {
    // Single block: exclusive scan of up to 1024 * 8 block sums in place.
    __shared__ uint32_t warp_sums[32];
    constexpr int items = 8;
    uint32_t base = threadIdx.x * items;
    uint32_t v[items];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < items; ++k) {
        v[k] = base + k < n_blocks ? A.block_sums[base + k] : 0;
        sum += v[k];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_sums[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        warp_sums[lane] = w;
    }
    __syncthreads();
    uint32_t run = (warp > 0 ? warp_sums[warp - 1] : 0) + x - sum;
#pragma unroll
    for (int k = 0; k < items; ++k) {
        if (base + k < n_blocks) A.block_sums[base + k] = run;
        run += v[k];
    }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_apply(Arrays A, uint32_t n_cells) {
    uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        uint32_t c = base + k;
        v[k] = c < n_cells ? A.cell_count[c] : 0;
        sum += v[k];
    }
    uint32_t total;
    uint32_t run = block_exclusive_scan(sum, &total) + A.block_sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        uint32_t c = base + k;
        if (c < n_cells) A.cell_start[c] = run;
        run += v[k];
        if (c + 1 == n_cells) A.cell_start[n_cells] = run;
    }
}

__global__ void k_scatter(Arrays A, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    A.sorted_body[A.cell_start[A.body_cell[i]] + A.body_rank[i]] = i;
}

// One thread per space: order its bodies by index (the order in which update_checkerboard
// pushes them, parallel_sweep.rs:194-200, which IndexedRandom::choose indexes) and gather
// B, S = wrap(B), the FP32 offsets and orientations into cell order.
template <int DIM>
__global__ void k_finalize(Geometry g, Arrays A) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.n_cells) return;
    uint32_t s = A.cell_start[c], e = A.cell_start[c + 1];
    for (uint32_t k = s + 1; k < e; ++k) {
        uint32_t v = A.sorted_body[k];
        uint32_t j = k;
        while (j > s && A.sorted_body[j - 1] > v) {
            A.sorted_body[j] = A.sorted_body[j - 1];
            --j;
        }
        A.sorted_body[j] = v;
    }
    uint32_t m[3] = {0, 0, 0};
    uint32_t rem = c;
#pragma unroll
    for (int a = DIM - 1; a >= 0; --a) {
        m[a] = rem % g.shape[a];
        rem /= g.shape[a];
    }
    for (uint32_t k = s; k < e; ++k) {
        uint32_t i = A.sorted_body[k];
        A.slot_of_body[i] = k;
        double4 b = A.body_pos[i];
        A.sorted_b[k] = b;
        double sv[3] = {b.x, b.y, b.z};
        wrap<DIM>(g.L, sv);
        A.sorted_s[k] = make_double4(sv[0], sv[1], sv[2], 0.0);
        A.sorted_off[k] = cell_offsets<DIM>(g, sv, m);
        if (A.sorted_q) A.sorted_q[k] = A.body_ori[i];
    }
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

// ---- injected moves (delta_energy_one + Metropolis for hard spheres) -----------------------
template <int DIM, bool FP32>
__global__ void k_eval_sphere(Geometry g, Arrays A, Pair P, const uint64_t* bodies, const double4* trial, uint32_t n,
                              uint8_t* decisions, uint8_t* rechecked) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    PairStats st;
    if (i < n) {
        double4 w = trial[i];
        double t[3] = {w.x, w.y, DIM == 3 ? w.z : 0.0};
        wrap<DIM>(g.L, t);
        uint32_t m[3];
        bool ok = point_to_space<DIM>(g, t, m);
        uint8_t dec = 0;
        if (ok) {
            uint32_t self = A.slot_of_body[bodies[i]];
            float4 t32 = FP32 ? cell_offsets<DIM>(g, t, m) : make_float4(0.f, 0.f, 0.f, 0.f);
            dec = sphere_overlaps<DIM, FP32>(g, A, P, t, t32, m, self, st) ? 0 : 1;
        } else {
            atomicOr(&A.stats->error_flags, kErrOutsideCheckerboard);
        }
        decisions[i] = dec;
        rechecked[i] = st.rechecks > 0;
    }
    flush_stats(A.stats, st, false);
}

template <typename T>
inline uint32_t blocks_for(T n, uint32_t threads) {
    return (uint32_t)((n + threads - 1) / threads);
}

}  // namespace

cudaError_t launch_rebuild(int dim, const Geometry& g, const Arrays& a, uint32_t n, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(a.cell_count, 0, sizeof(uint32_t) * g.n_cells, s);
    if (e != cudaSuccess) return e;
    if (n > 0) {
        if (dim == 2)
            k_bin<2><<<blocks_for(n, 256), 256, 0, s>>>(g, a, n);
        else
            k_bin<3><<<blocks_for(n, 256), 256, 0, s>>>(g, a, n);
    }
    uint32_t nb = blocks_for(g.n_cells, kScanTile);
    k_scan_reduce<<<nb, kScanThreads, 0, s>>>(a, g.n_cells);
    k_scan_block_sums<<<1, 1024, 0, s>>>(a, nb);
    k_scan_apply<<<nb, kScanThreads, 0, s>>>(a, g.n_cells);
    if (n > 0) k_scatter<<<blocks_for(n, 256), 256, 0, s>>>(a, n);
    if (dim == 2)
        k_finalize<2><<<blocks_for(g.n_cells, 128), 128, 0, s>>>(g, a);
    else
        k_finalize<3><<<blocks_for(g.n_cells, 128), 128, 0, s>>>(g, a);
    return cudaGetLastError();
}

cudaError_t launch_sweep_sphere(int dim, bool fp32, const Geometry& g, const Arrays& a, const Pair& p,
                                const Launch& l, cudaStream_t s) {
    if (l.n_active == 0) return cudaSuccess;
    uint32_t grid = blocks_for(l.n_active, 128);
    if (dim == 2) {
        if (fp32)
            k_sweep_sphere<2, true><<<grid, 128, 0, s>>>(g, a, p, l);
        else
            k_sweep_sphere<2, false><<<grid, 128, 0, s>>>(g, a, p, l);
    } else {
        if (fp32)
            k_sweep_sphere<3, true><<<grid, 128, 0, s>>>(g, a, p, l);
        else
            k_sweep_sphere<3, false><<<grid, 128, 0, s>>>(g, a, p, l);
    }
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
