// Lennard-Jones Metropolis sweep: PairwiseCutoff<Isotropic<Shifted<LennardJones>>>.
//
// delta_energy_one (hoomd-interaction/src/pairwise_cutoff.rs:919-941) sums the pair energy of
// the trial site and of the current site over every other site within r_cut; the Metropolis
// test (hoomd-mc/src/parallel_sweep.rs:267-268) accepts when dH <= 0, else draws u and accepts
// when u < exp(-dH / kT). At rho = 0.8 with r_cut = 2.5 a space holds ~13 bodies, so a colour
// pass has few trials (~5k for 2^19 bodies) with ~340 candidates each: one warp per trial,
// which takes the candidates of all stencil rows 32 at a time (FlatStencil: ~11 steps instead
// of two per row), and warp reductions of the sums.
//
// FP32 + recheck: the warp sums FP32 pair energies together with a rigorous bound B on
// |dU32 - dU64| (r^2 error from the FP32 offsets, propagated through dE/dr^2; rounding of the
// energy formula; summation chains; the FP64 sum's own error). A decision that B cannot
// change is taken from the FP32 sums; otherwise the warp recomputes dU in FP64 with exactly
// the lane assignment and reduction order of the plain FP64 pass, so decisions equal it.
#include <cuda_runtime.h>

#include "hmc_device.cuh"

namespace hmc {
namespace {

// Resident blocks per SM the sweep pass is compiled for: 9 caps it at 56 registers, so that a
// colour pass of the 2^19-body LJ system (4,913 trials of one warp) runs in one wave; measured
// 1.32e8 (FP32) and 1.83e8 (FP64) trial moves/s there, against 1.01e8 and 1.24e8 uncapped.
#ifndef HMC_LJ_MIN_BLOCKS
#define HMC_LJ_MIN_BLOCKS 9
#endif
// The same for the batch passes: 7 (72 registers) still runs a colour pass of 64 replicas of
// 8192 bodies (4,096 trials) in one wave and spills less: 1.34e8 (FP32) and 1.15e8 (FP64)
// trial moves/s there, against 1.18e8 and 1.07e8 at 56 registers and 1.01e8 and 7.1e7 at 80.
#ifndef HMC_LJ_BATCH_MIN_BLOCKS
#define HMC_LJ_BATCH_MIN_BLOCKS 7
#endif

constexpr float kU32 = 5.9604645e-8f;  // 2^-24

// FP32 pair energy and a bound on its error against the exact energy of the FP64 sites, for
// a pair with r2 below the band's upper end (the caller skips pairs outside the cut-off).
// The r^2 error is bounded without a square root: sum |d_a| <= sqrt(3) r and
// r <= (r^2 + 1) / 2, so |r2_32 - r2| <= 3.5 E ((r^2 + 1)/2 + E) + 3.1 u32 r^2.
__device__ __forceinline__ void lj_pair32(const Pair& P, float r2, float& e, float& err) {
    if (r2 >= P.lj_rcut2_lo32) {  // the FP64 pass may or may not count this pair
        e = 0.f;
        err = P.lj_band_energy;
        return;
    }
    const float E = P.lj_disp_err;
    const float dr2 = 3.5f * E * (0.5f * (r2 + 1.f) + E) + 3.1f * kU32 * r2;
    const float inv = __frcp_rn(r2);
    const float sr2 = P.lj_sigma2_32 * inv;
    const float sr6 = sr2 * sr2 * sr2;
    const float b = P.lj_four_eps32 * sr6;  // 4 eps (sigma/r)^6
    const float a = b * sr6;                // 4 eps (sigma/r)^12
    e = (a - b) - P.lj_e_shift32;
    // |dE/dr^2| <= (6a + 3b) / r^2; 1.1 covers its variation over [r2 - dr2, r2 + dr2] and the
    // FP32 evaluation of this bound; 24 u32 covers the roundings of the energy formula.
    err = 1.1f * ((6.f * a + 3.f * b) * (dr2 * inv) + 24.f * kU32 * (a + b + fabsf(P.lj_e_shift32)));
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ uint32_t warp_maxu(uint32_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// FP64 energy of site ta (and, when TWO, of site tb in the same space) against the stencil
// fs, skipping slot self: the warp takes the stencil's candidates 32 at a time, each lane sums
// its own in that order, then a butterfly reduction (every lane ends with the same values).
// S of a candidate comes from sorted_s when have_s, else from wrap(sorted_b). The two sums of
// one call equal two calls of one sum each over the same stencil.
// mag receives sum |e| over both sums (for order_ambiguous).
// U: candidates a lane loads per step (U = 2 keeps two loads in flight); a lane still adds its
// terms in increasing candidate order, so the sums are the same bits for every U.
template <int DIM, bool TWO, bool GENERIC = true, int U = 1>
__device__ __forceinline__ void lj_energy64(const Geometry& g, const Arrays& A, const Pair& P, const double* ta,
                                            const double* tb, const FlatStencil& fs, uint32_t self, bool have_s,
                                            uint32_t lane, double& ea, double& eb, double& mag) {
    double a = 0.0, b = 0.0, am = 0.0;
#pragma unroll 1
    for (uint32_t j0 = 0; j0 < fs.total; j0 += 32u * U) {
        double4 v[U];
        bool ok[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t j = j0 + 32u * u + lane;
            uint32_t part;
            const uint32_t q = flat_slot(fs, j, part);
            ok[u] = j < fs.total && q != self;
            v[u] = ok[u] ? ldg4((have_s ? A.sorted_s : A.sorted_b) + q) : make_double4(0.0, 0.0, 0.0, 0.0);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (!ok[u]) continue;
            double sv[3] = {v[u].x, v[u].y, v[u].z};
            if (!have_s) wrap_inv<DIM>(g.L, g.invL, sv);
            const double ra = ref_dist2<DIM>(g, ta, sv);
            const double x = soft_pair64<GENERIC>(P, ra);
            a = dadd(a, x);
            am += GENERIC ? soft_pair_mag(P, ra, x) : fabs(x);
            if (TWO) {
                const double rb = ref_dist2<DIM>(g, tb, sv);
                const double y = soft_pair64<GENERIC>(P, rb);
                b = dadd(b, y);
                am += GENERIC ? soft_pair_mag(P, rb, y) : fabs(y);
            }
        }
    }
    ea = warp_sum(a);
    eb = TWO ? warp_sum(b) : 0.0;
    mag = warp_sum(am);
}

struct Sums32 {
    float e_new, e_old, err, mag;
    uint32_t terms, pairs;
};

// FP32 energies of the trial site (offsets t32) and the current site (offsets c32) against
// the stencil fs of their common space, with error bounds. Each lane takes U candidates per
// step (loads issued together); the order of a lane's terms does not enter the bound.
template <int DIM, int U = 1>
__device__ __forceinline__ Sums32 lj_energy32(const Geometry& g, const Arrays& A, const Pair& P, float4 t32,
                                               float4 c32, int mf, const FlatStencil& fs, uint32_t self,
                                               uint32_t lane) {
    Sums32 s{0.f, 0.f, 0.f, 0.f, 0u, 0u};
    const uint32_t sf = g.shape[DIM - 1];
#pragma unroll 1
    for (uint32_t j0 = 0; j0 < fs.total; j0 += 32u * U) {
        float4 o[U];
        float s0[U], s1[U];
        bool ok[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t j = j0 + 32u * u + lane;
            uint32_t part;
            const uint32_t q = flat_slot(fs, j, part);
            s0[u] = __shfl_sync(0xffffffffu, fs.s0, part);
            s1[u] = __shfl_sync(0xffffffffu, fs.s1, part);
            ok[u] = j < fs.total && q != self;
            o[u] = ok[u] ? __ldg(A.sorted_off + q) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (!ok[u]) continue;
            int dm = __float_as_int(o[u].w) - mf;
            if (sf >= 4) {
                if (dm > 1)
                    dm -= (int)sf;
                else if (dm < -1)
                    dm += (int)sf;
            }
            const float r2n = fp32_dist2<DIM>(g, t32, o[u], s0[u], s1[u], dm);
            const float r2o = fp32_dist2<DIM>(g, c32, o[u], s0[u], s1[u], dm);
            s.pairs += 2;
            if (r2n < P.lj_rcut2_hi32) {
                float e, err;
                lj_pair32(P, r2n, e, err);
                s.e_new += e;
                s.err += err;
                s.mag += fabsf(e);
                s.terms += 1;
            }
            if (r2o < P.lj_rcut2_hi32) {
                float e, err;
                lj_pair32(P, r2o, e, err);
                s.e_old += e;
                s.err += err;
                s.mag += fabsf(e);
                s.terms += 1;
            }
        }
    }
    s.e_new = warp_sumf(s.e_new);
    s.e_old = warp_sumf(s.e_old);
    s.err = warp_sumf(s.err);
    s.mag = warp_sumf(s.mag);
    s.terms = warp_maxu(s.terms);
    return s;
}

// Metropolis decision from the FP32 sums: 1 accept, 0 reject, -1 needs the FP64 sums. u is the
// uniform the reference draws only when dU > 0 (parallel_sweep.rs:267-268): the next value of
// the trial's stream, which nothing else draws from, so the kernel draws it up front.
__device__ __forceinline__ int decide32(const Sums32& s, double kt, double u) {
    const float d32 = s.e_new - s.e_old;
    // summation chains (per lane + 5 reduction levels + the final difference), FP64's own error
    const float b = s.err + (float)(s.terms + 7) * kU32 * s.mag * 1.01f + kU32 * fabsf(d32) + 1e-9f * (s.mag + 1.f);
    if (!isfinite(d32) || !isfinite(b)) return -1;
    const double lo = (double)d32 - (double)b, hi = (double)d32 + (double)b;
    if (hi <= 0.0) return 1;  // dU64 <= 0 for certain: accepted without a uniform
    if (lo <= 0.0) return -1;
    const double t_hi = exp(-lo / kt) * (1.0 + 1e-12);  // dU64 > 0 for certain
    const double t_lo = exp(-hi / kt) * (1.0 - 1e-12);
    if (u < t_lo) return 1;
    if (u >= t_hi) return 0;
    return -1;
}

// The trial moves of one round for all colour lists (generate_trial_moves, parallel_sweep.rs:
// 231-278, up to the Metropolis test): thread i takes entry i of the colour lists, draws the
// body (IndexedRandom::choose), the displacement (Ball::sample) and the uniform from
// Counter(step, substep + round, seed).index(space), wraps (W1) and checks that W1 stays in the
// space; the passes then give each trial a warp and read the move from here instead of having
// every lane of the warp compute it. A trial reads only the rebuild's arrays and the bodies of its
// own colour, which the previous colours of the round do not move.
template <int DIM, bool FP32>
__global__ void __launch_bounds__(128) k_propose_lj(Geometry g, Arrays A, Launch L) {
    const DeviceStats* st = A.stats;
    if (st->error_flags != 0u || L.round >= st->rounds) return;
    const uint32_t colors = 1u << DIM;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < colors * g.color_stride;
         i += gridDim.x * blockDim.x) {
        const uint32_t c = i / g.color_stride, w = i - c * g.color_stride;
        if (w >= st->color_count[c]) continue;
        uint32_t m[3] = {0, 0, 0};
        unpack_m<DIM>(__ldg(A.color_cells + i), m);
        const uint32_t cell = cell_index<DIM>(g, m);
        const uint32_t start = __ldg(A.cell_start + cell);
        const uint32_t count = __ldg(A.cell_start + cell + 1) - start;
        Sfc64 rng = make_rng(L.step, L.substep, L.seed, (uint64_t)cell);
        const uint32_t k = start + canon_range_u32(rng, count);
        const double4 b4 = A.sorted_b[k];
        double x[3] = {b4.x, b4.y, b4.z};
        double dv[3];
        ball_sample<DIM>(rng, L.max_move, A.zig_x, A.zig_f, dv);
        const double u = uniform01(rng);
#pragma unroll
        for (int a = 0; a < DIM; ++a) x[a] = dadd(x[a], dv[a]);
        wrap_inv<DIM>(g.L, g.invL, x);  // W1 = wrap(propose(..))
        uint32_t mt[3];
        if (!(point_to_space<DIM>(g, x, mt) && cell_index<DIM>(g, mt) == cell)) {
            A.trial_k[i] = kNoTrial;  // leaves its space: rejected before delta_energy_one
            continue;
        }
        double t[3] = {x[0], x[1], DIM == 3 ? x[2] : 0.0};
        wrap_inv<DIM>(g.L, g.invL, t);  // the trial site T = wrap(W1)
        A.trial_t[i] = make_double4(t[0], t[1], t[2], u);
        if (FP32) A.trial_o[i] = cell_offsets<DIM>(g, t, m);
        A.trial_k[i] = k;
    }
}

// Injected trial w of the probe mode (Injected) in a warp-per-trial pass: the body's slot and
// space, W1 and u from the list. The colour pass evaluates only trials that stay in their body's
// space; the others are rejected as in the sweep (kTrialOutsideSpace).
template <int DIM>
__device__ __forceinline__ void lj_inject(const Arrays& A, const Injected& J, uint32_t w, uint32_t* m, uint32_t& k,
                                          double* x, double& u) {
    const uint64_t body = J.bodies[w];
    k = A.slot_of_body[body];
    unpack_m<DIM>(A.body_m[body], m);
    const double4 w4 = J.trial[w];
    x[0] = w4.x;
    x[1] = w4.y;
    x[2] = DIM == 3 ? w4.z : 0.0;
    u = J.u[w];
}

// The FP64 pass: one warp per trial. INJ: the probe mode (decisions instead of commits).
template <int DIM, bool INJ = false, int MINB = HMC_LJ_MIN_BLOCKS, bool GENERIC = true, int U = 1>
__global__ void __launch_bounds__(128, MINB) k_sweep_lj(Geometry g, Arrays A, Pair P, Launch L, Injected J) {
    if (L.early_wait) grid_dependency_wait();  // first pass: the rebuild's arrays are read at once
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
    uint32_t n_accepted = 0;
    PairStats pst;
    const uint32_t n_active = INJ ? J.n : active_count(A, L.color, L.round);
    for (uint32_t w = warp; w < n_active; w += n_warps) {
        uint32_t m[3] = {0, 0, 0};
        uint32_t k = 0;
        double x[3] = {0.0, 0.0, 0.0};
        double u = 0.0;
        double t[3] = {0.0, 0.0, 0.0};
        if constexpr (INJ) {
            lj_inject<DIM>(A, J, w, m, k, x, u);
        } else {
            // the round's trial from k_propose_lj
            const size_t e = (size_t)L.color * g.color_stride + w;
            k = __ldg(A.trial_k + e);
            if (k == kNoTrial) continue;  // warp-uniform: the move left its space
            unpack_m<DIM>(__ldg(A.color_cells + e), m);
            const double4 t4 = ldg4(A.trial_t + e);
            t[0] = t4.x;
            t[1] = t4.y;
            t[2] = t4.z;
            u = t4.w;
        }
        const uint32_t cell = cell_index<DIM>(g, m);
        const FlatStencil fs = flat_stencil<DIM>(g, A.cell_start, m, lane);
        if constexpr (INJ) {
            uint32_t mt[3];
            if (!(point_to_space<DIM>(g, x, mt) && cell_index<DIM>(g, mt) == cell)) {
                if (lane == 0) {
                    J.decisions[w] = 0;
                    J.flags[w] = kTrialOutsideSpace;
                }
                continue;
            }
            t[0] = x[0];
            t[1] = x[1];
            t[2] = DIM == 3 ? x[2] : 0.0;
            wrap_inv<DIM>(g.L, g.invL, t);
        }
        grid_dependency_wait();  // the previous colour's moves are visible from here on
        allow_dependent_launch();
        const double4 s4 = ldg4(A.sorted_s + k);
        const double si[3] = {s4.x, s4.y, s4.z};
        double e_new, e_old, mag;
        lj_energy64<DIM, true, GENERIC, U>(g, A, P, t, si, fs, k, true, lane, e_new, e_old, mag);
        const double du = dsub(e_new, e_old);
        const double e0 = exp(ddiv(-du, L.kt));
        const bool amb = order_ambiguous(du, mag, fs.total, u, L.kt, e0);
        if constexpr (INJ) {
            if (lane == 0) {
                J.decisions[w] = du <= 0.0 || u < e0;
                J.flags[w] = amb ? kTrialAmbiguous : 0;
            }
            continue;
        }
        if (amb && lane == 0) pst.ambiguous++;
        if ((du <= 0.0 || u < e0) && lane == 0) {
            n_accepted++;
            double sv[3] = {t[0], t[1], t[2]};
            wrap_inv<DIM>(g.L, g.invL, sv);
            A.sorted_b[k] = make_double4(t[0], t[1], t[2], 0.0);
            A.sorted_s[k] = make_double4(sv[0], sv[1], sv[2], 0.0);
            A.sorted_off[k] = cell_offsets<DIM>(g, sv, m);
            A.body_pos[A.sorted_body[k]] = make_double4(t[0], t[1], t[2], 0.0);
        }
        __syncwarp();
    }
    grid_dependency_wait();
    allow_dependent_launch();
    flush_stats(A.stats, pst, n_accepted);
}

// A trial's stencil and sites published in shared memory for the block-cooperative recheck.
struct SharedTrial {
    uint32_t lo[32], pre[32];  // the owner warp's FlatStencil parts
    double t[3], si[3];        // trial site and current site
    uint32_t total, self;
};

// Slot of candidate j of a published stencil (the FlatStencil search over shared memory).
__device__ __forceinline__ uint32_t shared_slot(const SharedTrial& st, uint32_t j) {
    uint32_t s = 0;
#pragma unroll
    for (uint32_t step = 16; step > 0; step >>= 1)
        if (st.pre[s + step] <= j) s += step;
    return st.lo[s] + (j - st.pre[s]);
}

constexpr uint32_t kRecheckChunks = 8;  // 32-candidate chunks per shared-memory round

// The FP32 + recheck pass. One warp per trial as in the FP64 pass, the block's four warps
// taking four trials at a time. A trial whose FP32 sums cannot decide is rechecked by the whole
// block: each warp evaluates every fourth 32-candidate chunk of the FP64 walk into shared
// memory, and the trial's own warp adds them per lane in chunk order, which gives the FP64
// pass's sums bit for bit (lj_energy64: the same candidates per lane in the same order, the
// same butterfly; an empty slot adds +0, which leaves a sum that starts at +0 unchanged). A
// lone warp walking the stencil in FP64 would otherwise set the duration of a pass whose
// trials all run in one wave.
template <int DIM, bool INJ = false, int MINB = HMC_LJ_MIN_BLOCKS, int U = 1>
__global__ void __launch_bounds__(128, MINB) k_sweep_lj32(Geometry g, Arrays A, Pair P, Launch L, Injected J) {
    if (L.early_wait) grid_dependency_wait();  // first pass: the rebuild's arrays are read at once
    __shared__ double s_e[kRecheckChunks][2][32];
    __shared__ SharedTrial s_trial;
    __shared__ uint32_t s_active;
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    uint32_t n_accepted = 0;
    PairStats pst;
    if (threadIdx.x == 0) s_active = INJ ? J.n : active_count(A, L.color, L.round);
    __syncthreads();
    const uint32_t n_active = s_active;  // block-uniform: the loop below holds barriers
    for (uint32_t base = blockIdx.x * 4u; base < n_active; base += gridDim.x * 4u) {
        const uint32_t w = base + wib;
        uint32_t m[3] = {0, 0, 0};
        uint32_t k = 0;
        double t[3] = {0.0, 0.0, 0.0};
        double u = 0.0;
        bool trial = false;
        FlatStencil fs{0u, 0u, 0u, 0.f, 0.f};
        bool outside = false;
        float4 t32p = make_float4(0.f, 0.f, 0.f, 0.f);
        if (INJ && w < n_active) {  // warp-uniform
            double x[3];
            lj_inject<DIM>(A, J, w, m, k, x, u);
            const uint32_t cell = cell_index<DIM>(g, m);
            fs = flat_stencil<DIM>(g, A.cell_start, m, lane);
            uint32_t mt[3];
            trial = point_to_space<DIM>(g, x, mt) && cell_index<DIM>(g, mt) == cell;
            outside = !trial;
            t[0] = x[0];
            t[1] = x[1];
            t[2] = x[2];
            wrap_inv<DIM>(g.L, g.invL, t);
        } else if (w < n_active) {  // warp-uniform: the round's trial from k_propose_lj
            const size_t e = (size_t)L.color * g.color_stride + w;
            k = __ldg(A.trial_k + e);
            trial = k != kNoTrial;
            if (trial) {
                unpack_m<DIM>(__ldg(A.color_cells + e), m);
                fs = flat_stencil<DIM>(g, A.cell_start, m, lane);
                const double4 t4 = ldg4(A.trial_t + e);
                t[0] = t4.x;
                t[1] = t4.y;
                t[2] = t4.z;
                u = t4.w;
                t32p = __ldg(A.trial_o + e);
            }
        }
        grid_dependency_wait();  // the previous colour's moves are visible from here on
        allow_dependent_launch();
        int decision = 0;
        float d32 = 0.f;
        if (trial) {
            const float4 t32 = INJ ? cell_offsets<DIM>(g, t, m) : t32p;
            const float4 c32 = __ldg(A.sorted_off + k);
            const Sums32 s = lj_energy32<DIM, U>(g, A, P, t32, c32, (int)m[DIM - 1], fs, k, lane);
            pst.checks += s.pairs;
            decision = decide32(s, L.kt, u);
            d32 = s.e_new - s.e_old;
        }
        const bool unsure = decision < 0;
        bool amb = false;
        if (__syncthreads_or(unsure)) {
            for (uint32_t o = 0; o < 4u; ++o) {
                const bool mine = unsure && wib == o;
                if (mine) {
                    s_trial.lo[lane] = fs.lo;
                    s_trial.pre[lane] = fs.pre;
                    if (lane == 0) {
                        const double4 c4 = ldg4(A.sorted_b + k);
                        double si[3] = {c4.x, c4.y, c4.z};
                        wrap_inv<DIM>(g.L, g.invL, si);
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            s_trial.t[a] = t[a];
                            s_trial.si[a] = si[a];
                        }
                        s_trial.total = fs.total;
                        s_trial.self = k;
                    }
                }
                if (!__syncthreads_or(mine)) continue;  // also publishes s_trial
                const uint32_t total = s_trial.total, self = s_trial.self;
                const uint32_t n_chunks = (total + 31u) / 32u;
                double ea = 0.0, eb = 0.0, em = 0.0;
                for (uint32_t c0 = 0; c0 < n_chunks; c0 += kRecheckChunks) {
                    const uint32_t c1 = min(c0 + kRecheckChunks, n_chunks);
                    for (uint32_t c = c0 + wib; c < c1; c += 4u) {
                        const uint32_t j = c * 32u + lane;
                        double en = 0.0, eo = 0.0;
                        if (j < total) {
                            const uint32_t q = shared_slot(s_trial, j);
                            if (q != self) {
                                const double4 b4 = ldg4(A.sorted_b + q);
                                double sv[3] = {b4.x, b4.y, b4.z};
                                wrap_inv<DIM>(g.L, g.invL, sv);
                                en = lj_only64(P, ref_dist2<DIM>(g, s_trial.t, sv));
                                eo = lj_only64(P, ref_dist2<DIM>(g, s_trial.si, sv));
                            }
                        }
                        s_e[c - c0][0][lane] = en;
                        s_e[c - c0][1][lane] = eo;
                    }
                    __syncthreads();
                    if (wib == o) {
                        for (uint32_t c = c0; c < c1; ++c) {
                            ea = dadd(ea, s_e[c - c0][0][lane]);
                            eb = dadd(eb, s_e[c - c0][1][lane]);
                            em += fabs(s_e[c - c0][0][lane]) + fabs(s_e[c - c0][1][lane]);
                        }
                    }
                    __syncthreads();
                }
                if (wib == o) {
                    const double du = dsub(warp_sum(ea), warp_sum(eb));
                    const double mag = warp_sum(em);
                    const double e0 = exp(ddiv(-du, L.kt));
                    amb = order_ambiguous(du, mag, total, u, L.kt, e0);
                    if (lane == 0) {
                        pst.rechecks++;
                        pst.ambiguous += amb ? 1u : 0u;
                        const double err = fabs((double)d32 - du);
                        pst.max_err = err > pst.max_err ? err : pst.max_err;
                    }
                    decision = (du <= 0.0 || u < e0) ? 1 : 0;
                }
            }
        }
        if constexpr (INJ) {
            if (w < n_active && lane == 0) {
                J.decisions[w] = decision == 1;
                J.flags[w] = (outside ? kTrialOutsideSpace : 0) | (unsure ? kTrialRechecked : 0) |
                             (amb ? kTrialAmbiguous : 0);
            }
        } else if (decision == 1 && lane == 0) {
            n_accepted++;
            double sv[3] = {t[0], t[1], t[2]};
            wrap_inv<DIM>(g.L, g.invL, sv);
            A.sorted_b[k] = make_double4(t[0], t[1], t[2], 0.0);
            A.sorted_off[k] = cell_offsets<DIM>(g, sv, m);
            A.body_pos[A.sorted_body[k]] = make_double4(t[0], t[1], t[2], 0.0);
        }
        __syncwarp();
    }
    grid_dependency_wait();
    allow_dependent_launch();
    flush_stats(A.stats, pst, n_accepted);
}

// One colour pass over every replica of a batch that still runs round `round` of this sweep,
// FP64: one warp per trial as in k_sweep_lj, with the box, checkerboard, pair parameters,
// Counter, move size and kT of the trial's replica from the replica table.
template <int DIM, int MINB = HMC_LJ_BATCH_MIN_BLOCKS, int U = 1>
__global__ void __launch_bounds__(128, MINB)
    k_sweep_batch_lj(Batch B, Arrays A, uint32_t color, uint32_t round, uint32_t early_wait) {
    if (early_wait) grid_dependency_wait();  // first pass: the rebuild's arrays are read at once
    if (round == kRoundFromDevice) round = *B.round_dev;  // a captured sweep's rounds loop
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
    uint32_t n_accepted = 0;
    PairStats pst;
    const uint32_t n_active = active_count(A, color, round);
    for (uint32_t w = warp; w < n_active; w += n_warps) {
        const size_t e = (size_t)color * B.color_stride + w;
        const uint32_t r = __ldg(B.color_rep + e);
        const Replica& R = B.rep[r];
        if (round >= R.rounds) continue;  // warp-uniform
        const Geometry& g = R.g;
        const uint32_t* cs = A.cell_start + R.cell_base;
        uint32_t m[3] = {0, 0, 0};
        unpack_m<DIM>(__ldg(A.color_cells + e), m);
        const uint32_t cell = cell_index<DIM>(g, m);
        const FlatStencil fs = flat_stencil<DIM>(g, cs, m, lane);
        const uint32_t start = __ldg(cs + cell);
        const uint32_t count = __ldg(cs + cell + 1) - start;
        Sfc64 rng = make_rng(R.step, R.substep + round, R.seed, (uint64_t)cell);
        const uint32_t k = start + canon_range_u32(rng, count);
        const double4 b4 = A.sorted_b[k];
        double x[3] = {b4.x, b4.y, b4.z};
        double dv[3];
        ball_sample<DIM>(rng, R.max_move, A.zig_x, A.zig_f, dv);
        const double u = uniform01(rng);
#pragma unroll
        for (int a = 0; a < DIM; ++a) x[a] = dadd(x[a], dv[a]);
        wrap_inv<DIM>(g.L, g.invL, x);
        uint32_t mt[3];
        if (!(point_to_space<DIM>(g, x, mt) && cell_index<DIM>(g, mt) == cell)) continue;
        double t[3] = {x[0], x[1], DIM == 3 ? x[2] : 0.0};
        wrap_inv<DIM>(g.L, g.invL, t);
        grid_dependency_wait();  // the previous colour's moves are visible from here on
        allow_dependent_launch();
        const double4 s4 = ldg4(A.sorted_s + k);
        const double si[3] = {s4.x, s4.y, s4.z};
        double e_new, e_old, mag;
        lj_energy64<DIM, true, false, U>(g, A, R.p, t, si, fs, k, true, lane, e_new, e_old, mag);
        const double du = dsub(e_new, e_old);
        const double e0 = exp(ddiv(-du, R.kt));
        if (lane == 0 && order_ambiguous(du, mag, fs.total, u, R.kt, e0)) pst.ambiguous++;
        if ((du <= 0.0 || u < e0) && lane == 0) {
            n_accepted++;
            atomicAdd(B.accepted + r, 1ull);
            double sv[3] = {t[0], t[1], t[2]};
            wrap_inv<DIM>(g.L, g.invL, sv);
            A.sorted_b[k] = make_double4(t[0], t[1], t[2], 0.0);
            A.sorted_s[k] = make_double4(sv[0], sv[1], sv[2], 0.0);
            A.sorted_off[k] = cell_offsets<DIM>(g, sv, m);
            A.body_pos[A.sorted_body[k]] = make_double4(t[0], t[1], t[2], 0.0);
        }
        __syncwarp();
    }
    grid_dependency_wait();
    allow_dependent_launch();
    flush_stats(A.stats, pst, n_accepted);
}

// The FP32 + recheck pass over a batch: k_sweep_lj32 (four trials per block, an undecided
// trial rechecked by the whole block in the FP64 pass's order) with each trial's geometry and
// parameters from its replica; the owner also publishes its replica for the helping warps.
template <int DIM, int MINB = HMC_LJ_BATCH_MIN_BLOCKS, int U = 1>
__global__ void __launch_bounds__(128, MINB)
    k_sweep_batch_lj32(Batch B, Arrays A, uint32_t color, uint32_t round, uint32_t early_wait) {
    if (early_wait) grid_dependency_wait();  // first pass: the rebuild's arrays are read at once
    if (round == kRoundFromDevice) round = *B.round_dev;  // a captured sweep's rounds loop
    __shared__ double s_e[kRecheckChunks][2][32];
    __shared__ SharedTrial s_trial;
    __shared__ uint32_t s_active, s_rep;
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    uint32_t n_accepted = 0;
    PairStats pst;
    if (threadIdx.x == 0) s_active = active_count(A, color, round);
    __syncthreads();
    const uint32_t n_active = s_active;  // block-uniform: the loop below holds barriers
    for (uint32_t base = blockIdx.x * 4u; base < n_active; base += gridDim.x * 4u) {
        const uint32_t w = base + wib;
        uint32_t m[3] = {0, 0, 0};
        uint32_t k = 0, r = 0;
        double t[3] = {0.0, 0.0, 0.0};
        double u = 0.0;
        bool trial = false;
        FlatStencil fs{0u, 0u, 0u, 0.f, 0.f};
        if (w < n_active) {  // warp-uniform
            const size_t e = (size_t)color * B.color_stride + w;
            r = __ldg(B.color_rep + e);
            const Replica& R = B.rep[r];
            if (round < R.rounds) {
                const Geometry& g = R.g;
                const uint32_t* cs = A.cell_start + R.cell_base;
                unpack_m<DIM>(__ldg(A.color_cells + e), m);
                const uint32_t cell = cell_index<DIM>(g, m);
                fs = flat_stencil<DIM>(g, cs, m, lane);
                const uint32_t start = __ldg(cs + cell);
                const uint32_t count = __ldg(cs + cell + 1) - start;
                Sfc64 rng = make_rng(R.step, R.substep + round, R.seed, (uint64_t)cell);
                k = start + canon_range_u32(rng, count);
                const double4 b4 = A.sorted_b[k];
                double x[3] = {b4.x, b4.y, b4.z};
                double dv[3];
                ball_sample<DIM>(rng, R.max_move, A.zig_x, A.zig_f, dv);
                u = uniform01(rng);
#pragma unroll
                for (int a = 0; a < DIM; ++a) x[a] = dadd(x[a], dv[a]);
                wrap_inv<DIM>(g.L, g.invL, x);
                uint32_t mt[3];
                trial = point_to_space<DIM>(g, x, mt) && cell_index<DIM>(g, mt) == cell;
                t[0] = x[0];
                t[1] = x[1];
                t[2] = DIM == 3 ? x[2] : 0.0;
                wrap_inv<DIM>(g.L, g.invL, t);
            }
        }
        grid_dependency_wait();  // the previous colour's moves are visible from here on
        allow_dependent_launch();
        int decision = 0;
        float d32 = 0.f;
        if (trial) {
            const Replica& R = B.rep[r];
            const float4 t32 = cell_offsets<DIM>(R.g, t, m);
            const float4 c32 = __ldg(A.sorted_off + k);
            const Sums32 s = lj_energy32<DIM, U>(R.g, A, R.p, t32, c32, (int)m[DIM - 1], fs, k, lane);
            pst.checks += s.pairs;
            decision = decide32(s, R.kt, u);
            d32 = s.e_new - s.e_old;
        }
        const bool unsure = decision < 0;
        if (__syncthreads_or(unsure)) {
            for (uint32_t o = 0; o < 4u; ++o) {
                const bool mine = unsure && wib == o;
                if (mine) {
                    s_trial.lo[lane] = fs.lo;
                    s_trial.pre[lane] = fs.pre;
                    if (lane == 0) {
                        const Geometry& g = B.rep[r].g;
                        const double4 c4 = ldg4(A.sorted_b + k);
                        double si[3] = {c4.x, c4.y, c4.z};
                        wrap_inv<DIM>(g.L, g.invL, si);
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            s_trial.t[a] = t[a];
                            s_trial.si[a] = si[a];
                        }
                        s_trial.total = fs.total;
                        s_trial.self = k;
                        s_rep = r;
                    }
                }
                if (!__syncthreads_or(mine)) continue;  // also publishes s_trial and s_rep
                const Replica& RO = B.rep[s_rep];
                const uint32_t total = s_trial.total, self = s_trial.self;
                const uint32_t n_chunks = (total + 31u) / 32u;
                double ea = 0.0, eb = 0.0, em = 0.0;
                for (uint32_t c0 = 0; c0 < n_chunks; c0 += kRecheckChunks) {
                    const uint32_t c1 = min(c0 + kRecheckChunks, n_chunks);
                    for (uint32_t c = c0 + wib; c < c1; c += 4u) {
                        const uint32_t j = c * 32u + lane;
                        double en = 0.0, eo = 0.0;
                        if (j < total) {
                            const uint32_t q = shared_slot(s_trial, j);
                            if (q != self) {
                                const double4 b4 = ldg4(A.sorted_b + q);
                                double sv[3] = {b4.x, b4.y, b4.z};
                                wrap_inv<DIM>(RO.g.L, RO.g.invL, sv);
                                en = lj_only64(RO.p, ref_dist2<DIM>(RO.g, s_trial.t, sv));
                                eo = lj_only64(RO.p, ref_dist2<DIM>(RO.g, s_trial.si, sv));
                            }
                        }
                        s_e[c - c0][0][lane] = en;
                        s_e[c - c0][1][lane] = eo;
                    }
                    __syncthreads();
                    if (wib == o) {
                        for (uint32_t c = c0; c < c1; ++c) {
                            ea = dadd(ea, s_e[c - c0][0][lane]);
                            eb = dadd(eb, s_e[c - c0][1][lane]);
                            em += fabs(s_e[c - c0][0][lane]) + fabs(s_e[c - c0][1][lane]);
                        }
                    }
                    __syncthreads();
                }
                if (wib == o) {
                    const double du = dsub(warp_sum(ea), warp_sum(eb));
                    const double mag = warp_sum(em);
                    const double e0 = exp(ddiv(-du, RO.kt));
                    if (lane == 0) {
                        pst.rechecks++;
                        pst.ambiguous += order_ambiguous(du, mag, total, u, RO.kt, e0) ? 1u : 0u;
                        const double err = fabs((double)d32 - du);
                        pst.max_err = err > pst.max_err ? err : pst.max_err;
                    }
                    decision = (du <= 0.0 || u < e0) ? 1 : 0;
                }
            }
        }
        if (decision == 1 && lane == 0) {
            const Geometry& g = B.rep[r].g;
            n_accepted++;
            atomicAdd(B.accepted + r, 1ull);
            double sv[3] = {t[0], t[1], t[2]};
            wrap_inv<DIM>(g.L, g.invL, sv);
            A.sorted_b[k] = make_double4(t[0], t[1], t[2], 0.0);
            A.sorted_off[k] = cell_offsets<DIM>(g, sv, m);
            A.body_pos[A.sorted_body[k]] = make_double4(t[0], t[1], t[2], 0.0);
        }
        __syncwarp();
    }
    grid_dependency_wait();
    allow_dependent_launch();
    flush_stats(A.stats, pst, n_accepted);
}

// Injected moves: warp per move. delta_h gets dU64 (stencils around the trial's space for the
// final energy and around the body's space for the initial energy); the decision follows the
// precision mode with the given uniform.
template <int DIM, bool FP32>
__global__ void __launch_bounds__(128) k_eval_lj(Geometry g, Arrays A, Pair P, const uint64_t* bodies,
                                                 const double4* trial, const double* uu, double kt, uint32_t n,
                                                 uint8_t* decisions, uint8_t* rechecked, double* delta_h) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    PairStats pst;
    if (i < n) {
        const uint32_t k = A.slot_of_body[bodies[i]];
        const double4 w4 = trial[i];
        double t[3] = {w4.x, w4.y, DIM == 3 ? w4.z : 0.0};
        wrap_inv<DIM>(g.L, g.invL, t);
        const double4 s4 = ldg4(A.sorted_s + k);
        const double si[3] = {s4.x, s4.y, s4.z};
        uint32_t mt[3], mi[3];
        const bool ok = point_to_space<DIM>(g, t, mt) && point_to_space<DIM>(g, si, mi);
        uint8_t dec = 0, rech = 0;
        double du = 0.0;
        if (ok) {
            const FlatStencil ft = flat_stencil<DIM>(g, A.cell_start, mt, lane);
            const FlatStencil fi = flat_stencil<DIM>(g, A.cell_start, mi, lane);
            double e_new, e_old, unused;
            double mag_new, mag_old;
            lj_energy64<DIM, false>(g, A, P, t, nullptr, ft, k, true, lane, e_new, unused, mag_new);
            lj_energy64<DIM, false>(g, A, P, si, nullptr, fi, k, true, lane, e_old, unused, mag_old);
            du = dsub(e_new, e_old);
            const double u = uu[i];
            bool dec64 = du <= 0.0 || u < exp(ddiv(-du, kt));
            dec = dec64 ? 1 : 0;
            if (FP32) {
                // FP32 sums need a common space for both sites: when the trial left the body's
                // space, they are evaluated in FP64 as the sweep never sees such a trial.
                const bool same = mt[0] == mi[0] && mt[1] == mi[1] && (DIM == 2 || mt[2] == mi[2]);
                if (same) {
                    const float4 t32 = cell_offsets<DIM>(g, t, mt);
                    const float4 c32 = __ldg(A.sorted_off + k);
                    const Sums32 s = lj_energy32<DIM>(g, A, P, t32, c32, (int)mt[DIM - 1], ft, k, lane);
                    const float d32 = s.e_new - s.e_old;
                    const float b = s.err + (float)(s.terms + 7) * kU32 * s.mag * 1.01f + kU32 * fabsf(d32) +
                                    1e-9f * (s.mag + 1.f);
                    int d = -1;
                    if (isfinite(d32) && isfinite(b)) {
                        const double lo = (double)d32 - b, hi = (double)d32 + b;
                        if (hi <= 0.0) {
                            d = 1;
                        } else if (lo > 0.0) {
                            const double t_hi = exp(-lo / kt) * (1.0 + 1e-12), t_lo = exp(-hi / kt) * (1.0 - 1e-12);
                            d = u < t_lo ? 1 : (u >= t_hi ? 0 : -1);
                        }
                    }
                    if (d < 0) {
                        rech = 1;
                        d = dec64 ? 1 : 0;  // the FP64 recheck
                    }
                    dec = (uint8_t)d;
                } else {
                    rech = 1;
                }
            }
        } else if (lane == 0) {
            atomicOr(&A.stats->error_flags, kErrOutsideCheckerboard);
        }
        if (lane == 0) {
            decisions[i] = dec;
            rechecked[i] = rech;
            delta_h[i] = du;
        }
    }
    flush_stats(A.stats, pst, 0u);
}

// The sequential-stream tuner for Lennard-Jones and the overlap penalty (tune_stream_run):
// dH = E_final - E_initial in FP64 (the warp over the stencils of the trial site's and of the
// current site's spaces), then the reference's test: rejected at dH = inf, accepted at dH <= 0
// without a uniform, else the stream's next uniform against exp(-dH / kT). A decision that
// another summation order could change (order_ambiguous; also a dH <= 0 whose bound reaches
// above 0, where another order would draw a uniform) is counted in J.ambiguous.
template <int DIM>
__global__ void __launch_bounds__(32) k_tune_stream_lj(TuneJob* jobs, uint32_t n_jobs) {
    if (blockIdx.x >= n_jobs) return;
    TuneJob& J = jobs[blockIdx.x];
    const Geometry& g = J.g;
    const Arrays& A = J.a;
    const Pair& P = J.p;
    const uint32_t lane = threadIdx.x & 31u;
    unsigned long long ambiguous = 0;
    tune_stream_run(
        J, [&](Sfc64& rng, double m, uint32_t b, double* x, double*) { tune_translate<DIM>(rng, g, A, m, b, x); },
        [&](Sfc64& rng, uint32_t b, const double* x, const double*) -> bool {
            double t[3] = {x[0], x[1], x[2]};
            wrap_inv<DIM>(g.L, g.invL, t);
            const uint32_t k = A.slot_of_body[b];
            const double4 s4 = ldg4(A.sorted_s + k);
            const double si[3] = {s4.x, s4.y, s4.z};
            uint32_t mt[3] = {0, 0, 0}, mi[3] = {0, 0, 0};
            if (!(point_to_space<DIM>(g, t, mt) && point_to_space<DIM>(g, si, mi))) {
                if (lane == 0) atomicOr(&A.stats->error_flags, kErrOutsideCheckerboard);
                return false;
            }
            const FlatStencil ft = flat_stencil<DIM>(g, A.cell_start, mt, lane);
            const FlatStencil fi = flat_stencil<DIM>(g, A.cell_start, mi, lane);
            double e_new, e_old, unused, mag_new, mag_old;
            lj_energy64<DIM, false>(g, A, P, t, nullptr, ft, k, true, lane, e_new, unused, mag_new);
            if (e_new == __longlong_as_double(0x7ff0000000000000ll)) return false;  // the reference stops here
            lj_energy64<DIM, false>(g, A, P, si, nullptr, fi, k, true, lane, e_old, unused, mag_old);
            const double du = dsub(e_new, e_old);
            if (!(du != __longlong_as_double(0x7ff0000000000000ll))) return false;
            const uint32_t n = ft.total + fi.total;
            const double mag = mag_new + mag_old;
            if (du <= 0.0) {
                if (isfinite(mag) && du + order_bound(du, mag, n) > 0.0) ambiguous++;
                return true;
            }
            const double u = uniform01(rng);
            const double e0 = exp(ddiv(-du, J.kt));
            if (order_ambiguous(du, mag, n, u, J.kt, e0)) ambiguous++;
            return u < e0;
        });
    if (lane == 0) J.ambiguous = ambiguous;
}

// Total pair energy, pairs (i < j) in FP64 (PairwiseCutoff::total_energy,
// pairwise_cutoff.rs:720-745); one thread per body, atomically summed.
template <int DIM>
__global__ void k_energy_lj(Geometry g, Arrays A, Pair P, uint32_t n, double* out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (k < n) {
        const uint32_t bi = A.sorted_body[k];
        const double4 s4 = A.sorted_s[k];
        const double t[3] = {s4.x, s4.y, s4.z};
        uint32_t m[3];
        uint32_t c = A.body_cell[bi];
#pragma unroll
        for (int a = DIM - 1; a >= 0; --a) {
            m[a] = c % g.shape[a];
            c /= g.shape[a];
        }
        for_each_neighbor<DIM>(g, A.cell_start, m, [&](uint32_t q, const float*) -> bool {
            if (A.sorted_body[q] <= bi) return false;
            const double4 o4 = A.sorted_s[q];
            const double sv[3] = {o4.x, o4.y, o4.z};
            e += lj_pair64(P, ref_dist2<DIM>(g, t, sv));
            return false;
        });
        atomicAdd(out, e);
    }
}

}  // namespace

cudaError_t launch_sweep_lj(int dim, bool fp32, bool generic, const Geometry& g, const Arrays& a, const Pair& p,
                            const Launch& l, cudaStream_t s, uint32_t variant) {
    if (l.n_active == 0) return cudaSuccess;
    static int max_blocks = 0;
    if (max_blocks == 0) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        max_blocks = sms * 16;
    }
    uint32_t blocks = (l.n_active + 3) / 4;  // four warps (trials) per block
    if (blocks > (uint32_t)max_blocks) blocks = (uint32_t)max_blocks;
    PassLaunch pl(blocks, l.overlap_previous != 0 || l.early_wait != 0, s);
    using LjKernel = void (*)(Geometry, Arrays, Pair, Launch, Injected);
    // the compiled launch variants, in the order of kLjShapes ([dim == 3][fp32][variant])
    // (variants 3 and 4 take two candidates per lane and step)
    static const LjKernel kernels[2][2][5] = {
        {{k_sweep_lj<2, false, 9, false>, k_sweep_lj<2, false, 7, false>, k_sweep_lj<2, false, 11, false>,
          k_sweep_lj<2, false, 7, false, 2>, k_sweep_lj<2, false, 9, false, 2>},
         {k_sweep_lj32<2, false, 9>, k_sweep_lj32<2, false, 7>, k_sweep_lj32<2, false, 11>,
          k_sweep_lj32<2, false, 7, 2>, k_sweep_lj32<2, false, 9, 2>}},
        {{k_sweep_lj<3, false, 9, false>, k_sweep_lj<3, false, 7, false>, k_sweep_lj<3, false, 11, false>,
          k_sweep_lj<3, false, 7, false, 2>, k_sweep_lj<3, false, 9, false, 2>},
         {k_sweep_lj32<3, false, 9>, k_sweep_lj32<3, false, 7>, k_sweep_lj32<3, false, 11>,
          k_sweep_lj32<3, false, 7, 2>, k_sweep_lj32<3, false, 9, 2>}}};
    // the overlap penalty and Isotropic: the FP64 pass with the dispatching pair energy
    static const LjKernel generic_kernels[2][5] = {
        {k_sweep_lj<2, false, 9, true>, k_sweep_lj<2, false, 7, true>, k_sweep_lj<2, false, 11, true>,
         k_sweep_lj<2, false, 7, true, 2>, k_sweep_lj<2, false, 9, true, 2>},
        {k_sweep_lj<3, false, 9, true>, k_sweep_lj<3, false, 7, true>, k_sweep_lj<3, false, 11, true>,
         k_sweep_lj<3, false, 7, true, 2>, k_sweep_lj<3, false, 9, true, 2>}};
    static_assert(n_shapes(kLjShapes) == 5, "one compiled kernel per Lennard-Jones variant");
    const LjKernel k = generic ? generic_kernels[dim == 3][variant < 5 ? variant : 0]
                               : kernels[dim == 3][fp32][variant < 5 ? variant : 0];
    return cudaLaunchKernelEx(&pl.cfg, k, g, a, p, l, Injected{});
}

cudaError_t launch_propose_lj(int dim, bool fp32, const Geometry& g, const Arrays& a, const Launch& l, cudaStream_t s) {
    const uint64_t n = (uint64_t)g.color_stride << dim;
    if (n == 0) return cudaSuccess;
    static int max_blocks = 0;
    if (max_blocks == 0) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        max_blocks = sms * 16;
    }
    uint32_t blocks = (uint32_t)((n + 127) / 128);
    if (blocks > (uint32_t)max_blocks) blocks = (uint32_t)max_blocks;
    if (dim == 2)
        fp32 ? k_propose_lj<2, true><<<blocks, 128, 0, s>>>(g, a, l) : k_propose_lj<2, false><<<blocks, 128, 0, s>>>(g, a, l);
    else
        fp32 ? k_propose_lj<3, true><<<blocks, 128, 0, s>>>(g, a, l) : k_propose_lj<3, false><<<blocks, 128, 0, s>>>(g, a, l);
    return cudaGetLastError();
}

cudaError_t launch_tune_stream_lj(int dim, TuneJob* jobs, uint32_t n_jobs, cudaStream_t s) {
    if (n_jobs == 0) return cudaSuccess;
    if (dim == 2)
        k_tune_stream_lj<2><<<n_jobs, 32, 0, s>>>(jobs, n_jobs);
    else
        k_tune_stream_lj<3><<<n_jobs, 32, 0, s>>>(jobs, n_jobs);
    return cudaGetLastError();
}

cudaError_t launch_trials_lj(int dim, bool fp32, const Geometry& g, const Arrays& a, const Pair& p, double kt,
                             const Injected& j, cudaStream_t s) {
    if (j.n == 0) return cudaSuccess;
    Launch l{};
    l.kt = kt;
    const uint32_t blocks = (j.n + 3) / 4;  // four warps (trials) per block
    if (dim == 2) {
        if (fp32)
            k_sweep_lj32<2, true><<<blocks, 128, 0, s>>>(g, a, p, l, j);
        else
            k_sweep_lj<2, true><<<blocks, 128, 0, s>>>(g, a, p, l, j);
    } else {
        if (fp32)
            k_sweep_lj32<3, true><<<blocks, 128, 0, s>>>(g, a, p, l, j);
        else
            k_sweep_lj<3, true><<<blocks, 128, 0, s>>>(g, a, p, l, j);
    }
    return cudaGetLastError();
}

cudaError_t launch_sweep_batch_lj(int dim, bool fp32, const Batch& b, const Arrays& a, uint32_t color, uint32_t round,
                                  uint32_t max_active, bool overlap_previous, bool early_wait, cudaStream_t s,
                                  uint32_t variant) {
    if (max_active == 0) return cudaSuccess;
    static int max_blocks = 0;
    if (max_blocks == 0) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        max_blocks = sms * 16;
    }
    uint32_t blocks = (max_active + 3) / 4;  // four warps (trials) per block
    if (blocks > (uint32_t)max_blocks) blocks = (uint32_t)max_blocks;
    PassLaunch pl(blocks, overlap_previous || early_wait, s);
    const uint32_t ew = early_wait ? 1u : 0u;
    using BatchLjKernel = void (*)(Batch, Arrays, uint32_t, uint32_t, uint32_t);
    // the compiled launch variants, in the order of kBatchLjShapes ([dim == 3][fp32][variant])
    // (variants 3 and 4 take two candidates per lane and step)
    static const BatchLjKernel kernels[2][2][5] = {
        {{k_sweep_batch_lj<2, 7>, k_sweep_batch_lj<2, 9>, k_sweep_batch_lj<2, 5>, k_sweep_batch_lj<2, 7, 2>,
          k_sweep_batch_lj<2, 9, 2>},
         {k_sweep_batch_lj32<2, 7>, k_sweep_batch_lj32<2, 9>, k_sweep_batch_lj32<2, 5>, k_sweep_batch_lj32<2, 7, 2>,
          k_sweep_batch_lj32<2, 9, 2>}},
        {{k_sweep_batch_lj<3, 7>, k_sweep_batch_lj<3, 9>, k_sweep_batch_lj<3, 5>, k_sweep_batch_lj<3, 7, 2>,
          k_sweep_batch_lj<3, 9, 2>},
         {k_sweep_batch_lj32<3, 7>, k_sweep_batch_lj32<3, 9>, k_sweep_batch_lj32<3, 5>, k_sweep_batch_lj32<3, 7, 2>,
          k_sweep_batch_lj32<3, 9, 2>}}};
    static_assert(n_shapes(kBatchLjShapes) == 5, "one compiled kernel per Lennard-Jones batch variant");
    return cudaLaunchKernelEx(&pl.cfg, kernels[dim == 3][fp32][variant < 5 ? variant : 0], b, a, color, round, ew);
}

cudaError_t launch_eval_lj(int dim, bool fp32, const Geometry& g, const Arrays& a, const Pair& p,
                           const uint64_t* bodies, const double4* trial, const double* u, double kt, uint32_t n,
                           uint8_t* decisions, uint8_t* rechecked, double* delta_h, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const uint32_t blocks = (n + 3) / 4;
    if (dim == 2) {
        if (fp32)
            k_eval_lj<2, true><<<blocks, 128, 0, s>>>(g, a, p, bodies, trial, u, kt, n, decisions, rechecked, delta_h);
        else
            k_eval_lj<2, false><<<blocks, 128, 0, s>>>(g, a, p, bodies, trial, u, kt, n, decisions, rechecked, delta_h);
    } else {
        if (fp32)
            k_eval_lj<3, true><<<blocks, 128, 0, s>>>(g, a, p, bodies, trial, u, kt, n, decisions, rechecked, delta_h);
        else
            k_eval_lj<3, false><<<blocks, 128, 0, s>>>(g, a, p, bodies, trial, u, kt, n, decisions, rechecked, delta_h);
    }
    return cudaGetLastError();
}

cudaError_t launch_energy_lj(int dim, const Geometry& g, const Arrays& a, const Pair& p, uint32_t n, double* out,
                             cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    if (dim == 2)
        k_energy_lj<2><<<(n + 127) / 128, 128, 0, s>>>(g, a, p, n, out);
    else
        k_energy_lj<3><<<(n + 127) / 128, 128, 0, s>>>(g, a, p, n, out);
    return cudaGetLastError();
}

}  // namespace hmc
