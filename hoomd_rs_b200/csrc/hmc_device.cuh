// Device helpers shared by the sweep kernels of every interaction: checkerboard maps,
// the reference's FP64 image-rule distance, trial moves, the stencil walk over cell-ordered
// rows and the per-warp statistics.
#pragma once

#include <cuda_runtime.h>

#include "hmc_internal.cuh"

namespace hmc {

// Outcome of a pair scan.
enum : int { kClear = 0, kOverlap = 1, kUncertain = 2 };

// ---- checkerboard maps --------------------------------------------------------------------
// point_to_space_index for a periodic checkerboard (hypercuboid.rs:85-128). Returns false
// for None. m receives the multi-index.
template <int DIM>
__device__ __forceinline__ bool point_to_space(const Geometry& g, const double* x, uint32_t* m) {
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
        double p = dsub(x[a], g.origin[a]);
        double f = floor(div_fixed(p, g.width[a], g.invW[a]));
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

// ref_dist2 that also returns the per-axis difference d = t - image of the chosen image.
template <int DIM>
__device__ __forceinline__ double ref_disp(const Geometry& g, const double* t, const double* s, double* dout) {
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
        dout[a] = d;
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
        double p[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
        for (int i = 0; i < 3; ++i) {
            double z = standard_normal(r, zx, zf);
            if (i == 0)
                p[0] = z;
            else if (i == 1)
                p[1] = z;
            else
                p[2] = z;
        }
        double norm = dsqrt(dot<3>(p, p));
        double u = uniform01(r);
        double scale = dmul(ddiv(radius, norm), portable_cbrt(u));
        out[0] = dmul(p[0], scale);
        out[1] = dmul(p[1], scale);
        out[2] = dmul(p[2], scale);
    }
}

// ---- neighbour stencil over cell-ordered rows ----------------------------------------------
__device__ __forceinline__ uint32_t wrap_index(int i, uint32_t n) {
    return i < 0 ? (uint32_t)(i + (int)n) : ((uint32_t)i >= n ? (uint32_t)i - n : (uint32_t)i);
}

// Packed multi-index of a space in a colour list: 10 bits per axis in 3-D, 16 in 2-D.
template <int DIM>
__device__ __forceinline__ uint32_t pack_m(const uint32_t* m) {
    return DIM == 3 ? (m[0] | (m[1] << 10) | (m[2] << 20)) : (m[0] | (m[1] << 16));
}
template <int DIM>
__device__ __forceinline__ void unpack_m(uint32_t p, uint32_t* m) {
    if (DIM == 3) {
        m[0] = p & 1023u;
        m[1] = (p >> 10) & 1023u;
        m[2] = p >> 20;
    } else {
        m[0] = p & 0xffffu;
        m[1] = p >> 16;
    }
}

// Rows of the 3^DIM stencil around space m, as ranges of cell-ordered slots. A row is
// the run of three spaces m[last]-1 .. m[last]+1 along the fast axis at one offset of the
// slow axes; it is contiguous unless it wraps around the fast axis (m[last] at either end).
// Row r (r = 3*(i0+1) + (i1+1) in 3-D, i1+1 in 2-D) has slow-axis offsets (i0, i1). When a
// slow axis has two spaces its offset -1 names the same space as +1; that row is left empty.
template <int DIM>
constexpr int kRows = DIM == 3 ? 9 : 3;

// Row ranges of the stencil around space m: for each of the 3^(DIM-1) rows along the fast
// (last) axis, [a0, a1) covers the contiguous spaces lo .. hi-1 of that row in cell order.
// A slow axis with two spaces contributes each neighbour row once.
template <int DIM>
__device__ __forceinline__ void load_rows(const Geometry& g, const uint32_t* __restrict__ cs, const uint32_t* m,
                                          uint32_t lo, uint32_t hi, uint32_t* a0, uint32_t* a1) {
    const uint32_t sf = g.shape[DIM - 1];
#pragma unroll
    for (int r = 0; r < kRows<DIM>; ++r) {
        int i0 = DIM == 3 ? r / 3 - 1 : 0;
        int i1 = DIM == 3 ? r % 3 - 1 : r - 1;
        uint32_t base;
        bool skip;
        if (DIM == 3) {
            uint32_t c0 = wrap_index((int)m[0] + i0, g.shape[0]);
            uint32_t c1 = wrap_index((int)m[1] + i1, g.shape[1]);
            skip = (i0 == -1 && g.shape[0] == 2) || (i1 == -1 && g.shape[1] == 2);
            base = (c0 * g.shape[1] + c1) * sf;
        } else {
            uint32_t c0 = wrap_index((int)m[0] + i1, g.shape[0]);
            skip = i1 == -1 && g.shape[0] == 2;
            base = c0 * sf;
        }
        a0[r] = skip ? 0u : __ldg(cs + base + lo);
        a1[r] = skip ? 0u : __ldg(cs + base + hi);
    }
}

// The fast-axis span of the row ranges: spaces mf-1 .. mf+1 when they are contiguous; at
// the two ends of a periodic fast axis the span stops at the end and the wrapped space
// (sf-1 for mf = 0, 0 for mf = sf-1) is covered by a second pass with `wrapped_lo`.
__device__ __forceinline__ void row_span(uint32_t sf, uint32_t mf, uint32_t* lo, uint32_t* hi) {
    *lo = sf == 2 ? 0u : (mf == 0 ? 0u : mf - 1u);
    *hi = sf == 2 ? 2u : (mf + 1u == sf ? sf : mf + 2u);
}

// Generic stencil walk (any position of m, including the fast-axis ends): calls
// f(q, slow_shift) for every slot q of the 3^DIM spaces around m and stops when f returns
// true. Each space is visited once, also when an axis has two spaces.
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
                uint32_t c0 = wrap_index((int)m[0] + i0, g.shape[0]);
                uint32_t c1 = wrap_index((int)m[1] + i1, g.shape[1]);
                row_base = (c0 * g.shape[1] + c1) * sf;
                slow_shift[0] = (float)i0 * g.w32[0];
                slow_shift[1] = (float)i1 * g.w32[1];
            } else {
                uint32_t c0 = wrap_index((int)m[0] + i1, g.shape[0]);
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

// The stencil around space m spread over a warp, for the kernels that give a trial one warp:
// lane i < 2·kRows holds part i%2 of row i/2 (part 1 is the wrapped space of a row at a
// fast-axis end, empty elsewhere) as a slot range, with the row's slow-axis shifts and the
// exclusive prefix of the parts' lengths. The warp then takes the stencil's candidates 32 at
// a time (flat_slot), whatever the lengths of the single rows.
struct FlatStencil {
    uint32_t lo, pre;  // this lane's part: first slot; candidates in the parts before it
    uint32_t total;    // candidates in the whole stencil (the same in every lane)
    float s0, s1;      // slow-axis shifts of this lane's row
};

// Part `wrapped_part` of stencil row r around space m (the row's spaces m[last]-1 .. m[last]+1,
// split where the fast axis wraps): its first slot and length, and the row's slow-axis shifts.
// A row repeated on a two-space slow axis, and the wrapped part of a row that does not wrap,
// are empty.
template <int DIM>
__device__ __forceinline__ void stencil_part(const Geometry& g, const uint32_t* __restrict__ cs, const uint32_t* m,
                                             int r, bool wrapped_part, uint32_t& lo, uint32_t& len, float& s0,
                                             float& s1) {
    const int i0 = DIM == 3 ? r / 3 - 1 : 0;
    const int i1 = DIM == 3 ? r % 3 - 1 : r - 1;
    const uint32_t sf = g.shape[DIM - 1], mf = m[DIM - 1];
    uint32_t base;
    bool skip;
    if (DIM == 3) {
        skip = (i0 == -1 && g.shape[0] == 2) || (i1 == -1 && g.shape[1] == 2);
        base = (wrap_index((int)m[0] + i0, g.shape[0]) * g.shape[1] + wrap_index((int)m[1] + i1, g.shape[1])) * sf;
        s0 = (float)i0 * g.w32[0];
        s1 = (float)i1 * g.w32[1];
    } else {
        skip = i1 == -1 && g.shape[0] == 2;
        base = wrap_index((int)m[0] + i1, g.shape[0]) * sf;
        s0 = (float)i1 * g.w32[0];
        s1 = 0.f;
    }
    // spaces [a, b) of the row along the fast axis
    uint32_t a = 0, b = 0;
    if (sf == 2) {
        b = wrapped_part ? 0u : 2u;
    } else if (mf >= 1 && mf + 1 < sf) {
        if (!wrapped_part) a = mf - 1, b = mf + 2;
    } else if (mf == 0) {
        if (wrapped_part) a = sf - 1, b = sf;
        else a = 0, b = 2;
    } else {
        if (wrapped_part) a = 0, b = 1;
        else a = sf - 2, b = sf;
    }
    lo = 0;
    len = 0;
    if (!skip && a < b) {
        lo = __ldg(cs + base + a);
        len = __ldg(cs + base + b) - lo;
    }
}

// Call with all 32 lanes of the warp. wrapped_only: only the wrapped parts (the spaces across
// the fast-axis end from a space at an end).
template <int DIM>
__device__ __forceinline__ FlatStencil flat_stencil(const Geometry& g, const uint32_t* __restrict__ cs,
                                                    const uint32_t* m, uint32_t lane, bool wrapped_only = false) {
    FlatStencil fs{0u, 0u, 0u, 0.f, 0.f};
    uint32_t len = 0;
    if (lane < 2u * kRows<DIM> && (!wrapped_only || (lane & 1u)))
        stencil_part<DIM>(g, cs, m, (int)(lane >> 1), (lane & 1u) != 0, fs.lo, len, fs.s0, fs.s1);
    const unsigned full = 0xffffffffu;
    uint32_t x = len;
#pragma unroll
    for (uint32_t o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(full, x, o);
        if (lane >= o) x += y;
    }
    fs.total = __shfl_sync(full, x, 31);
    fs.pre = x - len;
    return fs;
}

// Candidate j of the stencil (valid for j < total; all 32 lanes call this together): its
// slot, and the lane holding its part. The prefixes grow with the lane (empty parts repeat
// the next part's prefix), so the part is the last lane whose prefix is at most j.
__device__ __forceinline__ uint32_t flat_slot(const FlatStencil& fs, uint32_t j, uint32_t& part) {
    const unsigned full = 0xffffffffu;
    uint32_t s = 0;
#pragma unroll
    for (uint32_t step = 16; step > 0; step >>= 1) {
        const uint32_t p = __shfl_sync(full, fs.pre, s + step);
        if (p <= j) s += step;
    }
    part = s;
    return __shfl_sync(full, fs.lo, s) + (j - __shfl_sync(full, fs.pre, s));
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
    uint32_t ambiguous = 0;  // soft-potential decisions that the summation order could change
    double max_err = 0.0;
};

// The FP32 displacement (trial minus candidate) from the FP32 offsets, given the shift of
// the candidate's space corner along the slow axes and its fast-axis space offset dm.
template <int DIM>
__device__ __forceinline__ float fp32_dist2(const Geometry& g, float4 t32, float4 o, float s0, float s1, int dm) {
    float d[3];
    if (DIM == 3) {
        d[0] = t32.x - (o.x + s0);
        d[1] = t32.y - (o.y + s1);
        d[2] = t32.z - (o.z + (float)dm * g.w32[2]);
    } else {
        d[0] = t32.x - (o.x + s0);
        d[1] = t32.y - (o.y + (float)dm * g.w32[1]);
        d[2] = 0.f;
    }
    if (g.any_two) {
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
    return dd;
}

// The length of the colour's list of non-empty spaces for this pass, or 0 when the pass is
// beyond the sweep's rounds or the rebuild flagged an error (the state then stays untouched).
__device__ __forceinline__ uint32_t active_count(const Arrays& A, uint32_t color, uint32_t round) {
    const DeviceStats* st = A.stats;
    if (st->error_flags != 0u || round >= st->rounds) return 0u;
    return st->color_count[color];
}

// Whether another order of the same FP64 sums could change the Metropolis decision. The pair
// energies are the same numbers in any order, and recursive summation of n terms in any order
// (any summation tree) lies within gamma_{n-1} sum|e| of the exact sum, gamma_k = k u / (1 - k u),
// u = 2^-53 (Higham, Accuracy and Stability of Numerical Algorithms, 2nd ed., 2002, section
// 4.2). So dU = E_final - E_initial summed in any two orders (this pass's lanes and
// butterfly, the reference's cell-list order) differ by at most
// B = 2 gamma_{n-1} (sum|e_final| + sum|e_initial|) + 2 u |dU|. The decision (dU <= 0, else
// u < exp(-dU / kT), parallel_sweep.rs:267-268) is monotone in dU: it is the same in every order
// when dU - B and dU + B decide alike, with exp allowed 4 ulp either way (the reference calls
// the platform libm, this pass CUDA's exp). n = the candidates of the stencil (>= the terms);
// e0 = exp(-dU / kT) as the decision computed it. Over [dU - B, dU + B] exp(-x / kT) stays
// within a factor exp(B / kT) <= 1 + 2 B / kT of e0 (B / kT < 1e-3), so a uniform farther than
// e0 (4 B / kT + 1e-14) from e0 settles the trial without evaluating the ends.
__device__ __forceinline__ double order_bound(double du, double mag, uint32_t n) {
    const double unit = 1.1102230246251565e-16;  // 2^-53
    const double k = (double)(n > 1u ? n - 1u : 1u);
    const double gamma = k * unit / (1.0 - k * unit);
    return 1.01 * (2.0 * gamma * mag + 2.0 * unit * fabs(du)) + 1e-300;
}
__device__ __forceinline__ bool order_ambiguous(double du, double mag, uint32_t n, double u, double kt, double e0) {
    if (!isfinite(du) || !isfinite(mag)) return false;  // an infinite pair energy decides in any order
    const double unit = 1.1102230246251565e-16;        // 2^-53
    const double b = order_bound(du, mag, n);
    const double lo = du - b, hi = du + b;
    if (hi <= 0.0) return false;  // accepted in every order, without a uniform
    const double rel = b / kt;
    if (lo > 0.0 && rel < 1e-3 && fabs(u - e0) > e0 * (4.0 * rel + 1e-14)) return false;
    const double ulp4 = 8.0 * unit;
    const bool acc_at_lo = lo <= 0.0 || u < exp(-lo / kt) * (1.0 + ulp4);
    const bool acc_at_hi = u < exp(-hi / kt) * (1.0 - ulp4);
    return acc_at_lo != acc_at_hi;
}

// OverlapPenalty::energy (overlap_penalty.rs:109-115) at r = -d, d an approximate separation:
// infinite below -maximum_allowed_overlap, (0.5 k) r^2 + epsilon_shoulder below 0, else 0.
__device__ __forceinline__ double separation_penalty(const ShapeOverlap& so, double d) {
    const double r = -d;
    if (r < -so.dmax) return __longlong_as_double(0x7ff0000000000000ll);
    if (r < 0.0) return dadd(dmul(so.half_k, dmul(r, r)), so.shoulder);
    return 0.0;
}

// Butterfly sum over the warp (every lane ends with the same value).
__device__ __forceinline__ double warp_sum64(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ---- the sequential-stream tuner -------------------------------------------------------------
// tune_local_trial (hoomd-mc/src/tune_local.rs:42-88) on one warp for job J (TuneJob). Every lane
// runs the same single stream Counter(step, substep, seed).make_rng() (index 0), so the trial is
// computed redundantly and stays warp-uniform; only the pair work is spread over the lanes.
// Per sample: random_range(0..n) for the body (rand's UniformUsize samples a u32 for ranges
// that fit one: Canon's method, as IndexedRandom::choose), propose(rng, m, b, x, q) writes
// W1 = wrap(propose(..)) and the proposed orientation, and accept(rng, b, x, q) decides the trial
// (drawing the uniform itself when 0 < dH < infinity, as the reference does). After each round:
// maximum *= (acceptance + 1.5) / (target + 1.5) (tune_by_scaling, lib.rs:514-524), clamped at
// J.cap for rotations.
template <typename Propose, typename Accept>
__device__ __forceinline__ void tune_stream_run(TuneJob& J, Propose&& propose, Accept&& accept) {
    Sfc64 rng = make_rng(J.step, J.substep, J.seed, 0);
    double m = J.maximum;
    uint32_t acc = 0;
    for (uint32_t t = 0; t < J.steps; ++t) {
        acc = 0;
        for (uint32_t j = 0; j < J.samples; ++j) {
            const uint32_t b = canon_range_u32(rng, J.n_bodies);
            double x[3] = {0.0, 0.0, 0.0}, q[4] = {1.0, 0.0, 0.0, 0.0};
            propose(rng, m, b, x, q);
            if (accept(rng, b, x, q)) acc++;
        }
        const double ratio = ddiv((double)acc, (double)J.samples);
        m = dmul(m, ddiv(dadd(ratio, 1.5), dadd(J.target, 1.5)));
        if (J.cap > 0.0 && m > J.cap) m = J.cap;
    }
    if ((threadIdx.x & 31u) == 0) {
        J.maximum = m;
        J.accepted = acc;
    }
}

// Translate<Cartesian<DIM>>::propose (translate/cartesian.rs:40-51) of body b, then wrap.
template <int DIM>
__device__ __forceinline__ void tune_translate(Sfc64& rng, const Geometry& g, const Arrays& A, double m, uint32_t b,
                                               double* x) {
    const double4 b4 = A.body_pos[b];
    x[0] = b4.x;
    x[1] = b4.y;
    x[2] = DIM == 3 ? b4.z : 0.0;
    double dv[3];
    ball_sample<DIM>(rng, m, A.zig_x, A.zig_f, dv);
#pragma unroll
    for (int a = 0; a < DIM; ++a) x[a] = dadd(x[a], dv[a]);
    wrap_inv<DIM>(g.L, g.invL, x);
}

__device__ __forceinline__ void flush_stats(DeviceStats* stats, const PairStats& st, uint32_t accepted) {
    const unsigned full = 0xffffffffu;
    unsigned acc = __reduce_add_sync(full, accepted);
    unsigned checks = __reduce_add_sync(full, st.checks);
    unsigned rech = __reduce_add_sync(full, st.rechecks);
    if ((threadIdx.x & 31) == 0) {
        if (acc) atomicAdd(&stats->accepted, (unsigned long long)acc);
        if (checks) atomicAdd(&stats->pair_checks, (unsigned long long)checks);
        if (rech) atomicAdd(&stats->rechecks, (unsigned long long)rech);
    }
    if (st.max_err > 0.0) atomicMax(&stats->max_err_bits, (unsigned long long)__double_as_longlong(st.max_err));
    if (st.ambiguous) atomicAdd(&stats->ambiguous, (unsigned long long)st.ambiguous);
}


}  // namespace hmc
