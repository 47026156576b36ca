// Sweep::apply_with_filter (hoomd-mc/src/sweep.rs:159-224) for hard and overlap-penalty disks
// and spheres, and QuickInsert's insertion loop: one
// trial per body in index order, all from ONE sequential random stream
// Counter(step, substep, seed).make_rng() (index 0), each trial seeing every earlier accepted
// move. The chain is sequential by definition, so one warp runs it: the 32 lanes keep the same
// stream and trial, and each lane tests the sites of one cell of the 3^d stencil around the
// trial site (cells at least one diameter wide, kept current after every accepted move). This
// is the exact serial Markov chain on the device, not a fast path: the checkerboard sweep is.
#include <cuda_runtime.h>

#include "hmc_serial.cuh"

namespace hmc {
namespace {

// Soft pair energy (Lennard-Jones or the overlap penalty) of site t against every site of the
// stencil around t's cell except body `self`: per-lane sums over the lane's cell, then a
// butterfly reduction (all lanes agree). mag += sum |e|, terms += the sites visited (for
// order_ambiguous).
template <int DIM>
__device__ __forceinline__ double serial_energy(const Geometry& g, const SerialGrid& G, const Pair& P, const double* t,
                                                uint32_t self, uint32_t lane, double& mag, uint32_t& terms) {
    uint32_t m[3] = {0, 0, 0}, cell;
    serial_cell<DIM>(g, G, t, m);
    double e = 0.0, am = 0.0;
    uint32_t cnt = 0;
    if (lane_cell<DIM>(G, m, lane, &cell)) {
        cnt = G.size[cell];
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t j = G.items[(size_t)cell * G.cap + k];
            if (j == self) continue;
            const double4 s4 = G.site[j];
            const double sv[3] = {s4.x, s4.y, s4.z};
            const double r2 = ref_dist2<DIM>(g, t, sv);
            const double x = lj_pair64(P, r2);
            e = dadd(e, x);
            am += soft_pair_mag(P, r2, x);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        e = dadd(e, __shfl_xor_sync(0xffffffffu, e, o));
        am += __shfl_xor_sync(0xffffffffu, am, o);
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    }
    mag += am;
    terms += cnt;
    return e;
}

// SOFT = false: hard spheres (the trial is rejected on any overlap, no uniform is drawn).
// SOFT = true: the overlap penalty; dH = E(trial site) - E(current site) and the Metropolis
// test of sweep.rs:207-209 (u drawn from the stream only when 0 < dH < inf).
template <int DIM, bool SOFT>
__global__ void __launch_bounds__(32) k_serial_sphere(Geometry g, Arrays A, SerialGrid G, Pair P, Launch L,
                                                      const uint8_t* __restrict__ mask) {
    const uint32_t lane = threadIdx.x;
    if (A.stats->error_flags) return;
    Sfc64 rng = make_rng(L.step, L.substep, L.seed, 0);
    uint64_t accepted = 0, ambiguous = 0;
    for (uint32_t b = 0; b < L.n_bodies; ++b) {
        if (mask && !mask[b]) continue;
        const double4 b4 = A.body_pos[b];
        double x[3] = {b4.x, b4.y, b4.z};
        double dv[3];
        ball_sample<DIM>(rng, L.max_move, A.zig_x, A.zig_f, dv);
#pragma unroll
        for (int a = 0; a < DIM; ++a) x[a] = dadd(x[a], dv[a]);
        wrap_inv<DIM>(g.L, g.invL, x);  // wrap(propose(..)) = W1
        double t[3] = {x[0], x[1], DIM == 3 ? x[2] : 0.0};
        wrap_inv<DIM>(g.L, g.invL, t);  // delta_energy_one wraps the site: T = wrap(W1)
        if (SOFT) {
            double mag = 0.0;
            uint32_t terms = 0;
            const double ef = serial_energy<DIM>(g, G, P, t, b, lane, mag, terms);
            if (ef == __longlong_as_double(0x7ff0000000000000ll)) continue;  // early infinity
            const double4 s4 = G.site[b];
            const double si[3] = {s4.x, s4.y, s4.z};
            const double dh = dsub(ef, serial_energy<DIM>(g, G, P, si, b, lane, mag, terms));
            if (!(dh != __longlong_as_double(0x7ff0000000000000ll))) continue;
            bool acc;
            if (dh <= 0.0) {
                // another summation order could give dH > 0, draw a uniform and change the stream
                if (isfinite(mag) && dh + order_bound(dh, mag, terms) > 0.0) ambiguous++;
                acc = true;
            } else {
                const double u = uniform01(rng);
                const double e0 = exp(ddiv(-dh, L.kt));
                if (order_ambiguous(dh, mag, terms, u, L.kt, e0)) ambiguous++;
                acc = u < e0;
            }
            if (!acc) continue;
        } else {
            uint32_t m[3] = {0, 0, 0}, cell;
            serial_cell<DIM>(g, G, t, m);
            bool overlap = false;
            if (lane_cell<DIM>(G, m, lane, &cell)) {
                const uint32_t cnt = G.size[cell];
                for (uint32_t k = 0; k < cnt && !overlap; ++k) {
                    const uint32_t j = G.items[(size_t)cell * G.cap + k];
                    if (j == b) continue;
                    const double4 s4 = G.site[j];
                    const double sv[3] = {s4.x, s4.y, s4.z};
                    overlap = ref_dist2<DIM>(g, t, sv) < P.sigma2;
                }
            }
            if (__any_sync(0xffffffffu, overlap)) continue;
        }
        accepted++;
        if (lane == 0) {
            // update_body_properties: body = wrap(W1) = T, site = wrap(body)
            double sv[3] = {t[0], t[1], t[2]};
            wrap_inv<DIM>(g.L, g.invL, sv);
            A.body_pos[b] = make_double4(t[0], t[1], t[2], 0.0);
            G.site[b] = make_double4(sv[0], sv[1], sv[2], 0.0);
            serial_move<DIM>(g, G, A, b, sv);
        }
        __syncwarp();
        if (A.stats->error_flags) break;
    }
    if (lane == 0) {
        A.stats->accepted = accepted;
        A.stats->rechecks = 0;
        A.stats->ambiguous = ambiguous;
    }
}

// QuickInsert::apply's insertion loop (hoomd-mc/src/quick_insert.rs:243-265): up to `attempts`
// bodies drawn from UniformIn (per axis Uniform(low, low + scale), rand's UniformFloat: 52 bits
// in [1, 2) minus 1, times scale, plus low) from one stream; a body whose insertion energy is
// finite is appended (Microstate::add_body: B = wrap(x), S = wrap(B)); the loop stops once
// `to_insert` bodies are in or `allowed` inserted bodies overlapped (energy > 0). The insertion
// energy is evaluated at wrap(x) (filtered_body_energy_final, pairwise_cutoff.rs:420-450); only
// whether it is infinite or positive matters, and with non-negative pair energies both follow
// from single pairs, so no sum is formed. out: inserted, overlapping, rejected, final n.
template <int DIM>
__global__ void __launch_bounds__(32) k_quick_insert(Geometry g, Arrays A, SerialGrid G, Pair P, Launch L,
                                                     QuickInsertArgs q, BodyTags T, unsigned long long* out) {
    const uint32_t lane = threadIdx.x;
    if (A.stats->error_flags) return;
    Sfc64 rng = make_rng(L.step, L.substep, L.seed, 0);
    uint32_t n = q.n0;
    uint64_t inserted = 0, overlapping = 0, rejected = 0;
    for (uint64_t attempt = 0; attempt < q.attempts; ++attempt) {
        double x[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
            const double u = dsub(as_double(0x3FF0000000000000ULL | (rng.next_u64() >> 12)), 1.0);
            x[a] = dadd(dmul(u, q.scale[a]), q.low[a]);
        }
        double t[3] = {x[0], x[1], x[2]};
        wrap_inv<DIM>(g.L, g.invL, t);
        uint32_t m[3] = {0, 0, 0}, cell;
        serial_cell<DIM>(g, G, t, m);
        bool inf = false, pos = false;
        if (lane_cell<DIM>(G, m, lane, &cell)) {
            const uint32_t cnt = G.size[cell];
            for (uint32_t k = 0; k < cnt && !inf; ++k) {
                const uint32_t j = G.items[(size_t)cell * G.cap + k];
                const double4 s4 = G.site[j];
                const double sv[3] = {s4.x, s4.y, s4.z};
                const double r2 = ref_dist2<DIM>(g, t, sv);
                if (q.soft) {
                    const double e = penalty_pair64(P, r2);
                    inf = e == __longlong_as_double(0x7ff0000000000000ll);
                    pos = pos || e > 0.0;
                } else {
                    inf = r2 < P.sigma2;
                }
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
        if (lane == 0) grid_append<DIM>(g, A, G, T, n, x);
        __syncwarp();
        n++;
        inserted++;
        if (pos) overlapping++;
        if (inserted == q.to_insert || overlapping >= q.allowed) break;
        if (A.stats->error_flags) break;
    }
    if (lane == 0) {
        out[0] = inserted;
        out[1] = overlapping;
        out[2] = rejected;
        out[3] = n;
    }
}

// Insertion energy at site t (no body excluded): the overlap penalty's sum, or 0 / infinity for
// hard spheres.
template <int DIM>
__device__ __forceinline__ double insert_energy(const Geometry& g, const SerialGrid& G, const Pair& P,
                                                const double* t, bool soft, uint32_t lane) {
    double mag = 0.0;
    uint32_t terms = 0;
    if (soft) return serial_energy<DIM>(g, G, P, t, 0xffffffffu, lane, mag, terms);
    uint32_t m[3] = {0, 0, 0}, cell;
    serial_cell<DIM>(g, G, t, m);
    bool overlap = false;
    if (lane_cell<DIM>(G, m, lane, &cell)) {
        const uint32_t cnt = G.size[cell];
        for (uint32_t k = 0; k < cnt && !overlap; ++k) {
            const double4 s4 = G.site[G.items[(size_t)cell * G.cap + k]];
            const double sv[3] = {s4.x, s4.y, s4.z};
            overlap = ref_dist2<DIM>(g, t, sv) < P.sigma2;
        }
    }
    return __any_sync(0xffffffffu, overlap) ? __longlong_as_double(0x7ff0000000000000ll) : 0.0;
}

// GrandCanonical::apply (hoomd-mc/src/grand_canonical.rs:49-110), n_trials times in sequence,
// trial i drawing from Counter(step, substep + i, seed): a fair coin (rand's bool: the sign bit
// of next_u32) picks insertion (a UniformIn body, kept when V f exp(-dU/kT) / (N + 1) > u) or
// removal (a body by random_range(..N), removed when N exp(-dU/kT) / (V f) > u, or always for
// f <= 0) with swap_remove. out: insert accepted / rejected, remove accepted / rejected, final N.
template <int DIM>
__global__ void __launch_bounds__(32) k_grand_canonical(Geometry g, Arrays A, SerialGrid G, Pair P,
                                                        GrandCanonicalArgs q, BodyTags T, unsigned long long* out) {
    const uint32_t lane = threadIdx.x;
    if (A.stats->error_flags) return;
    uint32_t n = q.n0;
    unsigned long long ia = 0, ir = 0, ra = 0, rr = 0;
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    for (uint32_t t = 0; t < q.n_trials; ++t) {
        Sfc64 rng = make_rng(q.step, q.substep + t, q.seed, 0);
        if (n == 0 && q.fugacity <= 0.0) continue;
        const bool insert = (int32_t)rng.next_u32() < 0;
        if (insert) {
            double x[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int a = 0; a < DIM; ++a) {
                const double u = dsub(as_double(0x3FF0000000000000ULL | (rng.next_u64() >> 12)), 1.0);
                x[a] = dadd(dmul(u, q.scale[a]), q.low[a]);
            }
            double tt[3] = {x[0], x[1], x[2]};
            wrap_inv<DIM>(g.L, g.invL, tt);
            const double de = insert_energy<DIM>(g, G, P, tt, q.soft != 0, lane);
            bool accept = false;
            if (de != inf && de == de) {  // is_finite
                const double p =
                    ddiv(dmul(dmul(q.volume, q.fugacity), exp(ddiv(-de, q.temperature))), dadd((double)n, 1.0));
                accept = p > uniform01(rng);
            }
            if (accept) {
                if (n >= q.capacity) {
                    if (lane == 0) atomicOr(&A.stats->error_flags, kErrCellOverflow);
                    break;
                }
                if (lane == 0) grid_append<DIM>(g, A, G, T, n, x);
                __syncwarp();
                n++;
                ia++;
            } else {
                ir++;
            }
        } else if (n > 0) {
            const uint32_t idx = canon_range_u32(rng, n);
            double e_initial = 0.0;
            if (q.soft) {
                const double4 s4 = G.site[idx];
                const double si[3] = {s4.x, s4.y, s4.z};
                double mag = 0.0;
                uint32_t terms = 0;
                e_initial = serial_energy<DIM>(g, G, P, si, idx, lane, mag, terms);
            }
            const double de = -e_initial;  // delta_energy_remove
            const double p = q.fugacity <= 0.0
                                 ? 1.0
                                 : ddiv(dmul((double)n, exp(ddiv(-de, q.temperature))), dmul(q.volume, q.fugacity));
            if (p > uniform01(rng)) {
                if (lane == 0) {
                    // Microstate::remove_body (microstate.rs:917-943): the last body takes idx
                    const uint32_t last = n - 1;
                    const uint32_t oc = G.cell_of[idx];
                    const uint32_t osz = G.size[oc];
                    for (uint32_t k = 0; k < osz; ++k)
                        if (G.items[(size_t)oc * G.cap + k] == idx) {
                            G.items[(size_t)oc * G.cap + k] = G.items[(size_t)oc * G.cap + osz - 1];
                            break;
                        }
                    G.size[oc] = osz - 1;
                    if (T.tag) tag_free(T, T.tag[idx]);
                    if (idx != last) {
                        const uint32_t lc = G.cell_of[last];
                        const uint32_t lsz = G.size[lc];
                        for (uint32_t k = 0; k < lsz; ++k)
                            if (G.items[(size_t)lc * G.cap + k] == last) {
                                G.items[(size_t)lc * G.cap + k] = idx;
                                break;
                            }
                        A.body_pos[idx] = A.body_pos[last];
                        G.site[idx] = G.site[last];
                        G.cell_of[idx] = lc;
                        if (T.tag) T.tag[idx] = T.tag[last];
                    }
                }
                __syncwarp();
                n--;
                ra++;
            } else {
                rr++;
            }
        }
        if (A.stats->error_flags) break;
    }
    if (lane == 0) {
        out[0] = ia;
        out[1] = ir;
        out[2] = ra;
        out[3] = rr;
        out[4] = n;
    }
}

}  // namespace

namespace {
}  // namespace

cudaError_t launch_serial_sphere(int dim, bool soft, const Geometry& g, const Arrays& a, const Pair& p,
                                 const Launch& l, const uint32_t* nc, const double* w, uint32_t cap, uint32_t* size,
                                 uint32_t* items, uint32_t* cell_of, double4* site, const uint8_t* mask,
                                 cudaStream_t s) {
    const SerialGrid G = make_grid(dim, nc, w, cap, size, items, cell_of, site);
    const uint32_t n = l.n_bodies;
    cudaError_t e = build_grid(dim, g, a, G, n, s);
    if (e != cudaSuccess || n == 0) return e;
    if (dim == 2) {
        if (soft)
            k_serial_sphere<2, true><<<1, 32, 0, s>>>(g, a, G, p, l, mask);
        else
            k_serial_sphere<2, false><<<1, 32, 0, s>>>(g, a, G, p, l, mask);
    } else {
        if (soft)
            k_serial_sphere<3, true><<<1, 32, 0, s>>>(g, a, G, p, l, mask);
        else
            k_serial_sphere<3, false><<<1, 32, 0, s>>>(g, a, G, p, l, mask);
    }
    return cudaGetLastError();
}

cudaError_t launch_quick_insert(int dim, const Geometry& g, const Arrays& a, const Pair& p, const Launch& l,
                                const QuickInsertArgs& q, const BodyTags& tags, const uint32_t* nc, const double* w,
                                uint32_t cap, uint32_t* size, uint32_t* items, uint32_t* cell_of, double4* site,
                                unsigned long long* out, cudaStream_t s) {
    const SerialGrid G = make_grid(dim, nc, w, cap, size, items, cell_of, site);
    cudaError_t e = build_grid(dim, g, a, G, q.n0, s);
    if (e != cudaSuccess) return e;
    if (dim == 2)
        k_quick_insert<2><<<1, 32, 0, s>>>(g, a, G, p, l, q, tags, out);
    else
        k_quick_insert<3><<<1, 32, 0, s>>>(g, a, G, p, l, q, tags, out);
    return cudaGetLastError();
}

cudaError_t launch_grand_canonical(int dim, const Geometry& g, const Arrays& a, const Pair& p,
                                   const GrandCanonicalArgs& q, const BodyTags& tags, const uint32_t* nc,
                                   const double* w, uint32_t cap, uint32_t* size, uint32_t* items, uint32_t* cell_of,
                                   double4* site, unsigned long long* out, cudaStream_t s) {
    const SerialGrid G = make_grid(dim, nc, w, cap, size, items, cell_of, site);
    cudaError_t e = build_grid(dim, g, a, G, q.n0, s);
    if (e != cudaSuccess) return e;
    if (dim == 2)
        k_grand_canonical<2><<<1, 32, 0, s>>>(g, a, G, p, q, tags, out);
    else
        k_grand_canonical<3><<<1, 32, 0, s>>>(g, a, G, p, q, tags, out);
    return cudaGetLastError();
}

}  // namespace hmc
