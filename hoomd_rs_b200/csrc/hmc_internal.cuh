// Internal types shared by the kernels (hmc_kernels.cu) and the C ABI (hmc_capi.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "hmc_math.cuh"

namespace hmc {

// Device-side error flags (DeviceStats::error_flags).
enum : uint32_t {
    kErrOutsideCheckerboard = 1u << 0,
    kErrNonFinite = 1u << 1,
    kErrAngleRange = 1u << 2,  // a 2-D orientation angle at or beyond 2^19 rad
    kErrCellOverflow = 1u << 3,  // a cell of the serial sweep's grid is full
    kErrIterationCap = 1u << 4,  // an approximate separation loop ran past ShapeOverlap::max_steps
    kErrAborted = 1u << 5,       // a sweep of a pipelined call after one that stopped the call
};

// Counters written by the kernels. Zeroed by the host before a sweep.
struct DeviceStats {
    unsigned long long accepted;
    unsigned long long rechecks;
    unsigned long long pair_checks;
    unsigned long long max_err_bits;  // bits of the largest non-negative FP32 error
    unsigned int nonempty;            // non-empty checkerboard spaces after a rebuild
    unsigned int error_flags;
    unsigned long long overlaps;      // pairs found by the overlap check
    unsigned int color_count[8];      // non-empty spaces per colour after a rebuild
    unsigned int rounds;              // full colour sets of the sweep: ceil(N / non-empty spaces)
    unsigned long long ambiguous;     // soft-potential trials whose decision the order of the
                                      // FP64 pair-energy sum could change (order_ambiguous)
};

// The checkerboard (hoomd-mc/src/hypercuboid.rs) together with the periodic box.
struct Geometry {
    double L[3];        // box edge lengths
    double half[3];     // L / 2
    double ghost_hi[3]; // half - boundary_range: a site beyond has an image at x - L
    double ghost_lo[3]; // -half + boundary_range: a site below has an image at x + L
    double origin[3];   // checkerboard origin (shifted each sweep)
    double width[3];    // space width
    double invL[3];     // RN(1 / L), for div_fixed
    double invW[3];     // RN(1 / width), for div_fixed
    float w32[3];       // width rounded to FP32
    uint32_t shape[3];  // spaces per axis (even)
    uint32_t half_shape[3];
    uint32_t n_cells;
    uint32_t color_stride;  // capacity of one colour's list of non-empty spaces (n_cells >> dim)
    uint32_t any_two;       // some axis has exactly two spaces (minimum-image fix-up needed)
};

// Sorted (cell-ordered) and body-ordered device arrays of one system.
struct Arrays {
    double4* body_pos;       // [n] body positions B, body order (x, y, z, 0)
    double4* body_ori;       // [n] body versors (s, x, y, z), body order; may be null
    double4* sorted_b;       // [n] body positions B in cell order (proposal source)
    double4* sorted_s;       // [n] site positions S = wrap(B) in cell order (neighbour tests)
    float4* sorted_off;      // [n] FP32 offsets of S from its cell corner; .w = fast-axis cell index bits
    double4* sorted_q;       // [n] versors in cell order; may be null
    uint32_t* sorted_body;   // [n] cell-order slot -> body index
    uint32_t* slot_of_body;  // [n] body index -> cell-order slot
    uint32_t* body_cell;     // [n]
    uint32_t* body_rank;     // [n]
    uint32_t* body_m;        // [n] packed multi-index of each body's space (from the binning pass)
    uint32_t* cell_count;    // [cells]
    uint32_t* cell_start;    // [cells + 1]
    uint32_t* block_sums;    // scan scratch
    uint32_t* color_cells;   // [cells] per-colour lists of non-empty spaces, packed multi-indices
    DeviceStats* stats;
    uint32_t* abort_word;    // pipelined sweeps: nonzero once a sweep stopped the call (may be null)
    const double* zig_x;     // ziggurat tables (257 each)
    const double* zig_f;
    // A round's trial moves, one per colour-list entry (soft potentials: k_propose_lj writes them
    // before the round's colour passes, which give each trial a warp): trial site T = wrap(W1) and
    // the Metropolis uniform in trial_t, T's FP32 offsets in trial_o, the chosen slot in trial_k
    // (kNoTrial when the move leaves its space or the entry is empty).
    double4* trial_t;        // [cells]
    float4* trial_o;         // [cells]
    uint32_t* trial_k;       // [cells]
    double4* trial_q;        // [cells] shapes: the proposed versor (2-D: the angle in .x)
};
constexpr uint32_t kNoTrial = 0xffffffffu;

// Pair interaction parameters.
struct Pair {
    double sigma2;     // HardSphere diameter^2
    float sig2_lo32;   // FP32 certain-overlap threshold (sigma^2 - bound, rounded down)
    float sig2_hi32;   // FP32 certain-clear threshold (sigma^2 + bound, rounded up)
    // Isotropic<Shifted<LennardJones>> (isotropic.rs:147-156, shifted.rs:92-94,
    // lennard_jones.rs:107-111)
    double lj_sigma;
    double lj_four_eps;   // 4.0 * epsilon
    double lj_rcut2;      // r_cut.powi(2)
    double lj_e_shift;    // LennardJones::energy(r_shift)
    float lj_sigma2_32;   // sigma^2 in FP32
    float lj_four_eps32;
    float lj_e_shift32;
    float lj_rcut2_lo32;  // r_cut^2 minus the r^2 error bound: below, the pair is inside for certain
    float lj_rcut2_hi32;  // r_cut^2 plus the bound: at or above, outside for certain
    float lj_disp_err;    // per-axis FP32 displacement error bound E
    float lj_band_energy; // bound on |pair energy| for a pair inside the cut-off band
    // Isotropic<Expanded<OverlapPenalty>> (overlap_penalty.rs:109-115, expanded.rs:64-66):
    // r^2 >= r_cut^2 -> 0; x = sqrt(r^2) - delta; x < -d_max -> inf; x < 0 -> (0.5 k) x^2 + eps
    uint32_t penalty;     // the soft pair energy: 0 Lennard-Jones, 1 the overlap penalty, 2 Isotropic (below)
    double op_rcut2;      // r_cut.powi(2)
    double op_delta;
    double op_dmax;       // maximum_allowed_overlap
    double op_half_k;     // 0.5 * k
    double op_shoulder;   // epsilon_shoulder
    // Isotropic { W(F), r_cut } for the univariates of hmc_univariate (hmc.h): penalty = 2
    uint32_t uv_kind, uv_wrap;  // hmc_univariate, hmc_univariate_wrap
    double uv_p[4];             // F's parameters (WeeksChandlerAnderson: p[2] = 2^(1/6), the host's pow)
    double uv_w[2];             // W's parameters: Shifted {r_shift}, Expanded {delta}, Xplor {r_cut, r_smooth}
    double uv_shift;            // Shifted: F(r_shift), evaluated once on the host with the same arithmetic
    double uv_rcut2;            // Isotropic::r_cut.powi(2)
};

// The univariate energies of hoomd-interaction/src/univariate/*.rs in FP64 with the reference's
// order of operations: LennardJones<12, 6> (lennard_jones.rs:107-111, powi by repeated squaring),
// WeeksChandlerAnderson (LJ + epsilon below 2^(1/6) sigma), Harmonic (0.5 k (r - r_0) (r - r_0)),
// HarmonicRepulsion (0.5 a / r_cut (r - r_cut)^2 below r_cut), Boxcar (epsilon on [left, right)),
// OverlapPenalty (overlap_penalty.rs:109-115).
enum : uint32_t { kUvLennardJones = 0, kUvWca = 1, kUvHarmonic = 2, kUvHarmonicRepulsion = 3, kUvBoxcar = 4,
                  kUvOverlapPenalty = 5, kUvLjGauss = 6 };
enum : uint32_t { kUvwNone = 0, kUvwShifted = 1, kUvwExpanded = 2, kUvwXplor = 3 };
__device__ __forceinline__ double univariate64(uint32_t kind, const double* p, double r) {
    switch (kind) {
        case kUvLennardJones:
        case kUvWca: {
            if (kind == kUvWca && !(r < dmul(p[2], p[1]))) return 0.0;
            const double sr = ddiv(p[1], r);
            const double s2 = dmul(sr, sr), s4 = dmul(s2, s2), s8 = dmul(s4, s4);
            const double e = dmul(dmul(4.0, p[0]), dsub(dmul(s4, s8), dmul(s2, s4)));
            return kind == kUvWca ? dadd(e, p[0]) : e;
        }
        case kUvHarmonic: {
            const double d = dsub(r, p[1]);
            return dmul(dmul(dmul(0.5, p[0]), d), d);
        }
        case kUvHarmonicRepulsion: {
            if (!(r < p[1])) return 0.0;
            const double d = dsub(r, p[1]);
            return dmul(ddiv(dmul(0.5, p[0]), p[1]), dmul(d, d));
        }
        case kUvBoxcar:
            return r < p[1] ? 0.0 : (r < p[2] ? p[0] : 0.0);
        case kUvLjGauss: {  // lennard_jones_gauss.rs: r_inv^12 - 2 r_inv^6 - eps exp(-(r / scale - r_0)^2 / (2 s^2))
            const double ri = ddiv(p[3], r);
            const double x = dsub(ddiv(r, p[3]), p[2]);
            const double arg = ddiv(-dmul(x, x), dmul(2.0, p[1]));
            const double s2 = dmul(ri, ri), s4 = dmul(s2, s2), s8 = dmul(s4, s4);
            return dsub(dsub(dmul(s4, s8), dmul(2.0, dmul(s2, s4))), dmul(p[0], exp(arg)));
        }
        default:
            if (r < -p[1]) return __longlong_as_double(0x7ff0000000000000ll);
            if (r < 0.0) return dadd(dmul(dmul(0.5, p[0]), dmul(r, r)), p[2]);
            return 0.0;
    }
}
// Isotropic::site_pair_energy (isotropic.rs:147-156) of W(F): Shifted (shifted.rs:92-94),
// Expanded (expanded.rs:64-66) or Xplor (xplor.rs: s(r) F(r), s the smoothing polynomial between
// r_smooth and r_cut).
__device__ __forceinline__ double isotropic_pair64(const Pair& P, double r2) {
    if (r2 >= P.uv_rcut2) return 0.0;
    double r = dsqrt(r2);
    switch (P.uv_wrap) {
        case kUvwShifted:
            return dsub(univariate64(P.uv_kind, P.uv_p, r), P.uv_shift);
        case kUvwExpanded:
            return univariate64(P.uv_kind, P.uv_p, dsub(r, P.uv_w[0]));
        case kUvwXplor: {
            double sm;
            if (r < P.uv_w[1]) {
                sm = 1.0;
            } else if (r > P.uv_w[0]) {
                sm = 0.0;
            } else {
                const double r_sq = dmul(r, r), rc_sq = dmul(P.uv_w[0], P.uv_w[0]), rs_sq = dmul(P.uv_w[1], P.uv_w[1]);
                const double a = dsub(rc_sq, r_sq), d = dsub(rc_sq, rs_sq);
                sm = ddiv(dmul(dmul(a, a), dsub(dadd(rc_sq, dmul(2.0, r_sq)), dmul(3.0, rs_sq))), dmul(dmul(d, d), d));
            }
            return dmul(sm, univariate64(P.uv_kind, P.uv_p, r));
        }
        default:
            return univariate64(P.uv_kind, P.uv_p, r);
    }
}

// The overlap penalty's pair energy in FP64 with the reference's operation order.
__device__ __forceinline__ double penalty_pair64(const Pair& P, double r2) {
    if (r2 >= P.op_rcut2) return 0.0;
    const double x = dsub(dsqrt(r2), P.op_delta);
    if (x < -P.op_dmax) return __longlong_as_double(0x7ff0000000000000ll);
    if (x < 0.0) return dadd(dmul(P.op_half_k, dmul(x, x)), P.op_shoulder);
    return 0.0;
}

// Soft pair energy in FP64 exactly as the reference evaluates it: the overlap penalty above, or
// Isotropic::site_pair_energy (isotropic.rs:147-156: r^2 >= r_cut^2 -> 0, else energy(sqrt(r^2)))
// of Shifted (shifted.rs:92-94: f(r) - f(r_shift)) LennardJones (lennard_jones.rs:107-111:
// 4 eps ((sigma/r)^12 - (sigma/r)^6) with powi by repeated squaring).
__device__ __forceinline__ double lj_only64(const Pair& P, double r2) {
    if (r2 >= P.lj_rcut2) return 0.0;
    const double r = dsqrt(r2);
    const double sr = ddiv(P.lj_sigma, r);
    const double s2 = dmul(sr, sr), s4 = dmul(s2, s2), s8 = dmul(s4, s4);
    return dsub(dmul(P.lj_four_eps, dsub(dmul(s4, s8), dmul(s2, s4))), P.lj_e_shift);
}
// The magnitude a soft pair energy adds to the order bound: |e|, and for LennardJonesGauss
// 16 |epsilon| more (its exp is the device's, within a few ulp of the platform's, on the pair's
// energy and on a Shifted constant; exp of a non-positive argument is at most 1).
__device__ __forceinline__ double soft_pair_mag(const Pair& P, double r2, double e) {
    if (P.penalty == 2u && P.uv_kind == kUvLjGauss && r2 < P.uv_rcut2) return fabs(e) + 16.0 * fabs(P.uv_p[0]);
    return fabs(e);
}
__device__ __forceinline__ double lj_pair64(const Pair& P, double r2) {
    if (P.penalty) return P.penalty == 1u ? penalty_pair64(P, r2) : isotropic_pair64(P, r2);
    return lj_only64(P, r2);
}
// GENERIC = false: the kernel serves Shifted Lennard-Jones only (its FP32 passes and batches), so
// the other energies stay out of its code and registers.
template <bool GENERIC>
__device__ __forceinline__ double soft_pair64(const Pair& P, double r2) {
    return GENERIC ? lj_pair64(P, r2) : lj_only64(P, r2);
}

// One sweep launch: counter, move and colour.
struct Launch {
    uint64_t step;
    uint32_t substep;
    uint32_t seed;
    uint32_t color;       // parity offsets: bit a of color (last axis = bit 0) is the offset on axis a
    uint32_t n_active;    // upper bound of the colour's list length (grid size); the kernels read
                          // the length itself from DeviceStats::color_count
    uint32_t round;       // colour set within the sweep; kernels skip it when >= DeviceStats::rounds
    double max_move;      // Translate maximum distance
    double kt;            // Isothermal temperature
    uint32_t n_bodies;
    uint32_t overlap_previous;  // 1: the previous launch on the stream is a colour pass of the
                                // same sweep (this pass may start before it ends)
    uint32_t early_wait;        // 1: the previous launch is the rebuild's last kernel: launch
                                // early but wait for it before reading anything
};

// Injected trials for the probe mode of the colour-pass kernels (hmc_eval_trials): trial i
// moves body bodies[i] to W1 = trial[i] (the body position wrap(propose(..)) returns) with the
// versor trial_q[i] and the Metropolis uniform u[i]. The kernel then runs the pass's own
// decision code on it against the unchanged state and writes decisions[i] and flags[i]
// instead of committing the move.
struct Injected {
    const uint64_t* bodies = nullptr;
    const double4* trial = nullptr;
    const double4* trial_q = nullptr;  // shapes
    const double* u = nullptr;         // Lennard-Jones and the overlap penalty
    uint8_t* decisions = nullptr;
    uint8_t* flags = nullptr;
    uint32_t n = 0;
};
enum : uint8_t {
    kTrialRechecked = 1,     // the FP32 pass settled the trial with FP64 pair evaluations
    kTrialOutsideSpace = 2,  // W1 lies outside the body's checkerboard space (the colour pass
                             // rejects such a move before any pair test, parallel_sweep.rs:253-258)
    kTrialAmbiguous = 4,     // another summation order of the FP64 pair energies could change the
                             // Metropolis decision (order_ambiguous)
};

// One tuning run of tune_local_trial (hoomd-mc/src/tune_local.rs:42-88) with the reference's
// single sequential stream: a warp per job runs `steps` rounds of `samples` trials from
// Counter(step, substep, seed) (index 0) against the unchanged state in `a` (cell-ordered with
// FP64 sites and body slots), scaling `maximum` after each round. A system's tuning is one job;
// a batch's is one job per replica (a views the replica's part of the batch arrays).
struct TuneJob {
    Geometry g;
    Arrays a;
    Pair p;
    uint64_t step;
    uint32_t substep, seed;
    uint32_t n_bodies, samples, steps, rotate;
    double maximum;            // in: the start; out: the tuned maximum
    double kt, target;
    double cap;                // Rotate<Versor>: pi/2, Rotate<Angle>: pi; 0 = no clamp (Translate)
    unsigned long long accepted;   // out: accepted trials of the last round
    unsigned long long ambiguous;  // out: soft-potential decisions another summation order could change
};

// Launch variants of the colour-pass kernels (the autotuner's search space, hmc_autotune): each
// variant is a compiled instantiation; index 0 of every table is the default. blocks_per_sm is
// the resident-block target the kernel is compiled for (its register cap), trials_per_warp the
// trials a warp of the packed polyhedron pass takes, own_steps the candidates per row a lane of
// the warp-cooperative sphere pass tests before handing the rest to its warp. Every variant makes
// the same pair tests and decisions, so the trajectory does not depend on the choice.
struct LaunchShape {
    uint32_t blocks_per_sm, trials_per_warp, own_steps;
};
constexpr LaunchShape kSphereDirectShapes[] = {{6, 1, 0}, {5, 1, 0}, {7, 1, 0}};
constexpr LaunchShape kSphereCoopShapes[] = {{6, 1, 2}, {6, 1, 1}, {6, 1, 3}, {5, 1, 2}, {7, 1, 2}};
// Lennard-Jones and Isotropic passes; own_steps 2: two candidates per lane and step
constexpr LaunchShape kLjShapes[] = {{9, 1, 0}, {7, 1, 0}, {11, 1, 0}, {7, 1, 2}, {9, 1, 2}};
constexpr LaunchShape kPolyShapes[] = {{5, 4, 0}, {5, 2, 0}, {5, 8, 0}};
constexpr LaunchShape kBatchShapes[] = {{4, 1, 0}, {3, 1, 0}, {5, 1, 0}, {6, 1, 0}, {7, 1, 0}, {8, 1, 0}};
// The polygon pass: one compiled shape; in the FP32 mode, variant 1 runs the FP64 pass instead
// of the FP32 prefilter (the same decisions; the prefilter saves little where the FP64
// circumsphere test is cheap against the separating-axis or XenoCollide test behind it).
constexpr LaunchShape kPoly2Shapes[] = {{8, 4, 0}, {8, 4, 0}};
// the Lennard-Jones replica passes; own_steps 2: two candidates per lane and step
constexpr LaunchShape kBatchLjShapes[] = {{7, 1, 0}, {9, 1, 0}, {5, 1, 0}, {7, 1, 2}, {9, 1, 2}};
template <size_t N>
constexpr uint32_t n_shapes(const LaunchShape (&)[N]) {
    return (uint32_t)N;
}

// Blocks in one resident wave of a 128-thread kernel on the current device (SMs x resident
// blocks per SM), cached per kernel.
int resident_wave(const void* kernel);

// Launch configuration of a colour pass: 128 threads per block; overlap = programmatic
// dependent launch after the previous colour pass of the same sweep (the kernel waits with
// griddepcontrol.wait before it reads neighbour sites and lets the next pass launch after).
struct PassLaunch {
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    PassLaunch(uint32_t grid, bool overlap, cudaStream_t s, uint32_t block = 128) {
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(block);
        cfg.stream = s;
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = overlap ? 1 : 0;
    }
    PassLaunch(const PassLaunch&) = delete;
};

// In a colour pass: wait for the previous pass (a no-op without programmatic dependent
// launch), and allow the next pass to launch. Everything a pass reads before the wait was
// written before the previous pass began: the rebuild's arrays, and the bodies of the pass's
// own colour (only the same colour, one round earlier, moved them). At most two passes overlap.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void allow_dependent_launch() { asm volatile("griddepcontrol.launch_dependents;"); }

// One replica of a batch of independent boxes (hmc_batch_*): its box, checkerboard, pair
// thresholds, counter and place in the batch's concatenated arrays.
struct Replica {
    Geometry g;          // box and checkerboard; the origin is re-drawn every sweep
    Pair p;              // pair parameters and FP32 thresholds (hard spheres or Lennard-Jones)
    uint32_t cell_base;  // first space of the replica in the batch's space arrays
    uint32_t body_base;  // first body of the replica
    uint32_t n_bodies;
    uint32_t rounds;     // full colour sets of the current sweep
    uint64_t step;       // Counter at the start of the sweep
    uint32_t substep;
    uint32_t seed;
    double max_move;
    double kt;           // Isothermal kT of the current sweep (Lennard-Jones)
};

// Batch-wide tables; the Arrays of a batch span all replicas (bodies, spaces, colour lists).
struct Batch {
    const Replica* rep;             // [R]
    const uint32_t* cell_base;      // [R + 1] prefix sums of the replicas' space counts
    const uint32_t* body_rep;       // [N] replica of each body
    uint32_t* color_rep;            // [2^d * color_stride] replica of each colour-list entry
    unsigned long long* accepted;   // [R] per sweep
    unsigned int* nonempty;         // [R] after a rebuild
    unsigned long long* overlaps;   // [R] overlap check
    const uint32_t* round_dev;      // the colour set a pass launched with kRoundFromDevice runs
    uint32_t n_replicas;
    uint32_t n_cells;               // all replicas
    uint32_t color_stride;          // capacity of one colour's list
};
// The round argument of a batch pass that reads its colour set from Batch::round_dev (the passes
// of a captured sweep, whose rounds loop runs on the device).
constexpr uint32_t kRoundFromDevice = 0xffffffffu;

// What the sweeps of one captured-sweep call add up on the device: per replica the accepted and
// rejected moves (rep_counts[2 r], [2 r + 1]), and for the batch the sums of the per-sweep
// statistics, the error flags of every sweep, and the sweeps that ran.
struct BatchSweepTotals {
    unsigned long long rechecks;
    unsigned long long pair_checks;
    unsigned long long ambiguous;
    unsigned long long max_err_bits;
    unsigned long long sweeps;
    unsigned long long colour_sets;  // the colour sets (rounds) run, summed over the sweeps
    unsigned int error_flags;
    unsigned int pad;
};

// Kernel launchers (hmc_kernels.cu). All return cudaGetLastError() after enqueueing.
// write_s: also store the FP64 site positions S = wrap(B) in cell order (needed by the
// plain FP64 pair test, the overlap check and injected-move evaluation).
// write_slots: also store each body's cell-order slot (slot_of_body), which only the
// injected-move and tuner kernels read; a sweep's own rebuild skips it.
cudaError_t launch_rebuild(int dim, const Geometry& g, const Arrays& a, uint32_t n, bool write_s, cudaStream_t s,
                           bool write_slots = true);
// After a sweep of a pipelined call: raise the abort word when the sweep needed more colour sets
// than the `enqueued` ones or flagged an error.
cudaError_t launch_sweep_guard(const DeviceStats* stats, uint32_t enqueued, uint32_t* abort_word, cudaStream_t s);
// Per-replica rounds of a batch sweep into Replica::rounds, their maximum into DeviceStats::rounds.
cudaError_t launch_batch_rounds(const Batch& b, Replica* rep, DeviceStats* stats, cudaStream_t s);
// The device side of a captured batch sweep: every replica's checkerboard origin from its own
// Counter (update_checkerboard); the rounds loop's first test and its step to the next colour
// set (a while node's condition); each replica's counts and Counter after the sweep.
cudaError_t launch_batch_origins(int dim, const Batch& b, Replica* rep, cudaStream_t s);
cudaError_t launch_batch_round_first(cudaGraphConditionalHandle h, const DeviceStats* stats, uint32_t* round_dev,
                                     const BatchSweepTotals* totals, cudaStream_t s);
cudaError_t launch_batch_round_next(cudaGraphConditionalHandle h, const DeviceStats* stats, uint32_t* round_dev,
                                    cudaStream_t s);
cudaError_t launch_batch_sweep_end(const Batch& b, Replica* rep, const DeviceStats* stats,
                                   unsigned long long* rep_counts, BatchSweepTotals* totals, bool increment_step,
                                   cudaStream_t s);
// Batches of replicas: the rebuild and the hard-sphere colour pass over all replicas at once.
cudaError_t launch_rebuild_batch(int dim, const Batch& b, const Arrays& a, uint32_t n, bool write_s, cudaStream_t s);
cudaError_t launch_sweep_batch(int dim, bool fp32, const Batch& b, const Arrays& a, uint32_t color, uint32_t round,
                               uint32_t max_active, bool overlap_previous, bool early_wait, cudaStream_t s,
                               uint32_t variant = 0);
cudaError_t launch_overlap_batch(int dim, const Batch& b, const Arrays& a, uint32_t n, cudaStream_t s);
// Batches of Lennard-Jones replicas: one warp per trial over every replica's colour list (hmc_lj.cu).
cudaError_t launch_sweep_batch_lj(int dim, bool fp32, const Batch& b, const Arrays& a, uint32_t color, uint32_t round,
                                  uint32_t max_active, bool overlap_previous, bool early_wait, cudaStream_t s,
                                  uint32_t variant = 0);
// coop selects the warp-cooperative pass (the per-lane pass otherwise).
cudaError_t launch_sweep_sphere(int dim, bool fp32, const Geometry& g, const Arrays& a, const Pair& p,
                                const Launch& l, bool coop, cudaStream_t s, uint32_t variant = 0);
cudaError_t launch_overlap_sphere(int dim, const Geometry& g, const Arrays& a, const Pair& p, uint32_t n,
                                  cudaStream_t s);
// generic: the system's energy is not Shifted Lennard-Jones (the overlap penalty, Isotropic).
cudaError_t launch_sweep_lj(int dim, bool fp32, bool generic, const Geometry& g, const Arrays& a, const Pair& p,
                            const Launch& l,
                            cudaStream_t s, uint32_t variant = 0);
// The trial moves of round l.round for every colour list at once (Arrays::trial_*), one thread
// per trial; launched in stream order before the round's colour passes of the passes that give a
// trial several lanes (LJ and the overlap penalty, convex polyhedra, convex polygons).
cudaError_t launch_propose_lj(int dim, bool fp32, const Geometry& g, const Arrays& a, const Launch& l, cudaStream_t s);
// soft: the trial also draws the Metropolis uniform after the move (trial_t.w in 3-D, .z in 2-D).
cudaError_t launch_propose_poly(bool fp32, const Geometry& g, const Arrays& a, const Launch& l, bool rotate,
                                bool soft, cudaStream_t s);
cudaError_t launch_propose_poly2(bool fp32, const Geometry& g, const Arrays& a, const Launch& l, bool rotate,
                                 bool soft, cudaStream_t s);

// Anisotropic { ApproximateShapeOverlap { Convex(shape), OverlapPenalty, resolution }, r_cut }
// (hoomd-interaction/src/pairwise/anisotropic.rs:120-135, approximate_shape_overlap.rs:122-131):
// the insertion hamiltonian that place_single_site_orientable_bodies (benchmarks/src/place.rs:
// 120-219) prepares convex shapes with. A pair closer than r_cut costs OverlapPenalty(-d), d the
// distance (in steps of `resolution`) the other shape moves along the line of centres until the
// two no longer intersect (IntersectsAt::approximate_separation_distance, hoomd-geometry/src/
// lib.rs:307-325).
struct ShapeOverlap {
    double resolution;
    double rcut;      // Anisotropic::r_cut, compared with the centre distance
    double rr;        // (R + R)^2: the bounding-sphere test of Convex::intersects_at
    double dmax;      // OverlapPenalty::maximum_allowed_overlap
    double half_k;    // 0.5 * OverlapPenalty::k
    double shoulder;  // OverlapPenalty::epsilon_shoulder
    uint32_t max_steps;  // the separation loop ends within this many steps for every pair the host
                         // admits (|v| < r_cut); more sets kErrIterationCap
};
// ParallelSweep colour pass under ShapeOverlap, FP64, one warp per trial (trials from
// launch_propose_poly / launch_propose_poly2 with soft = true).
cudaError_t launch_sweep_poly3_soft(const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                                    const ShapeOverlap& so, const Launch& l, cudaStream_t s);
cudaError_t launch_sweep_poly2_soft(bool sat, const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                                    const ShapeOverlap& so, const Launch& l, cudaStream_t s);
// PairwiseCutoff::total_energy under ShapeOverlap (pairs i < j in body order, i's frame), summed
// into *out with atomics.
cudaError_t launch_energy_poly3_soft(const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                                     const ShapeOverlap& so, uint32_t n, double* out, cudaStream_t s);
cudaError_t launch_energy_poly2_soft(bool sat, const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                                     const ShapeOverlap& so, uint32_t n, double* out, cudaStream_t s);
// delta_energy_one in FP64 for injected trial positions (LJ); u < 0 means no decision needed.
cudaError_t launch_eval_lj(int dim, bool fp32, const Geometry& g, const Arrays& a, const Pair& p,
                           const uint64_t* bodies, const double4* trial, const double* u, double kt, uint32_t n,
                           uint8_t* decisions, uint8_t* rechecked, double* delta_h, cudaStream_t s);
cudaError_t launch_energy_lj(int dim, const Geometry& g, const Arrays& a, const Pair& p, uint32_t n, double* out,
                             cudaStream_t s);
cudaError_t launch_sweep_poly(bool fp32, const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                              double rcut2, float rcut2_hi32, const Launch& l, bool rotate, cudaStream_t s,
                              uint32_t variant = 0);
cudaError_t launch_eval_poly(bool fp32, const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                             double rcut2, float rcut2_hi32, const uint64_t* bodies, const double4* trial,
                             const double4* trial_q, uint32_t n, uint8_t* decisions, cudaStream_t s);
cudaError_t launch_overlap_poly(const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv, double rcut2,
                                uint32_t n, cudaStream_t s);
cudaError_t launch_tune_moves(int dim, const Geometry& g, const Arrays& a, const Launch& l, uint32_t tune_step,
                              uint32_t samples, bool rotate, uint64_t* bodies, double4* trial, double4* trial_q,
                              double* u, cudaStream_t s);
// Hard convex polygons (hmc_poly2.cu): XenoCollide (sat = false) or separating axes (sat =
// true); orientations are angles in .x of body_ori / sorted_q / trial_q.
cudaError_t launch_sweep_poly2(bool fp32, bool sat, const Geometry& g, const Arrays& a, const double4* verts,
                               uint32_t nv, double rcut2, float rcut2_hi32, const Launch& l, bool rotate,
                               cudaStream_t s);
cudaError_t launch_eval_poly2(bool fp32, bool sat, const Geometry& g, const Arrays& a, const double4* verts,
                              uint32_t nv, double rcut2, float rcut2_hi32, const uint64_t* bodies,
                              const double4* trial, const double4* trial_q, uint32_t n, uint8_t* decisions,
                              cudaStream_t s);
cudaError_t launch_overlap_poly2(bool sat, const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                                 double rcut2, uint32_t n, cudaStream_t s);
// The correctly rounded sin/cos of the rotation path over an array; *bad |= 1 when an
// argument is out of range.
cudaError_t launch_sincos(const double* x, uint64_t n, double* sn, double* cs, uint32_t* bad, cudaStream_t s);
// 2-D orientations through the staging array: check (finite, |theta| < 2^19; smallest bad
// index into first_bad), unpack into .x of body_ori, pack from it.
cudaError_t launch_check_angles(const double* packed, uint64_t n, unsigned long long* first_bad, cudaStream_t s);
cudaError_t launch_unpack_angles(const double* packed, double4* body_ori, uint64_t n, cudaStream_t s);
cudaError_t launch_pack_angles(const double4* body_ori, double* packed, uint64_t n, cudaStream_t s);
// Pair histograms over the current cell list (built with spaces at least `limit` wide, FP64 S):
// SDF (x = 1 - sigma/r in [0, limit)) or g(r) (r in [0, limit)), bins of 1/inv_width.
cudaError_t launch_pair_histogram(int dim, bool sdf, const Geometry& g, const Arrays& a, uint32_t n, double sigma,
                                  double limit, double inv_width, uint32_t n_bins, unsigned long long* counts,
                                  cudaStream_t s);
// Sweep::apply_with_filter for hard (soft = false) or overlap-penalty spheres (hmc_serial.cu):
// one warp, one sequential stream. nc/w: the serial grid (cells per axis, widths); mask (may be
// null): bodies to move.
cudaError_t launch_serial_sphere(int dim, bool soft, const Geometry& g, const Arrays& a, const Pair& p,
                                 const Launch& l, const uint32_t* nc, const double* w, uint32_t cap, uint32_t* size,
                                 uint32_t* items, uint32_t* cell_of, double4* site, const uint8_t* mask,
                                 cudaStream_t s);
// Sweep::apply_with_filter for hard convex polyhedra (hmc_poly.cu) and polygons (hmc_poly2.cu;
// sat: separating axes) on the serial grid, Translate or Rotate moves.
cudaError_t launch_serial_poly(const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv, double rcut2,
                               const Launch& l, bool rotate, const uint32_t* nc, const double* w, uint32_t cap,
                               uint32_t* size, uint32_t* items, uint32_t* cell_of, double4* site, const uint8_t* mask,
                               cudaStream_t s);
cudaError_t launch_serial_poly2(bool sat, const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                                double rcut2, const Launch& l, bool rotate, const uint32_t* nc, const double* w,
                                uint32_t cap, uint32_t* size, uint32_t* items, uint32_t* cell_of, double4* site,
                                const uint8_t* mask, cudaStream_t s);
// QuickInsert's insertion loop on the serial grid (one warp): bodies appended from index n0.
struct QuickInsertArgs {
    uint32_t n0;         // bodies before the call
    uint32_t capacity;   // bodies the arrays hold
    uint64_t attempts;   // draws at most (QuickInsert::target)
    uint64_t to_insert;  // target - inserted
    uint64_t allowed;    // allowed_overlaps
    double low[3];       // Uniform low per axis (-L/2)
    double scale[3];     // Uniform scale per axis
    uint32_t soft;       // 1: overlap penalty, 0: hard spheres
};
// Body tags: tag[capacity], a min-heap of free tags heap[capacity], meta = {heap size, tag bound};
// tag == null: tags are not tracked.
struct BodyTags {
    uint32_t* tag;
    uint32_t* heap;
    uint32_t* meta;
};
cudaError_t launch_quick_insert(int dim, const Geometry& g, const Arrays& a, const Pair& p, const Launch& l,
                                const QuickInsertArgs& q, const BodyTags& tags, const uint32_t* nc, const double* w,
                                uint32_t cap, uint32_t* size, uint32_t* items, uint32_t* cell_of, double4* site,
                                unsigned long long* out, cudaStream_t s);
// The same for oriented convex shapes under ShapeOverlap: each UniformIn body also draws a uniform
// random orientation (uniform_in.rs:158-176).
cudaError_t launch_quick_insert_poly3(const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                                      const ShapeOverlap& so, const Launch& l, const QuickInsertArgs& q,
                                      const BodyTags& tags, const uint32_t* nc, const double* w, uint32_t cap,
                                      uint32_t* size, uint32_t* items, uint32_t* cell_of, double4* site,
                                      unsigned long long* out, cudaStream_t s);
cudaError_t launch_quick_insert_poly2(bool sat, const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                                      const ShapeOverlap& so, const Launch& l, const QuickInsertArgs& q,
                                      const BodyTags& tags, const uint32_t* nc, const double* w, uint32_t cap,
                                      uint32_t* size, uint32_t* items, uint32_t* cell_of, double4* site,
                                      unsigned long long* out, cudaStream_t s);
// GrandCanonical::apply, n_trials in sequence on the serial grid (one warp).
struct GrandCanonicalArgs {
    uint64_t step;
    uint32_t substep;      // of the first trial; trial i uses substep + i
    uint32_t seed;
    uint32_t n_trials;
    uint32_t n0;
    uint32_t capacity;
    uint32_t soft;
    double temperature, fugacity, volume;
    double low[3], scale[3];  // UniformIn per axis
};
cudaError_t launch_grand_canonical(int dim, const Geometry& g, const Arrays& a, const Pair& p,
                                   const GrandCanonicalArgs& q, const BodyTags& tags, const uint32_t* nc,
                                   const double* w, uint32_t cap, uint32_t* size, uint32_t* items, uint32_t* cell_of,
                                   double4* site, unsigned long long* out, cudaStream_t s);
// Clone with boundary (hmc_set_box): every body x -> clamp(scale x, lo, hi) per axis, then
// B = wrap(.) in the new box; first_outside receives the smallest body index that is not
// inside the old box (the reference's map_point fails there).
cudaError_t launch_map_bodies(int dim, const Geometry& g_new, const double* old_half, const double* scale,
                              const double* lo, const double* hi, double4* body_pos, uint64_t n,
                              unsigned long long* first_outside, cudaStream_t s);
// State transfer through a packed staging array of n x dim doubles (the host layout):
// first_nonfinite receives the smallest body index with a non-finite coordinate (it must hold
// ~0 before the launch); unpack writes body positions, pack reads them.
cudaError_t launch_check_finite(const double* packed, uint64_t count, uint32_t dim,
                                unsigned long long* first_nonfinite, cudaStream_t s);
cudaError_t launch_unpack_positions(int dim, const double* packed, double4* body_pos, uint64_t n, cudaStream_t s);
cudaError_t launch_pack_positions(int dim, const double4* body_pos, double* packed, uint64_t n, cudaStream_t s);
// GSD frame encoding: FP32 site positions (n x 3) and, for ori_kind 1 (versors, 3-D) or 2
// (angles, 2-D), FP32 site versors (n x 4), in body order.
cudaError_t launch_gsd_encode(int dim, int ori_kind, const Geometry& g, const double4* body_pos,
                              const double4* body_ori, uint64_t n, float* pos, float* ori, cudaStream_t s);
// Injected trials through the colour-pass kernels themselves (the probe mode, Injected): the
// hard-sphere passes (FP32: the per-lane pass, FP64: the warp-cooperative pass, or the one
// `coop` names), the Lennard-Jones and overlap-penalty passes, the packed polyhedron pass.
cudaError_t launch_trials_sphere(int dim, bool fp32, bool coop, const Geometry& g, const Arrays& a, const Pair& p,
                                 const Injected& j, cudaStream_t s);
cudaError_t launch_trials_lj(int dim, bool fp32, const Geometry& g, const Arrays& a, const Pair& p, double kt,
                             const Injected& j, cudaStream_t s);
cudaError_t launch_trials_poly(bool fp32, const Geometry& g, const Arrays& a, const double4* verts, uint32_t nv,
                               double rcut2, float rcut2_hi32, const Injected& j, cudaStream_t s);
// The sequential-stream tuner (TuneJob), one warp per job (jobs in device memory): hard spheres,
// Lennard-Jones / overlap penalty, convex polyhedra, convex polygons (sat: separating axes).
cudaError_t launch_tune_stream_sphere(int dim, TuneJob* jobs, uint32_t n_jobs, cudaStream_t s);
cudaError_t launch_tune_stream_lj(int dim, TuneJob* jobs, uint32_t n_jobs, cudaStream_t s);
cudaError_t launch_tune_stream_poly(TuneJob* jobs, uint32_t n_jobs, const double4* verts, uint32_t nv, double rcut2,
                                    cudaStream_t s);
cudaError_t launch_tune_stream_poly2(bool sat, TuneJob* jobs, uint32_t n_jobs, const double4* verts, uint32_t nv,
                                     double rcut2, cudaStream_t s);
// Sampler probe (hmc_sample_moves): n proposals from Counter(step, substep, seed).index(i) for a
// body at the origin, identity orientation; zig: the context's tables (x then f).
cudaError_t launch_sample_moves(int dim, uint32_t kind, double maximum, uint64_t step, uint32_t substep,
                                uint32_t seed, uint64_t n, const double* zig, double* out, cudaStream_t s);
// Injected moves: positions (n x 4 doubles), result decisions and recheck flags.
cudaError_t launch_eval_sphere(int dim, bool fp32, const Geometry& g, const Arrays& a, const Pair& p,
                               const uint64_t* bodies, const double4* trial, uint32_t n, uint8_t* decisions,
                               uint8_t* rechecked, cudaStream_t s);

}  // namespace hmc
