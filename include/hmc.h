/*
 * hmc.h -- C ABI of the B200 (sm_100a) Monte Carlo sweep library, libhmc_b200.so.
 *
 * The library runs the local-move Metropolis sweep of hoomd-rs's hoomd-mc crate
 * (glotzerlab/hoomd-rs v1.4.0) on one GPU. The reference has no FFI; these entry points
 * are the ones a Rust `GpuSweep` type would bind to replace the monomorphised generic
 * calls on the sweep path (citations are file:line in the reference):
 *
 *   hmc_system_create / hmc_set_state / hmc_get_state
 *       replace building a Microstate<B,S,VecCell,Periodic<Hypercuboid>> with
 *       Microstate::builder()...try_build() / add_body (hoomd-microstate/src/microstate.rs:777-835)
 *       and reading microstate.bodies() back. step/substep/seed are the Counter fields
 *       (microstate.rs:529).
 *   hmc_sweep
 *       replaces Trial::apply (hoomd-mc/src/lib.rs:134-147) as implemented by
 *       ParallelSweep::apply (hoomd-mc/src/parallel_sweep.rs:390-421), with the trial moves
 *       Translate<Cartesian<N>> (translate/cartesian.rs:40-51), Rotate<Versor>
 *       (rotate/versor.rs:112-123), the Hamiltonian PairwiseCutoff::delta_energy_one
 *       (hoomd-interaction/src/pairwise_cutoff.rs:919-941) over HardSphere, HardShape<Convex<
 *       ConvexPolyhedron>> or Isotropic<Shifted<LennardJones>>, and the Isothermal macrostate.
 *       Returns the Count (hoomd-mc/src/lib.rs:206-294).
 *   hmc_tune
 *       replaces Tune::tune_with_options (hoomd-mc/src/lib.rs:430-449, tune_local.rs:21-89).
 *   hmc_overlap_check
 *       replaces PairwiseCutoff::total_energy (pairwise_cutoff.rs:720-745) as an overlap check.
 *   hmc_eval_moves
 *       evaluates injected trial moves against the current state: delta_energy_one plus the
 *       Metropolis test of sweep.rs:207-208. It is the decision-parity probe.
 *
 * Conventions. Every call returns hmc_status; no call aborts. On failure,
 * hmc_last_error_message() gives a thread-local description. Host arrays are owned by the
 * caller and copied; no pointer is retained across calls. One hmc_system is driven by one
 * host thread at a time. All device work of a system runs on one CUDA stream.
 */
#ifndef HMC_H
#define HMC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HMC_ABI_VERSION 3u  /* 2: hmc_count gained order_ambiguous; 3: HMC_ISOTROPIC and its
                               hmc_system_desc fields, hmc_set_shape_overlap */

typedef enum hmc_status {
    HMC_OK = 0,
    HMC_INVALID_ARGUMENT = 1,     /* bad sizes, NULL pointers, non-positive lengths */
    HMC_RANGE_TOO_LARGE = 2,      /* interaction range leaves < 2 checkerboard spaces per axis
                                     (hypercuboid.rs:196-199 panics) or exceeds L/2
                                     (boundary/periodic.rs:97-107) */
    HMC_OVERLAP_IN_INPUT = 3,     /* reserved: reported by hmc_overlap_check callers */
    HMC_CELL_OVERFLOW = 4,        /* a cell holds more bodies than a kernel supports */
    HMC_NAN_STATE = 5,            /* a non-finite coordinate was found */
    HMC_ITERATION_CAP = 6,        /* a bounded device loop reached its bound (an approximate
                                     separation, hmc_set_shape_overlap) */
    HMC_TIMEOUT = 7,              /* reserved */
    HMC_CUDA_ERROR = 8,           /* a CUDA runtime call failed */
    HMC_OUT_OF_MEMORY = 9,
    HMC_NOT_SUPPORTED = 10,       /* combination not implemented */
    HMC_OUTSIDE_CHECKERBOARD = 11, /* a body maps to no space (parallel_sweep.rs:198 panics) */
    HMC_IO_ERROR = 12              /* a GSD file could not be read or written, or is corrupt */
} hmc_status;

typedef enum hmc_interaction {
    HMC_HARD_SPHERE = 0,            /* PairwiseCutoff(HardSphere { diameter }) */
    HMC_HARD_CONVEX_POLYGON = 1,    /* PairwiseCutoff(HardShape(Convex(ConvexPolygon))) */
    HMC_HARD_CONVEX_POLYHEDRON = 2, /* PairwiseCutoff(HardShape(Convex(ConvexPolyhedron))) */
    HMC_LENNARD_JONES = 3,          /* PairwiseCutoff(Isotropic { Shifted { LennardJones }, r_cut }) */
    HMC_HARD_CONVEX_SURFACE_MESH_2D = 4, /* PairwiseCutoff(HardShape(ConvexSurfaceMesh2d)): vertices are
                                           the counter-clockwise hull (convex_surface_mesh_2d.rs) */
    HMC_OVERLAP_PENALTY = 5,        /* PairwiseCutoff(Isotropic { Expanded { delta: diameter,
                                       OverlapPenalty { k, maximum_allowed_overlap, epsilon_shoulder } },
                                       r_cut: diameter }): the soft sphere that QuickInsert and
                                       QuickCompress use (univariate/overlap_penalty.rs:42-116,
                                       expanded.rs:62-67, benchmarks/src/mc/hard_sphere.rs:191-199) */
    HMC_ISOTROPIC = 6               /* PairwiseCutoff(Isotropic { W(F), r_cut }) for a univariate F
                                       (hmc_system_desc.univariate, hmc_univariate) in a wrapper W
                                       (univariate_wrap, hmc_univariate_wrap), isotropic.rs:88-187;
                                       FP64 in both precision modes */
} hmc_interaction;

/* The univariate energies of HMC_ISOTROPIC (hoomd-interaction/src/univariate/), with their
 * parameters in hmc_system_desc.univariate_params in this order. */
typedef enum hmc_univariate {
    HMC_UV_LENNARD_JONES = 0,          /* {epsilon, sigma}: LennardJones<12, 6> */
    HMC_UV_WEEKS_CHANDLER_ANDERSON = 1, /* {epsilon, sigma} */
    HMC_UV_HARMONIC = 2,               /* {k, r_0} */
    HMC_UV_HARMONIC_REPULSION = 3,     /* {a, r_cut} */
    HMC_UV_BOXCAR = 4,                 /* {epsilon, left, right} */
    HMC_UV_OVERLAP_PENALTY = 5,        /* {k, maximum_allowed_overlap, epsilon_shoulder} */
    HMC_UV_LENNARD_JONES_GAUSS = 6     /* {epsilon, sigma_squared, r_0, scale}: exp is the device's, within
                                          a few ulp of the platform's, and the order bound covers it */
} hmc_univariate;
/* The wrapper around the univariate, with its parameters in hmc_system_desc.wrap_params. */
typedef enum hmc_univariate_wrap {
    HMC_UVW_NONE = 0,
    HMC_UVW_SHIFTED = 1,  /* {r_shift}: Shifted, F(r) - F(r_shift) */
    HMC_UVW_EXPANDED = 2, /* {delta}: Expanded, F(r - delta) */
    HMC_UVW_XPLOR = 3     /* {r_cut, r_smooth}: Xplor, s(r) F(r) */
} hmc_univariate_wrap;

typedef enum hmc_move {
    HMC_TRANSLATE = 0, /* Translate::with_maximum_distance(maximum) */
    HMC_ROTATE = 1     /* Rotate::with_maximum_rotation(maximum) */
} hmc_move;

typedef enum hmc_precision {
    HMC_FP64 = 0,        /* every pair test in FP64, the reference's arithmetic */
    HMC_FP32_RECHECK = 1 /* FP32 pair tests under a forward-error bound; pairs inside the
                            bound are re-evaluated in FP64, so decisions equal HMC_FP64 */
} hmc_precision;

typedef struct hmc_context hmc_context;
typedef struct hmc_system hmc_system;
typedef struct hmc_batch hmc_batch;

typedef struct hmc_device_opts {
    uint32_t struct_size; /* sizeof(hmc_device_opts) */
    int32_t device;       /* CUDA device ordinal */
} hmc_device_opts;

typedef struct hmc_system_desc {
    uint32_t struct_size;        /* sizeof(hmc_system_desc) */
    uint32_t dim;                /* 2 or 3 */
    double edge_lengths[3];      /* periodic box, centred on the origin: [-L/2, L/2) */
    uint64_t n_bodies;
    uint64_t step;               /* Counter step */
    uint32_t substep;            /* Counter substep */
    uint32_t seed;               /* Counter seed */
    uint32_t interaction;        /* hmc_interaction */
    uint32_t n_vertices;         /* convex polytope vertex count (<= 32; polygons >= 3) */
    const double* vertices;      /* n_vertices * dim, FP64 */
    double diameter;             /* HardSphere */
    double lj_epsilon, lj_sigma, lj_r_cut, lj_r_shift; /* Isotropic<Shifted<LennardJones>> */
    double boundary_range;       /* Periodic::new maximum_interaction_range; 0 = the pair range */
    double body_interaction_range; /* ParallelSweep::new range; 0 = the pair range */
    double penalty_k;            /* OverlapPenalty::k (default 10000) */
    double penalty_maximum_overlap; /* OverlapPenalty::maximum_allowed_overlap (default 0.2) */
    double penalty_shoulder;     /* OverlapPenalty::epsilon_shoulder (default 100) */
    uint64_t capacity;           /* bodies the system can hold (>= n_bodies; 0 = n_bodies);
                                    hmc_quick_insert_apply adds bodies up to it */
    uint32_t univariate;         /* HMC_ISOTROPIC: hmc_univariate */
    uint32_t univariate_wrap;    /* HMC_ISOTROPIC: hmc_univariate_wrap */
    double univariate_params[4]; /* HMC_ISOTROPIC: the univariate's parameters */
    double wrap_params[2];       /* HMC_ISOTROPIC: the wrapper's parameters */
    double isotropic_r_cut;      /* HMC_ISOTROPIC: Isotropic::r_cut (the pair range) */
} hmc_system_desc;

typedef struct hmc_sweep_params {
    uint32_t struct_size;     /* sizeof(hmc_sweep_params) */
    uint32_t move;            /* hmc_move */
    double maximum;           /* maximum distance (translate) or rotation (rotate) */
    double temperature;       /* Isothermal kT */
    uint32_t precision;       /* hmc_precision */
    uint32_t n_sweeps;        /* number of ParallelSweep::apply calls */
    uint32_t increment_step;  /* 1: Microstate::increment_step() after every apply */
    uint32_t flags;           /* hmc_tune / hmc_batch_tune: HMC_TUNE_* bits; 0 otherwise */
} hmc_sweep_params;

/* hmc_sweep_params.flags for hmc_tune and hmc_batch_tune. By default the tuner is
 * tune_local_trial as the reference runs it (hoomd-mc/src/tune_local.rs:42-88): every sample of
 * every round from the one stream Counter(step, substep, seed).make_rng(), in order, on one warp
 * (one warp per replica for a batch), so the tuned maximum equals the reference's for the same
 * state. HMC_TUNE_PER_SAMPLE_STREAMS instead gives sample j of round t its own stream
 * Counter(step, substep, seed).index(2^63 | t << 32 | j) and evaluates a round's samples in
 * parallel: the same distribution, much faster, but not the reference's numbers. */
#define HMC_TUNE_PER_SAMPLE_STREAMS 1u

typedef struct hmc_count {
    uint64_t accepted;
    uint64_t rejected;
    uint64_t rechecks;       /* FP32 pair results re-evaluated in FP64 */
    uint64_t pair_checks;    /* pair evaluations in the FP32 path */
    double max_fp32_error;   /* largest |FP32 - FP64| over rechecked pair quantities */
    uint64_t order_ambiguous; /* Lennard-Jones and overlap-penalty trials whose FP64 dU lies so close
                                 to the Metropolis threshold that summing the same pair energies in
                                 another order (the reference's cell-list order) could change the
                                 decision; 0 proves every decision equal to any order's */
} hmc_count;

/* One injected trial move for hmc_eval_moves. */
typedef struct hmc_injected_move {
    uint64_t body;           /* body index */
    double position[3];      /* trial body position as returned by wrap(propose(..)) */
    double orientation[4];   /* trial versor (s, x, y, z) or angle in [0] */
    double u;                /* the Metropolis uniform in [0, 1); ignored for hard shapes */
} hmc_injected_move;

/* 2-D orientations are angles (Angle, hoomd-vector angle.rs) with |theta| < 2^19; the
 * rotation path turns them into matrices with correctly rounded sin and cos. */

/* Device-time profile of a system's kernels, collected with CUDA events on the system's
 * stream while profiling is enabled. */
typedef struct hmc_profile {
    uint64_t kernel_launches;       /* every kernel this system enqueued (profiling on or off) */
    uint64_t sweep_launches;        /* colour-pass sweep kernels timed */
    double sweep_ms;                /* device time of the timed colour-pass kernels */
    uint64_t rebuild_launches;      /* cell-list kernels timed */
    double rebuild_ms;              /* device time of the timed cell-list rebuilds */
    uint64_t sweeps;                /* ParallelSweep::apply calls timed */
} hmc_profile;

/* ---- context and errors ---- */
uint32_t hmc_abi_version(void);
const char* hmc_status_string(hmc_status status);
const char* hmc_last_error_message(void);
hmc_status hmc_context_create(const hmc_device_opts* opts, hmc_context** out);
void hmc_context_destroy(hmc_context* ctx);

/* ---- systems ---- */
hmc_status hmc_system_create(hmc_context* ctx, const hmc_system_desc* desc, const double* positions,
                             const double* orientations, hmc_system** out);
void hmc_system_destroy(hmc_system* sys);
/* Run the system's device work on an external cudaStream_t (NULL: the library's own). */
hmc_status hmc_system_set_stream(hmc_system* sys, void* cuda_stream);
void* hmc_system_stream(hmc_system* sys);
/* positions: n*dim; orientations: n*4 (3-D) or n (2-D) or NULL for unoriented bodies.
 * Each host array moves with one copy (direct DMA from pinned buffers); both calls return
 * after their copies complete. set_state returns HMC_NAN_STATE, leaving the device state
 * unchanged, when a coordinate is not finite. */
hmc_status hmc_set_state(hmc_system* sys, const double* positions, const double* orientations, uint64_t step,
                         uint32_t substep);
hmc_status hmc_get_state(hmc_system* sys, double* positions, double* orientations, uint64_t* step,
                         uint32_t* substep);
/* Microstate::increment_step (hoomd-microstate/src/microstate.rs:412-415): step += 1, substep = 0. */
hmc_status hmc_increment_step(hmc_system* sys);

/* ---- the sweep ----
 * n_sweeps ParallelSweep::apply calls; out receives their summed Count. With n_sweeps > 1 and
 * increment_step (and profiling off) the sweeps are enqueued back to back and the host waits
 * once per 64 sweeps rather than once per sweep; a sweep that needs more colour sets than were
 * enqueued stops the ones after it on the device, is completed, and they are enqueued again, so
 * the trajectory, Count and Counter are those of one call per sweep. On an error the sweeps
 * before the failing one stay applied and counted in the system's Counter; out is not written. */
hmc_status hmc_sweep(hmc_system* sys, const hmc_sweep_params* params, hmc_count* out);
hmc_status hmc_tune(hmc_system* sys, hmc_sweep_params* params, double target_acceptance, uint32_t samples,
                    uint32_t steps);
/* Sweep::apply_with_filter (hoomd-mc/src/sweep.rs:159-224), every interaction (hard and
 * overlap-penalty spheres, Lennard-Jones, convex polyhedra and polygons; Translate, or Rotate for
 * shapes): one trial per body in index order from one sequential stream, then increment_substep.
 * move_mask (n_bodies bytes, may be NULL) selects the bodies to move (should_move_body). The exact
 * serial chain on one warp; the checkerboard hmc_sweep is the fast path. For soft potentials
 * out->order_ambiguous counts the decisions another summation order could change. */
hmc_status hmc_serial_sweep(hmc_system* sys, const hmc_sweep_params* params, const uint8_t* move_mask,
                            hmc_count* out);
hmc_status hmc_overlap_check(hmc_system* sys, uint64_t* n_overlaps);
/* decisions[i] = 1 when move i would be accepted; rechecked[i] = 1 when the FP32 path had to
 * fall back to FP64 for it; delta_h[i] (may be NULL) = delta_energy_one in FP64. */
hmc_status hmc_eval_moves(hmc_system* sys, const hmc_injected_move* moves, uint64_t n, double temperature,
                          uint32_t precision, uint8_t* decisions, uint8_t* rechecked, double* delta_h);
/* The colour pass's own decision for injected trial moves: the kernel that hmc_sweep runs for
 * the system's interaction and `precision` (hard spheres: the per-lane FP32 pass or the
 * warp-cooperative FP64 pass; Lennard-Jones and the overlap penalty: the warp-per-trial passes;
 * convex polyhedra: the packed pass) takes each move in place of a drawn trial
 * (generate_trial_moves, parallel_sweep.rs:231-278) and writes its decision instead of
 * committing it; the state does not change. The checkerboard is the one the next hmc_sweep lays
 * out (update_checkerboard, parallel_sweep.rs:176-201: origin from the system's counter).
 * decisions[i] = 1 when the pass accepts move i. flags[i] (may be NULL): bit 0 = the FP32 pass
 * settled the move with FP64 pair evaluations; bit 1 = the move's position lies outside its
 * body's checkerboard space, which the colour pass rejects before any pair test
 * (parallel_sweep.rs:253-258). Lennard-Jones and penalty moves with bit 1 are not evaluated
 * (decision 0); for hard shapes the decision is still the pair walk's around the position's own
 * space. Convex polygons: HMC_NOT_SUPPORTED. */
hmc_status hmc_eval_trials(hmc_system* sys, const hmc_injected_move* moves, uint64_t n, double temperature,
                           uint32_t precision, uint8_t* decisions, uint8_t* flags);
/* PairwiseCutoff::total_energy (pairwise_cutoff.rs:720-745): the pair energy sum in FP64 for
 * Lennard-Jones and the overlap penalty (summed with atomics: the last bits depend on the
 * order); +infinity or 0 for hard shapes (any overlap / none). */
hmc_status hmc_total_energy(hmc_system* sys, double* energy);

/* ---- launch variants and the autotuner (no counterpart in the reference) ----
 * Every colour-pass kernel is compiled in a few launch shapes: the resident blocks per SM it
 * is built for (its register cap), the trials a warp takes (convex polyhedra: 4, 2 or 8) and,
 * for the warp-cooperative FP64 sphere pass, the candidates per stencil row a lane tests before
 * handing the rest to its warp; for convex polygons in HMC_FP32_RECHECK, variant 1 runs the FP64
 * pass instead of the FP32 prefilter. All take the same decisions, so the trajectory is the same
 * in every variant; only the speed differs, by shape and density. hmc_autotune times `sweeps`
 * sweeps of the system in every variant of its pass (precision and move from params), each from
 * the same saved state, keeps the fastest for this system and records it for every system and
 * batch of the process with the same pass, dimension, precision and density band (bodies per
 * checkerboard space, in quarter octaves); the state and counter are restored afterwards. A
 * system without its own choice uses the recorded one for its band, else variant 0. */
typedef struct hmc_launch_variant {
    uint32_t index;            /* in the variant table of the system's pass for this precision */
    uint32_t count;            /* variants in that table */
    uint32_t blocks_per_sm;    /* resident blocks per SM the kernel is compiled for */
    uint32_t trials_per_warp;  /* trials one warp takes at once (1: a lane or a warp per trial) */
    uint32_t own_steps;        /* warp-cooperative sphere pass: candidates per row a lane tests;
                                  Lennard-Jones / Isotropic passes: 2 = two candidates per lane
                                  and step */
} hmc_launch_variant;
/* index UINT32_MAX: the variant the next hmc_sweep in this precision runs. */
hmc_status hmc_get_launch_variant(hmc_system* sys, uint32_t precision, uint32_t index, hmc_launch_variant* out);
/* index UINT32_MAX: drop the system's own choice (the recorded one for its band, else 0). */
hmc_status hmc_set_launch_variant(hmc_system* sys, uint32_t precision, uint32_t index);
/* Hard spheres and disks: which colour pass a precision runs, one lane per trial (cooperative = 0,
 * the FP32 default) or the warp-cooperative pass (1, the FP64 default). Both make the same pair
 * tests, so the trajectory does not depend on the choice; the launch variants are those of the
 * chosen pass. A system without its own choice runs the one hmc_autotune recorded for its
 * dimension, precision and density band, else the default. HMC_NOT_SUPPORTED for other
 * interactions. */
hmc_status hmc_set_cooperative_pass(hmc_system* sys, uint32_t precision, uint32_t cooperative);
hmc_status hmc_get_cooperative_pass(hmc_system* sys, uint32_t precision, uint32_t* cooperative);
/* Hard spheres and disks without a pass set by hmc_set_cooperative_pass: hmc_autotune times the
 * variants of both passes and keeps the fastest pass and variant (and records both).
 * ms_per_sweep (may be NULL): chosen->count entries, the mean time of one sweep per variant of
 * the chosen pass. */
hmc_status hmc_autotune(hmc_system* sys, const hmc_sweep_params* params, uint32_t sweeps, hmc_launch_variant* chosen,
                        double* ms_per_sweep);
/* The same for a batch's replica pass (params: one per replica, as hmc_batch_sweep). */
hmc_status hmc_batch_autotune(hmc_batch* batch, const hmc_sweep_params* params, uint32_t sweeps,
                              hmc_launch_variant* chosen, double* ms_per_sweep);
hmc_status hmc_batch_set_launch_variant(hmc_batch* batch, uint32_t precision, uint32_t index);

/* ---- overlap count into caller buffers, with no device allocation ----
 * No counterpart in the reference (hoomd-rs has no GPU path); it serves callers that must
 * not call cudaMalloc when they run the check, for example a framework that hands out all
 * device memory from its own pre-reserved pool, or a plugin that may not grow the
 * process's device footprint after start-up. It counts the pairs (i < j) of hard spheres
 * of the given diameter whose sites overlap through any periodic image, with the same
 * arithmetic as hmc_overlap_check, and needs no hmc_context or hmc_system.
 *
 *   positions      device pointer, n_bodies * dim FP64 body positions (as hmc_get_state
 *                  returns them; sites are wrap(position))
 *   edge_lengths   host pointer, dim FP64 box edge lengths
 *   boundary_range Periodic::new maximum_interaction_range; 0 = diameter
 *   overlaps       device pointer to one uint64_t; set to the count
 *   cuda_stream    cudaStream_t (NULL: the default stream); runs on the current device
 *
 * Its cell list lives in a fixed device array inside the library (about 3.4 MB, held on
 * every GPU that loads the library until the process exits), so n_bodies is limited to
 * HMC_NOALLOC_MAX_BODIES (HMC_INVALID_ARGUMENT beyond). The first call on a device looks
 * up that array's device address (cudaGetSymbolAddress) with the device current; make it
 * before capturing any stream into a CUDA graph. CUDA loads device code lazily by default
 * (unless CUDA_MODULE_LOADING=EAGER), so that first call is also what creates the array on
 * the device: the footprint grows once, then never again. A caller that must not grow it
 * later makes one call at start-up (n_bodies = 0 is enough). The address is looked up again
 * when the device's context changes (after cudaDeviceReset). All calls share the array:
 * calls that overlap in time on the GPU (two streams, two threads) race with each other and
 * give wrong counts, so serialise them. Errors are reported by status only. */
#define HMC_NOALLOC_MAX_BODIES 65536u
#define HMC_NOALLOC_MAX_CELLS 65536u
hmc_status hmc_overlap_count_noalloc(const double* positions, uint64_t n_bodies, uint32_t dim,
                                     const double* edge_lengths, double diameter, double boundary_range,
                                     uint64_t* overlaps, void* cuda_stream);

/* ---- profiling ---- */
/* ---- equilibrium estimators (no counterpart in the reference) ----
 * Histograms of the pairs i < j by minimum-image distance r (FP64, per axis
 * d = t - s - L rint((t - s)/L)). hmc_sdf: hard spheres; bins of x = 1 - sigma/r over
 * [0, x_max), the scale distribution function: with s(x) = counts / (N dx), the pressure is
 * beta P / rho = 1 + s(0+) / dim. hmc_gr: bins of r over [0, r_max) (r_max < L/2); normalise by
 * the ideal-gas pair count. Both rebuild the cell list with wider spaces; the state and its
 * counter are not changed. */
hmc_status hmc_sdf(hmc_system* sys, double x_max, uint32_t n_bins, uint64_t* counts);
hmc_status hmc_gr(hmc_system* sys, double r_max, uint32_t n_bins, uint64_t* counts);

/* ---- batches of independent replicas ----
 * A batch runs many boxes (each its own hmc_system_desc: box, pair parameters, Counter, body
 * count) through one set of launches: one counting sort and one kernel per colour pass for all
 * replicas. Every replica's trajectory is the one hmc_system would produce from the same
 * description. The reference has no counterpart (a user would loop over Microstates, each
 * with its own ParallelSweep::apply, hoomd-mc/src/parallel_sweep.rs:390-421). */
/* positions[k]: descs[k].n_bodies * dim doubles. All replicas share dim and the interaction:
 * HMC_HARD_SPHERE, or HMC_LENNARD_JONES (each replica with its own epsilon, sigma, r_cut,
 * r_shift). */
hmc_status hmc_batch_create(hmc_context* ctx, uint32_t n_replicas, const hmc_system_desc* descs,
                            const double* const* positions, hmc_batch** out);
void hmc_batch_destroy(hmc_batch* batch);
/* params: one per replica (its own maximum and temperature, the kT of a Lennard-Jones replica);
 * move (HMC_TRANSLATE), precision, n_sweeps, increment_step must agree. counts (per replica,
 * may be NULL) receive accepted/rejected; total (may be NULL) also receives the batch's
 * rechecks, pair_checks and max_fp32_error. */
hmc_status hmc_batch_sweep(hmc_batch* batch, const hmc_sweep_params* params, hmc_count* counts, hmc_count* total);
/* enable = 1: hmc_batch_sweep runs each sweep as one launch of a CUDA graph (built on first use
 * for the precision, launch variant and increment_step, rebuilt when they change): the origins of
 * the replicas' checkerboards, the rebuild, the rounds (a while node over the colour sets) and the
 * per-replica counts and Counters all stay on the device, so the n_sweeps sweeps of one call are
 * launched back to back and the host waits once, at the end. Decisions, counts and Counters are
 * the launched sweep's (enable = 0, the default). A sweep whose rebuild flags an error runs no
 * colour pass, nor do the later sweeps of the call; the call then returns the error. */
hmc_status hmc_batch_set_captured_sweeps(hmc_batch* batch, uint32_t enable);
hmc_status hmc_batch_get_state(hmc_batch* batch, uint32_t replica, double* positions, uint64_t* step,
                               uint32_t* substep);
hmc_status hmc_batch_set_state(hmc_batch* batch, uint32_t replica, const double* positions, uint64_t step,
                               uint32_t substep);
/* Overlapping pairs per replica (n_overlaps: n_replicas entries); hard spheres only
 * (HMC_NOT_SUPPORTED for a Lennard-Jones batch). */
hmc_status hmc_batch_overlap_check(hmc_batch* batch, uint64_t* n_overlaps);
/* Tune::tune_with_options for every replica (hmc_tune on each replica's own state): params[k]
 * holds replica k's start maximum, temperature and precision and receives its tuned maximum,
 * equal to hmc_tune's on the same state (hoomd-mc/src/tune_local.rs:21-89). Translation only. */
hmc_status hmc_batch_tune(hmc_batch* batch, hmc_sweep_params* params, double target_acceptance, uint32_t samples,
                          uint32_t steps);
/* The scale distribution of every replica (hmc_sdf's pair counts by x = 1 - sigma/r over
 * [0, x_max)): counts receives n_replicas * n_bins entries, replica by replica. Hard spheres
 * only. The SDF pressure estimator is new (the reference has no counterpart). */
hmc_status hmc_batch_sdf(hmc_batch* batch, double x_max, uint32_t n_bins, uint64_t* counts);
/* Kernels this batch enqueued so far. */
uint64_t hmc_batch_kernel_launches(hmc_batch* batch);

/* The correctly rounded sin and cos that the 2-D rotation path uses (on the context's device);
 * no counterpart in the reference, which calls the platform libm (hoomd-vector angle.rs:120-150).
 * HMC_INVALID_ARGUMENT when some |x[i]| >= 2^20. */
hmc_status hmc_math_sincos(hmc_context* ctx, const double* x, uint64_t n, double* sin_out, double* cos_out);

/* The trial-move samplers on the device, as a probe (no counterpart in the reference, which tests
 * its samplers statistically: translate/cartesian.rs:65-100, rotate/versor.rs:151-184,
 * rotate/angle.rs:83-119). Sample i is drawn from Counter(step, substep, seed).index(i) for a
 * body at the origin with the identity orientation: kind 0 = Translate<Cartesian<dim>> with
 * maximum distance `maximum` (out: dim doubles, the displacement); kind 1 = Rotate with maximum
 * rotation `maximum` (3-D: the proposed versor, 4 doubles s, x, y, z; 2-D: the angle, 1 double);
 * kind 2 = one StandardNormal draw (1 double; `maximum` ignored). */
hmc_status hmc_sample_moves(hmc_context* ctx, uint32_t dim, uint32_t kind, double maximum, uint64_t step,
                            uint32_t substep, uint32_t seed, uint64_t n, double* out);

hmc_status hmc_profile_enable(hmc_system* sys, int enable);
hmc_status hmc_profile_read(hmc_system* sys, hmc_profile* out, int reset);

/* ---- preparing states: QuickInsert and QuickCompress (hoomd-mc) ----
 * Both hold their progress in a caller-owned struct, as the reference's QuickInsert and
 * QuickCompress values do; the microstate is the system's device state. Hard spheres and
 * HMC_OVERLAP_PENALTY spheres (the interaction the reference pairs them with).
 *
 * QuickInsert::apply (quick_insert.rs:228-280): when the total energy is <= 0 and bodies remain,
 * up to `target` bodies are drawn from UniformIn over the box (one Uniform(-L/2, L/2) per axis,
 * uniform_in.rs:112-130, cuboid.rs:568-596) from one stream Counter(step, substep, seed), each
 * kept when its insertion energy (delta_energy_insert, pairwise_cutoff.rs:1000-1009) is finite;
 * the call stops after `allowed_overlaps` kept bodies that overlap (energy > 0) or when all are
 * in, and increments the substep. It completes (complete = 1, no substep) once every body is in
 * and the energy is <= 0. Bodies are appended in order (new tags); the system must have the
 * capacity. The insertions are sequential by definition: one warp runs them on the device. */
typedef struct hmc_quick_insert {
    uint64_t target;           /* bodies to insert */
    uint64_t allowed_overlaps; /* QuickInsert::new: max(target / 8, 1) */
    uint64_t inserted;         /* bodies inserted so far */
    uint32_t complete;
    uint32_t reserved;
} hmc_quick_insert;
hmc_status hmc_quick_insert_apply(hmc_system* sys, hmc_quick_insert* qi, hmc_count* out);

/* QuickCompress::apply (quick_compress.rs:298-383): a state machine over Startup, Waiting,
 * Compressing and Complete. Compressing draws delta ~ Uniform(0, maximum_delta) from
 * Counter(step, substep, seed), scales the volume by (1 -/+ delta) towards the target (not
 * past it), maps every body into the scaled box (Hypercuboid::map_point, cuboid.rs:553-565,
 * then update_body_properties) and keeps the result when the total energy rose by at most
 * maximum_energy_per_site per site. Waiting moves on once the energy is <= 0. Every call
 * increments the substep. */
typedef enum hmc_quick_compress_state {
    HMC_QC_STARTUP = 0,
    HMC_QC_WAITING = 1,
    HMC_QC_COMPRESSING = 2,
    HMC_QC_COMPLETE = 3
} hmc_quick_compress_state;
typedef struct hmc_quick_compress {
    double target_volume;
    double maximum_energy_per_site; /* default 1000 */
    double maximum_delta;           /* default 0.05, in (0, 1) */
    uint32_t state;                 /* hmc_quick_compress_state */
    uint32_t is_final;              /* Waiting: the last accepted box had the target volume */
    double boundary[3];             /* Waiting / Complete: the box edge lengths they refer to */
} hmc_quick_compress;
hmc_status hmc_quick_compress_apply(hmc_system* sys, hmc_quick_compress* qc);

/* GrandCanonical::apply (grand_canonical.rs:49-110), n_trials times in sequence (each a full
 * apply that increments the substep): a fair coin picks an insertion of a UniformIn body,
 * accepted when V f exp(-dU/kT) / (N + 1) > u, or a removal of a uniformly chosen body, accepted
 * when N exp(-dU/kT) / (V f) > u (always when f <= 0); nothing happens when N = 0 and f <= 0.
 * dU is delta_energy_insert / delta_energy_remove (pairwise_cutoff.rs:1000-1031). Removal is
 * swap_remove: the last body takes the removed index, and freed tags are reused smallest
 * first, so GSD frames (tag order) follow the reference. Hard and overlap-penalty spheres. */
typedef struct hmc_grand_canonical_params {
    double temperature;   /* IsothermalIsofugacity temperature (> 0) */
    double fugacity;
    uint32_t n_trials;
    uint32_t reserved;
} hmc_grand_canonical_params;
typedef struct hmc_insert_remove_count {
    uint64_t insert_accepted, insert_rejected, remove_accepted, remove_rejected;
} hmc_insert_remove_count;
hmc_status hmc_grand_canonical_apply(hmc_system* sys, const hmc_grand_canonical_params* params,
                                     hmc_insert_remove_count* out);

/* The box edge lengths. hmc_set_box replaces the box as Microstate::clone_with_boundary does
 * (microstate.rs:1529-1565): every body is mapped into the new box (map_point), wrapped, and
 * the checkerboard is rebuilt; HMC_RANGE_TOO_LARGE when the box is too small for the
 * interaction range (the reference's Periodic::scale_length panics). */
hmc_status hmc_get_box(hmc_system* sys, double* edge_lengths);
hmc_status hmc_set_box(hmc_system* sys, const double* edge_lengths);
/* Bodies in the system (it grows under hmc_quick_insert_apply). */
hmc_status hmc_get_n_bodies(hmc_system* sys, uint64_t* n_bodies);

/* The insertion hamiltonian of oriented convex shapes: PairwiseCutoff(Anisotropic {
 * ApproximateShapeOverlap { Convex(shape), OverlapPenalty { k, maximum_allowed_overlap,
 * epsilon_shoulder }, resolution }, r_cut }) (hoomd-interaction/src/pairwise/anisotropic.rs:120-135,
 * approximate_shape_overlap.rs:122-131), which place_single_site_orientable_bodies
 * (benchmarks/src/place.rs:120-219) prepares convex shapes with. A pair closer than r_cut costs
 * OverlapPenalty(-d), d the distance, in steps of `resolution`, that the other shape moves along
 * the line of centres until the two no longer intersect (IntersectsAt::
 * approximate_separation_distance, hoomd-geometry/src/lib.rs:307-325).
 * hmc_set_shape_overlap(sys, params) makes it the system's hamiltonian for hmc_sweep (FP64 in both
 * precision modes; translation or rotation), hmc_quick_insert_apply (each UniformIn body also draws
 * a uniform random orientation), hmc_quick_compress_apply and hmc_total_energy;
 * hmc_set_shape_overlap(sys, NULL) returns to HardShape. Convex polyhedra and polygons
 * (HMC_HARD_CONVEX_POLYHEDRON, HMC_HARD_CONVEX_POLYGON: the bounding spheres, then XenoCollide;
 * HMC_HARD_CONVEX_SURFACE_MESH_2D: the separating-axis test alone); r_cut (0 = 2 x the bounding radius)
 * must not exceed 2 x the bounding radius. The serial sweep, the tuner, the autotuner and the
 * injected-move entry points return HMC_NOT_SUPPORTED while it is set. */
typedef struct hmc_shape_overlap_params {
    uint32_t struct_size;           /* sizeof(hmc_shape_overlap_params) */
    uint32_t reserved;
    double resolution;              /* ApproximateShapeOverlap::resolution (> 0) */
    double r_cut;                   /* Anisotropic::r_cut; 0 = 2 x the bounding radius */
    double penalty_k;               /* OverlapPenalty::k (default 10000) */
    double penalty_maximum_overlap; /* OverlapPenalty::maximum_allowed_overlap (default 0.2) */
    double penalty_shoulder;        /* OverlapPenalty::epsilon_shoulder (default 100) */
} hmc_shape_overlap_params;
hmc_status hmc_set_shape_overlap(hmc_system* sys, const hmc_shape_overlap_params* params);

/* ---- GSD files (hoomd-gsd) ----
 * The file layer replaces GsdFile (hoomd-gsd/src/file_layer.rs:559-2458): the same on-disk
 * format (GSD 2.1: 256-byte header, 32-byte index entries sorted by (frame, id), a packed list
 * of null-terminated chunk names), the same write buffering (chunks are appended to a write
 * buffer that is flushed once it holds >= the maximum write buffer size, 1 MiB by default;
 * names and index entries of completed frames reach the file only in sync), and the same
 * growth of the index and the name list (doubled, copied to the end of the file). The same
 * calls in the same order write byte-identical files.
 *
 * Errors: the calls return HMC_INVALID_ARGUMENT for caller errors and HMC_IO_ERROR for
 * failed reads/writes or a corrupt file; hmc_gsd_last_error() names the kind (the variants of
 * the reference's OpenError/DecodeError/EncodeError/ReadError/SyncError). Unlike the
 * reference, a corrupt index entry is an error, never a panic (file_layer.rs:1326-1360). */

typedef enum hmc_gsd_error {
    HMC_GSD_OK = 0,
    HMC_GSD_IO = 1,                   /* OpenError::IO, DecodeError::IO, SyncError::IO */
    HMC_GSD_NAME_TOO_LONG = 2,        /* OpenError::NameTooLong: application/schema > 63 bytes */
    HMC_GSD_NOT_WRITABLE = 3,         /* EncodeError/SyncError::NotWritable */
    HMC_GSD_DUPLICATE_CHUNK_NAME = 4, /* EncodeError::DuplicateChunkName (or in a decoded name list) */
    HMC_GSD_NAME_LIST_OVERFLOW = 5,   /* more than 65535 chunk names */
    HMC_GSD_INVALID_COLUMNS = 6,      /* EncodeError/DecodeError::InvalidColumns */
    HMC_GSD_INVALID_TYPE = 7,         /* DecodeError::InvalidType */
    HMC_GSD_CHUNK_NOT_FOUND = 8,      /* ReadError::ChunkNotFound */
    HMC_GSD_INCONSISTENT_LENGTH = 9,  /* hoomd AppendError::InconsistentLength */
    HMC_GSD_INVALID_FILE_IDENTIFIER = 10,
    HMC_GSD_UNSUPPORTED_VERSION = 11,
    HMC_GSD_INDEX_OUT_OF_BOUNDS = 12,
    HMC_GSD_NAME_LIST_OUT_OF_BOUNDS = 13,
    HMC_GSD_NAME_LIST_NOT_TERMINATED = 14,
    HMC_GSD_CORRUPT_INDEX_ENTRY = 15,
    HMC_GSD_INVALID_STRING = 16,      /* application, schema, chunk name or string chunk not UTF-8 */
    HMC_GSD_CHUNK_TOO_LARGE = 17      /* hoomd AppendError::ChunkTooLarge: N does not fit in u32 */
} hmc_gsd_error;

/* GSD data types (file_layer.rs DataType): the value stored in an index entry. */
typedef enum hmc_gsd_type {
    HMC_GSD_U8 = 1, HMC_GSD_U16 = 2, HMC_GSD_U32 = 3, HMC_GSD_U64 = 4,
    HMC_GSD_I8 = 5, HMC_GSD_I16 = 6, HMC_GSD_I32 = 7, HMC_GSD_I64 = 8,
    HMC_GSD_F32 = 9, HMC_GSD_F64 = 10, HMC_GSD_STRING = 11
} hmc_gsd_type;

/* One index entry (file_layer.rs IndexEntry): rows n, columns m, byte offset of the data. */
typedef struct hmc_gsd_chunk {
    uint64_t frame;
    uint64_t rows;
    uint64_t location;
    uint32_t columns;
    uint16_t id;
    uint8_t type;
    uint8_t flags;
} hmc_gsd_chunk;

typedef struct hmc_gsd hmc_gsd;

/* The kind of the calling thread's last failed hmc_gsd_* call (HMC_GSD_OK after a success). */
hmc_gsd_error hmc_gsd_last_error(void);

/* GsdFile::create (exclusive = 0: truncate an existing file) and GsdFile::create_new
 * (exclusive = 1: fail if the path exists); the file is open for writing. */
hmc_status hmc_gsd_create(const char* path, const char* application, const char* schema, uint16_t schema_major,
                          uint16_t schema_minor, int exclusive, hmc_gsd** out);
/* GsdFile::open; writable = 0: Mode::Read, 1: Mode::Write (appends after the last frame). */
hmc_status hmc_gsd_open(const char* path, int writable, hmc_gsd** out);
/* Drop: a writable file is synchronised first (its error is returned, the handle is freed). */
hmc_status hmc_gsd_close(hmc_gsd* file);

/* write_scalars / write_arrays / write_string: rows x columns values of type `type`
 * (columns = 1 for scalars; HMC_GSD_STRING: rows = byte length, columns = 1). */
hmc_status hmc_gsd_write_chunk(hmc_gsd* file, const char* name, uint32_t type, uint64_t rows, uint32_t columns,
                               const void* data);
/* write_strings_array: rows strings padded with zeros to (longest + 1) columns of type i8. */
hmc_status hmc_gsd_write_strings(hmc_gsd* file, const char* name, const char* const* strings, uint64_t count);
hmc_status hmc_gsd_end_frame(hmc_gsd* file);
hmc_status hmc_gsd_sync(hmc_gsd* file);
hmc_status hmc_gsd_set_maximum_write_buffer_size(hmc_gsd* file, uint64_t bytes);

/* File facts: frames in the file (n_frames), frames written so far including buffered ones,
 * file length in bytes, index entries in the file, chunk names known, header fields. Any
 * output pointer may be NULL. application/schema: buffers of >= 64 bytes. */
typedef struct hmc_gsd_info {
    uint64_t n_frames;
    uint64_t buffer_frame;
    uint64_t file_length;
    uint64_t index_entries;
    uint64_t index_allocated_entries;
    uint64_t namelist_allocated_entries;
    uint32_t n_names;
    uint16_t schema_major, schema_minor;
    uint16_t gsd_major, gsd_minor;
    int writable;
    uint64_t maximum_write_buffer_size;
    char application[64];
    char schema[64];
} hmc_gsd_info;
hmc_status hmc_gsd_get_info(hmc_gsd* file, hmc_gsd_info* out);
/* The i-th chunk name in id order (name_id); buffer of `capacity` bytes. */
hmc_status hmc_gsd_name(hmc_gsd* file, uint32_t id, char* buffer, uint64_t capacity);

/* find_chunk: *found = 0 when the frame is not in the file or the name is unknown. */
hmc_status hmc_gsd_find_chunk(hmc_gsd* file, uint64_t frame, const char* name, hmc_gsd_chunk* out, int* found);
/* iter_scalars / iter_arrays / read_string: copies the chunk's bytes into `out` after checking
 * its type (HMC_GSD_INVALID_TYPE) and columns (HMC_GSD_INVALID_COLUMNS; columns = 1 for
 * scalars and strings). capacity: bytes available at out; *rows receives the row count. */
hmc_status hmc_gsd_read_chunk(hmc_gsd* file, uint64_t frame, const char* name, uint32_t type, uint32_t columns,
                              void* out, uint64_t capacity, uint64_t* rows);

/* ---- HOOMD schema frames (hoomd-gsd/src/hoomd.rs) ----
 * hmc_gsd_create_hoomd: HoomdGsdFile::create/create_new: schema "hoomd" version 1.4 and the
 * given application (NULL: "hoomd-rs-b200"). */
hmc_status hmc_gsd_create_hoomd(const char* path, const char* application, int exclusive, hmc_gsd** out);
/* HoomdGsdFile::append_frame(step): writes configuration/step and opens a frame. */
hmc_status hmc_gsd_append_frame(hmc_gsd* file, uint64_t step);
/* Frame::particles_*: the first particles chunk of a frame writes particles/N (u32) = rows;
 * later ones must have the same rows (HMC_GSD_INCONSISTENT_LENGTH). */
hmc_status hmc_gsd_frame_particles(hmc_gsd* file, const char* name, uint32_t type, uint64_t rows, uint32_t columns,
                                   const void* data);
/* Frame::end (or drop): end_frame, then sync when the auto-sync delay (10 s by default)
 * has passed since the last sync. */
hmc_status hmc_gsd_frame_end(hmc_gsd* file);
hmc_status hmc_gsd_set_auto_sync_delay(hmc_gsd* file, double seconds);
/* AppendMicrostate::append_microstate (hoomd-microstate/src/append.rs:115-129) from the
 * device state: configuration/step, particles/N, particles/position (FP32 site positions
 * wrap(B), z = 0 in 2-D), particles/orientation (oriented shapes: FP32 site versors; in 2-D
 * the versor of the rotation by theta about z), configuration/dimensions and
 * configuration/box ([Lx, Ly, Lz or 0, 0, 0, 0]). The positions and versors are converted on
 * the GPU and copied to the host once. The frame stays open for more chunks (log/...) until
 * hmc_gsd_frame_end. */
hmc_status hmc_gsd_append_system(hmc_gsd* file, hmc_system* sys);

#ifdef __cplusplus
}
#endif
#endif /* HMC_H */
