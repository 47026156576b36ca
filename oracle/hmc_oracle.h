// CPU oracle for the hoomd-mc local-move sweep.
//
// TEST INFRASTRUCTURE ONLY. This is a plain FP64 C++ restatement of the
// reference's sweep path (glotzerlab/hoomd-rs v1.4.0, hoomd-mc and the crates it
// calls), used as the checker for the CUDA library in tests/, by
// __graft_entry__.smoke() and as the timed CPU baseline in bench.py. Nothing in
// the shipped library links, loads or calls it.
//
// It is compiled with -ffp-contract=off so that every product and sum rounds
// exactly where the reference's Rust code rounds; std::fma is called exactly
// where the reference calls f64::mul_add.
//
// All entry points use plain C types so that Python's ctypes can drive them.
#ifndef HMC_ORACLE_H
#define HMC_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

// ---- random numbers (hoomd-rand/src/sfc.rs, counter.rs) -----------------------
void oracle_sfc64_outputs(uint64_t a, uint64_t b, uint64_t c, uint64_t counter, uint64_t n_skip,
                          uint64_t n, uint64_t* out);
void oracle_sfc64_seed_from_u64(uint64_t state, uint64_t n_skip, uint64_t n, uint64_t* out);
void oracle_counter_outputs(uint64_t step, uint32_t substep, uint32_t seed, uint64_t index,
                            uint64_t n, uint64_t* out);
// Uniform f64 in [0, 1), standard normals and ball displacements from a counter stream.
void oracle_counter_uniforms(uint64_t step, uint32_t substep, uint32_t seed, uint64_t index,
                             uint64_t n, double* out);
void oracle_counter_normals(uint64_t step, uint32_t substep, uint32_t seed, uint64_t index,
                            uint64_t n, double* out);
void oracle_counter_ball(uint64_t step, uint32_t substep, uint32_t seed, uint64_t index,
                         uint32_t dim, double radius, uint64_t n, double* out);
uint32_t oracle_counter_choose(uint64_t step, uint32_t substep, uint32_t seed, uint64_t index,
                               uint32_t len);
double oracle_cbrt(double x);
void oracle_sincos_half(double theta, double* s, double* c);
// Correctly rounded sin and cos (the 2-D rotation path); returns 1 for |x| >= 2^20.
int oracle_cr_sincos(double x, double* s, double* c);
void oracle_ziggurat_tables(double* x_out /*257*/, double* f_out /*257*/);

// ---- boundary and checkerboard (hoomd-microstate boundary, hoomd-mc hypercuboid.rs) ----
void oracle_wrap(uint32_t dim, const double* edge_lengths, double* point);
// Returns the number of ghosts written (<= 7); ghosts holds dim doubles each.
uint32_t oracle_generate_ghosts(uint32_t dim, const double* edge_lengths, double range,
                                const double* point, double* ghosts);
// Returns 0 on success, 1 when the range is too large (the reference panics).
int oracle_checkerboard_dimensions(uint32_t dim, const double* edge_lengths, double range,
                                   int periodic, double* space_width, uint64_t* shape);
int64_t oracle_point_to_space_index(uint32_t dim, const double* origin, const double* space_width,
                                    const uint64_t* shape, int periodic, const double* point);
// Writes 2^dim colours x (num_spaces / 2^dim) indices.
void oracle_space_indices_by_color(uint32_t dim, const uint64_t* shape, uint64_t* out);
// Checkerboard used by ParallelSweep for the counter (step, substep, seed).
int oracle_checkerboard_for_counter(uint32_t dim, const double* edge_lengths, double range,
                                    uint64_t step, uint32_t substep, uint32_t seed,
                                    double* origin, double* space_width, uint64_t* shape);

// ---- geometry (hoomd-geometry) -----------------------------------------------------
// Convex::intersects_at in the local frame (v_ij, o_ij); q = (s, x, y, z) in 3-D,
// o_ij = theta in 2-D.
int oracle_convex_intersects_at_3d(const double* verts_a, uint32_t nv_a, const double* verts_b,
                                   uint32_t nv_b, const double* v_ij, const double* q_ij);
int oracle_convex_intersects_at_2d(const double* verts_a, uint32_t nv_a, const double* verts_b,
                                   uint32_t nv_b, const double* v_ij, double theta_ij);
// ConvexSurfaceMesh2d::intersects_at (separating axes) with theta_ij; CCW hull vertices.
int oracle_surface_mesh_intersects_at_2d(const double* verts_a, uint32_t nv_a, const double* verts_b,
                                         uint32_t nv_b, const double* v_ij, double theta_ij);
int oracle_convex_intersects_at_global_3d(const double* verts, uint32_t nv, const double* r_i,
                                          const double* q_i, const double* r_j,
                                          const double* q_j);
void oracle_versor_from_axis_angle(const double* axis, double angle, double* q);
void oracle_versor_combine(const double* a, const double* b, double* out);
void oracle_versor_rotate(const double* q, const double* v, double* out);
double oracle_lj_energy(double epsilon, double sigma, double r);
double oracle_shifted_lj_pair(double epsilon, double sigma, double r_cut, double r_shift,
                              double r_squared);

// ---- systems --------------------------------------------------------------------
enum { ORACLE_HARD_SPHERE = 0, ORACLE_HARD_CONVEX_POLYGON = 1, ORACLE_HARD_CONVEX_POLYHEDRON = 2,
       ORACLE_LENNARD_JONES = 3, ORACLE_HARD_CONVEX_SURFACE_MESH_2D = 4, ORACLE_OVERLAP_PENALTY = 5,
       ORACLE_CONVEX_POLYHEDRON_PENALTY = 6, ORACLE_CONVEX_POLYGON_PENALTY = 7, ORACLE_ISOTROPIC = 8,
       ORACLE_SURFACE_MESH_2D_PENALTY = 9 };
enum { ORACLE_TRANSLATE = 0, ORACLE_ROTATE = 1 };

typedef struct oracle_system oracle_system;

// positions: n*dim doubles; orientations: n*4 (3-D versor s,x,y,z) or n (2-D angle) or NULL.
oracle_system* oracle_system_create(uint32_t dim, const double* edge_lengths, uint64_t n,
                                    const double* positions, const double* orientations,
                                    uint64_t step, uint32_t substep, uint32_t seed,
                                    uint32_t interaction, double diameter,
                                    const double* vertices, uint32_t n_vertices, double lj_epsilon,
                                    double lj_sigma, double lj_r_cut, double lj_r_shift,
                                    double boundary_range);
void oracle_system_destroy(oracle_system* s);
void oracle_get_state(const oracle_system* s, double* positions, double* orientations,
                      uint64_t* step, uint32_t* substep);
void oracle_set_counter(oracle_system* s, uint64_t step, uint32_t substep);
// Isotropic<Expanded<OverlapPenalty>> parameters (interaction ORACLE_OVERLAP_PENALTY; the
// diameter is delta and r_cut).
void oracle_set_penalty(oracle_system* s, double k, double maximum_allowed_overlap, double epsilon_shoulder);
// Anisotropic { ApproximateShapeOverlap { shape, OverlapPenalty, resolution }, r_cut } (interactions
// ORACLE_CONVEX_POLYHEDRON_PENALTY, ORACLE_CONVEX_POLYGON_PENALTY, ORACLE_SURFACE_MESH_2D_PENALTY; the penalty's
// parameters come from oracle_set_penalty). r_cut is also the checkerboard's search range.
void oracle_set_shape_overlap(oracle_system* s, double resolution, double r_cut);
// Isotropic { W(F), r_cut } (interaction ORACLE_ISOTROPIC): F = kind (0 LennardJones {eps, sigma},
// 1 WeeksChandlerAnderson {eps, sigma}, 2 Harmonic {k, r_0}, 3 HarmonicRepulsion {a, r_cut},
// 4 Boxcar {eps, left, right}, 5 OverlapPenalty {k, d_max, eps}), W = wrap (0 none, 1 Shifted
// {r_shift}, 2 Expanded {delta}, 3 Xplor {r_cut, r_smooth}); r_cut is also the search range.
void oracle_set_isotropic(oracle_system* s, uint32_t kind, const double* params, uint32_t wrap,
                          const double* wrap_params, double r_cut);
// W(F).energy(r) for the same kinds.
double oracle_univariate_energy(uint32_t kind, const double* params, uint32_t wrap, const double* wrap_params,
                                double r);
// IntersectsAt::approximate_separation_distance of two equal convex polytopes (n_vertices x dim
// vertices): v_ij in the first shape's frame, o_ij a versor (s, x, y, z) or an angle; sat: the
// polygons are ConvexSurfaceMesh2d (the separating-axis test) instead of Convex (XenoCollide).
double oracle_approximate_separation(uint32_t dim, const double* vertices, uint32_t n_vertices, const double* v_ij,
                                     const double* o_ij, double resolution, uint32_t sat);
uint64_t oracle_n_bodies(const oracle_system* s);
void oracle_get_box(const oracle_system* s, double* edge_lengths);
// Microstate::clone_with_boundary onto a new box; 0 on success, -1 if a body is outside the box.
int oracle_set_box(oracle_system* s, const double* edge_lengths);
// QuickInsert::apply (quick_insert.rs:228-280); the progress lives in the caller's fields.
void oracle_quick_insert(oracle_system* s, uint64_t target, uint64_t allowed_overlaps, uint64_t* inserted,
                         uint32_t* complete, uint64_t* accepted, uint64_t* rejected);
// GrandCanonical::apply (grand_canonical.rs:49-110), one trial; counts[4] (insert accepted,
// insert rejected, remove accepted, remove rejected) are incremented.
void oracle_grand_canonical(oracle_system* s, double temperature, double fugacity, uint64_t* counts);
// QuickCompress::apply (quick_compress.rs:298-383); state 0..3 = Startup, Waiting, Compressing,
// Complete; boundary: the box Waiting/Complete refer to.
int oracle_quick_compress(oracle_system* s, double target_volume, double maximum_energy_per_site,
                          double maximum_delta, uint32_t* state, uint32_t* is_final, double* boundary);
// The FP32 site positions (n x 3) and site versors (n x 4, oriented shapes) that
// AppendMicrostate writes to a GSD frame (hoomd-microstate/src/append.rs:46-113).
void oracle_gsd_frame(const oracle_system* s, float* positions, float* orientations);
void oracle_increment_step(oracle_system* s);

// ParallelSweep::apply (parallel_sweep.rs:390-421). Returns 0, or 1 on a checkerboard error.
int oracle_parallel_sweep(oracle_system* s, uint32_t move, double maximum, double kt,
                          double body_interaction_range, uint64_t* accepted, uint64_t* rejected);
// The same sweep with the trials of each colour pass split over `threads` host threads;
// results are identical for every thread count.
int oracle_parallel_sweep_threads(oracle_system* s, uint32_t move, double maximum, double kt,
                                  double body_interaction_range, uint32_t threads, uint64_t* accepted,
                                  uint64_t* rejected);
// Sweep::apply (sweep.rs:159-224).
int oracle_serial_sweep(oracle_system* s, uint32_t move, double maximum, double kt,
                        uint64_t* accepted, uint64_t* rejected);
// The same with should_move_body as a mask (n bytes; NULL moves every body).
int oracle_serial_sweep_filter(oracle_system* s, uint32_t move, double maximum, double kt, const uint8_t* mask,
                               uint64_t* accepted, uint64_t* rejected);
// Move-size tuning (tune_local.rs:21-89) with per-sample counter streams; returns the tuned size.
/* Sampler probe: proposals for a body at the origin (kind 0 translate, 1 rotate, 2 normal). */
void oracle_sample_moves(uint32_t dim, uint32_t kind, double maximum, uint64_t step, uint32_t substep, uint32_t seed,
                         uint64_t n, double* out);
double oracle_tune(const oracle_system* s, uint32_t move, double maximum, double kt, double target, uint32_t samples,
                   uint32_t steps);
/* tune_local_trial with the reference's single sequential stream (tune_local.rs:42-88). */
double oracle_tune_stream(const oracle_system* s, uint32_t move, double maximum, double kt, double target,
                          uint32_t samples, uint32_t steps);
// Pair histograms (i < j) by minimum-image distance: scale distribution x = 1 - sigma/r over
// [0, x_max) and g(r) over [0, r_max); brute force over all pairs (small systems).
void oracle_sdf(const oracle_system* s, double x_max, uint32_t n_bins, uint64_t* counts);
void oracle_gr(const oracle_system* s, double r_max, uint32_t n_bins, uint64_t* counts);
// Number of overlapping pairs (hard) / total energy (LJ), pairs with tag_i < tag_j
// (pairwise_cutoff.rs:720-745).
uint64_t oracle_overlap_count(const oracle_system* s);
double oracle_total_energy(const oracle_system* s);
// delta_energy_one for one trial body (pairwise_cutoff.rs:919-941).
double oracle_delta_energy_one(const oracle_system* s, uint64_t body, const double* position,
                               const double* orientation);
// Metropolis decisions for injected moves: (body, trial properties, u). u < 0 means the
// decision needs no uniform (hard shapes). Returns decisions in out (0/1) and delta_h.
void oracle_eval_moves(const oracle_system* s, uint64_t n, const uint64_t* bodies,
                       const double* positions, const double* orientations, const double* u,
                       double kt, uint8_t* decisions, double* delta_h);

#ifdef __cplusplus
}
#endif
#endif
