// C ABI of libhmc_b200.so (declared in include/hmc.h): contexts, systems, state transfer
// and the host side of ParallelSweep::apply (hoomd-mc/src/parallel_sweep.rs:390-421).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "../../include/hmc.h"
#include "hmc_host.h"
#include "hmc_internal.cuh"

using namespace hmc;

namespace {

thread_local std::string g_last_error;

hmc_status fail(hmc_status st, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}

#define HMC_CUDA(call)                                                                                \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return fail(e_ == cudaErrorMemoryAllocation ? HMC_OUT_OF_MEMORY : HMC_CUDA_ERROR, "%s: %s (%s:%d)", \
                        #call, cudaGetErrorString(e_), __FILE__, __LINE__);                           \
    } while (0)

// HypercuboidCheckerboard::compute_dimensions for periodic axes (hypercuboid.rs:188-228).
bool compute_dimensions(int dim, const double* L, double range, double* width, uint32_t* shape) {
    for (int a = 0; a < dim; ++a) {
        double f = std::floor(L[a] / range);
        if (!(f >= 2.0) || f > 2.0e9) return false;
        uint64_t inside = (uint64_t)f;
        if (inside % 2 != 0) inside -= 1;
        width[a] = L[a] / (double)inside;
        shape[a] = (uint32_t)inside;
    }
    return true;
}

}  // namespace

// A context is shared by its systems: it is freed when hmc_context_destroy has been called
// and the last system created from it is destroyed, in whichever order these happen.
struct hmc_context {
    int device = 0;
    double* zig = nullptr;  // 2 x 257 doubles: x then f
    std::atomic<int> refs{1};
};

struct hmc_system {
    hmc_context* ctx = nullptr;
    int dim = 3;
    uint64_t n = 0;
    uint64_t step = 0;
    uint32_t substep = 0;
    uint32_t seed = 0;
    uint32_t interaction = HMC_HARD_SPHERE;
    double pair_range = 1.0;
    double boundary_range = 1.0;
    double body_range = 1.0;
    Geometry geom{};
    Pair pair{};
    Arrays arr{};
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    DeviceStats* host_stats = nullptr;  // pinned
    double* stage = nullptr;            // n x dim packed positions (host layout) for set/get_state
    unsigned long long* first_bad = nullptr;       // device word for the finiteness check
    unsigned long long* host_first_bad = nullptr;  // pinned mirror
    std::vector<void*> allocations;
    bool coop[2] = {true, false};  // warp-cooperative hard-sphere pass: [fp64, fp32]
    bool coop_set[2] = {false, false};  // coop chosen for this system (else the recorded choice)
    DeviceStats* host_slots = nullptr;  // pinned: per-sweep statistics of a pipelined call
    uint32_t slots_cap = 0;
    int32_t variant[2] = {-1, -1};  // launch variant per precision; -1: the cached choice or the default
    bool pdl = true;                // colour passes launch while the previous one finishes
    uint32_t rounds_guess = 2;      // colour sets enqueued before the sweep's count is known
    // serial sweep grid (allocated on first use)
    uint32_t serial_nc[3] = {0, 0, 0};
    double serial_w[3] = {0, 0, 0};
    uint32_t serial_cap = 0;
    uint32_t* serial_size = nullptr;
    uint32_t* serial_items = nullptr;
    uint32_t* serial_cell_of = nullptr;
    double4* serial_site = nullptr;
    uint8_t* serial_mask = nullptr;
    // convex polyhedron
    double4* verts = nullptr;
    uint32_t n_vertices = 0;
    double poly_rcut2 = 0.0;
    float poly_rcut2_hi32 = 0.f;
    bool polygon() const {
        return interaction == HMC_HARD_CONVEX_POLYGON || interaction == HMC_HARD_CONVEX_SURFACE_MESH_2D;
    }
    bool oriented() const { return interaction == HMC_HARD_CONVEX_POLYHEDRON || polygon(); }
    bool sat() const { return interaction == HMC_HARD_CONVEX_SURFACE_MESH_2D; }
    // GSD frames: FP32 positions (n x 3) then versors (n x 4), on the device and pinned
    float* gsd_dev = nullptr;
    float* gsd_host = nullptr;
    // bodies the per-body arrays hold (QuickInsert appends up to it)
    uint64_t capacity = 0;
    uint64_t cells_alloc = 0;           // spaces the checkerboard arrays hold
    double serial_L[3] = {0, 0, 0};     // box the serial grid was laid out for
    double4* backup = nullptr;          // [capacity] body positions kept across a box change
    unsigned long long* qi_out = nullptr;  // [4] QuickInsert results
    double lj_params[4] = {1, 1, 2.5, 2.5};  // epsilon, sigma, r_cut, r_shift
    // body tags (allocated when bodies are first inserted or removed on the device)
    uint32_t* tags = nullptr;
    uint32_t* tag_heap = nullptr;
    uint32_t* tag_meta = nullptr;
    bool tags_permuted = false;  // some body was removed: index order is not tag order
    bool penalty() const { return interaction == HMC_OVERLAP_PENALTY; }
    bool soft() const { return interaction == HMC_LENNARD_JONES || penalty() || interaction == HMC_ISOTROPIC; }
    // the soft interactions with an FP32 pass (the others run FP64 in both precision modes)
    bool soft_fp32() const { return interaction == HMC_LENNARD_JONES; }
    // the approximate shape overlap in place of HardShape (hmc_set_shape_overlap)
    bool shape_soft = false;
    ShapeOverlap so{};
    // profiling
    bool profiling = false;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    hmc_profile prof{};
};

namespace {

template <typename T>
hmc_status dalloc(hmc_system* s, T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * count);
    if (e != cudaSuccess)
        return fail(e == cudaErrorMemoryAllocation ? HMC_OUT_OF_MEMORY : HMC_CUDA_ERROR, "cudaMalloc(%zu bytes): %s",
                    sizeof(T) * count, cudaGetErrorString(e));
    s->allocations.push_back((void*)*p);
    return HMC_OK;
}

template <typename T>
void dfree(hmc_system* s, T** p) {
    if (!*p) return;
    auto it = std::find(s->allocations.begin(), s->allocations.end(), (void*)*p);
    if (it != s->allocations.end()) s->allocations.erase(it);
    cudaFree((void*)*p);
    *p = nullptr;
}

// HMC_B200_FP32_BAND_SCALE (> 1) widens the FP32 error bounds (the band of FP32 distances
// decided in FP64 for shapes, the LJ displacement error): decisions do not change, and the
// recheck paths become common enough to test.
double fp32_band_scale() {
    if (const char* e = std::getenv("HMC_B200_FP32_BAND_SCALE")) {
        const double f = std::atof(e);
        if (f > 1.0 && f < 1e12) return f;
    }
    return 1.0;
}

// The forward-error bound of the FP32 pair test for hard spheres. With u32 = 2^-24 and
// u64 = 2^-53, a stored FP32 offset differs from the exact offset of the FP64 site by at
// most u32*w + 4*u64*(L + w); the FP32 displacement of two offsets plus a cell shift
// then differs from the exact displacement by E <= 8*u32*w + 16*u64*(L + w) per axis.
// Near contact (d ~ sigma) the FP32 d^2 is within 2*E*sqrt(dim)*d + dim*E^2 + dim*u32*d^2
// of the exact d^2, and the reference FP64 d^2 is within 6*u64*(L+w)*sqrt(dim)*d +
// dim*u64*d^2 of it. A factor of two covers both and the rounding of the thresholds.
void sphere_bound_for(int dim, const Geometry& geom, Pair& pair) {
    const double u32 = std::ldexp(1.0, -24), u64 = std::ldexp(1.0, -53);
    double wmax = 0, Lmax = 0;
    for (int a = 0; a < dim; ++a) {
        wmax = std::max(wmax, geom.width[a]);
        Lmax = std::max(Lmax, geom.L[a]);
    }
    double sigma2 = pair.sigma2;
    double sigma = std::sqrt(sigma2);
    double E = 8.0 * u32 * wmax + 16.0 * u64 * (Lmax + wmax);
    double rd = std::sqrt((double)dim);
    double dmax = sigma * 1.01 + 1e-3;
    double b32 = 2.0 * E * rd * dmax + dim * E * E + dim * u32 * dmax * dmax;
    double b64 = 6.0 * u64 * (Lmax + wmax) * rd * dmax + dim * u64 * dmax * dmax;
    double B = 2.0 * (b32 + b64);
    B *= fp32_band_scale();
    pair.sig2_lo32 = std::nextafter((float)(sigma2 - B), -INFINITY);
    pair.sig2_hi32 = std::nextafter((float)(sigma2 + B), INFINITY);
}

void sphere_bound(hmc_system* s) { sphere_bound_for(s->dim, s->geom, s->pair); }

// LennardJones::energy (lennard_jones.rs:107-111), the host copy of the device formula.
double lj_energy_host(double four_eps, double sigma, double r) {
    double sr = sigma / r;
    double s2 = sr * sr, s4 = s2 * s2, s8 = s4 * s4;
    return four_eps * (s4 * s8 - s2 * s4);
}

// Parameters of Isotropic<Shifted<LennardJones>> and the error bounds of its FP32 pass:
// E bounds the per-axis FP32 displacement error (as for spheres); the cut-off band is the
// r^2 interval in which the FP32 r^2 cannot decide r^2 < r_cut^2, and band_energy bounds the
// energy the FP64 pass may count for a pair in it.
void lj_setup_for(int dim, const Geometry& geom, Pair& P, double eps, double sigma, double rcut, double rshift) {
    const double u32 = std::ldexp(1.0, -24), u64 = std::ldexp(1.0, -53);
    P.lj_sigma = sigma;
    P.lj_four_eps = 4.0 * eps;
    P.lj_rcut2 = rcut * rcut;
    P.lj_e_shift = lj_energy_host(P.lj_four_eps, sigma, rshift);
    P.lj_sigma2_32 = (float)(sigma * sigma);
    P.lj_four_eps32 = (float)P.lj_four_eps;
    P.lj_e_shift32 = (float)P.lj_e_shift;
    double wmax = 0, Lmax = 0;
    for (int a = 0; a < dim; ++a) {
        wmax = std::max(wmax, geom.width[a]);
        Lmax = std::max(Lmax, geom.L[a]);
    }
    // the FP32 sigma^2 and 4 eps carry one rounding each; fold them into E generously
    const double E = (8.0 * u32 * wmax + 16.0 * u64 * (Lmax + wmax) + 4.0 * u32 * sigma) * fp32_band_scale();
    P.lj_disp_err = (float)(E * 1.01);
    const double band = 2.0 * (3.5 * E * (rcut + E) + 3.1 * u32 * rcut * rcut);
    P.lj_rcut2_lo32 = std::nextafter((float)(P.lj_rcut2 - band), -INFINITY);
    P.lj_rcut2_hi32 = std::nextafter((float)(P.lj_rcut2 + band), INFINITY);
    double e_lo = lj_energy_host(P.lj_four_eps, sigma, std::sqrt(std::max(P.lj_rcut2 - 2.0 * band, 0.0))) - P.lj_e_shift;
    double e_hi = lj_energy_host(P.lj_four_eps, sigma, std::sqrt(P.lj_rcut2 + 2.0 * band)) - P.lj_e_shift;
    P.lj_band_energy = (float)(2.0 * std::max(std::fabs(e_lo), std::fabs(e_hi)) + 1e-7);
}

void lj_setup(hmc_system* s, double eps, double sigma, double rcut, double rshift) {
    lj_setup_for(s->dim, s->geom, s->pair, eps, sigma, rcut, rshift);
}

// The univariate energy F(r) of HMC_ISOTROPIC on the host (the Shifted constant F(r_shift)), in
// the same operations as univariate64 on the device (this file is compiled without contraction).
double univariate_host(uint32_t kind, const double* p, double r) {
    switch (kind) {
        case HMC_UV_LENNARD_JONES:
        case HMC_UV_WEEKS_CHANDLER_ANDERSON: {
            if (kind == HMC_UV_WEEKS_CHANDLER_ANDERSON && !(r < p[2] * p[1])) return 0.0;
            const double sr = p[1] / r;
            const double s2 = sr * sr, s4 = s2 * s2, s8 = s4 * s4;
            const double e = 4.0 * p[0] * (s4 * s8 - s2 * s4);
            return kind == HMC_UV_WEEKS_CHANDLER_ANDERSON ? e + p[0] : e;
        }
        case HMC_UV_HARMONIC:
            return 0.5 * p[0] * (r - p[1]) * (r - p[1]);
        case HMC_UV_HARMONIC_REPULSION:
            return r < p[1] ? 0.5 * p[0] / p[1] * ((r - p[1]) * (r - p[1])) : 0.0;
        case HMC_UV_BOXCAR:
            return r < p[1] ? 0.0 : (r < p[2] ? p[0] : 0.0);
        case HMC_UV_LENNARD_JONES_GAUSS: {
            const double ri = p[3] / r;
            const double x = r / p[3] - p[2];
            const double arg = -(x * x) / (2.0 * p[1]);
            const double s2 = ri * ri, s4 = s2 * s2, s8 = s4 * s4;
            return s4 * s8 - 2.0 * (s2 * s4) - p[0] * std::exp(arg);
        }
        default:
            if (r < -p[1]) return INFINITY;
            if (r < 0.0) return 0.5 * p[0] * (r * r) + p[2];
            return 0.0;
    }
}

// Pair thresholds that depend on the box (FP32 bounds use the space widths and box lengths).
void pair_setup(hmc_system* s) {
    if (s->interaction == HMC_HARD_SPHERE) {
        sphere_bound(s);
    } else if (s->oriented()) {
        s->pair.sigma2 = s->poly_rcut2;  // the FP32 prefilter threshold reuses the sphere bound
        sphere_bound(s);
        s->poly_rcut2_hi32 = s->pair.sig2_hi32;
    } else if (s->interaction == HMC_LENNARD_JONES) {
        lj_setup(s, s->lj_params[0], s->lj_params[1], s->lj_params[2], s->lj_params[3]);
    }
}

// The periodic box and its checkerboard: Periodic::new's range check (boundary/periodic.rs:
// 97-107) and HypercuboidCheckerboard::compute_dimensions (hypercuboid.rs:188-228). The
// checkerboard arrays grow when the box needs more spaces than they hold.
hmc_status setup_geometry(hmc_system* s, const double* L) {
    Geometry g = s->geom;
    for (int a = 0; a < 3; ++a) g.L[a] = a < s->dim ? L[a] : 1.0;
    double min_l = g.L[0];
    for (int a = 0; a < s->dim; ++a) {
        if (!(g.L[a] > 0.0) || !std::isfinite(g.L[a])) return fail(HMC_INVALID_ARGUMENT, "edge length %d must be positive", a);
        min_l = std::min(min_l, g.L[a]);
    }
    if (s->boundary_range > min_l / 2.0)
        return fail(HMC_RANGE_TOO_LARGE, "boundary interaction range %g exceeds L/2 = %g", s->boundary_range, min_l / 2.0);
    if (!compute_dimensions(s->dim, g.L, s->body_range, g.width, g.shape))
        return fail(HMC_RANGE_TOO_LARGE, "body interaction range %g leaves fewer than 2 spaces per axis", s->body_range);
    uint64_t cells = 1;
    g.any_two = 0;
    for (int a = 0; a < s->dim; ++a) {
        g.half[a] = g.L[a] / 2.0;
        g.ghost_hi[a] = g.half[a] - s->boundary_range;
        g.ghost_lo[a] = -g.half[a] + s->boundary_range;
        g.w32[a] = (float)g.width[a];
        g.invL[a] = 1.0 / g.L[a];
        g.invW[a] = 1.0 / g.width[a];
        g.half_shape[a] = g.shape[a] / 2;
        cells *= g.shape[a];
    }
    // 32-bit space indices and slot offsets; the packed multi-index caps the axes below
    if (cells > (1ull << 31))
        return fail(HMC_NOT_SUPPORTED, "%llu checkerboard spaces exceed the supported 2^31", (unsigned long long)cells);
    // colour lists pack the multi-index: 10 bits per axis in 3-D, 16 in 2-D
    for (int a = 0; a < s->dim; ++a) {
        if (g.shape[a] > (s->dim == 3 ? 1024u : 65535u))
            return fail(HMC_NOT_SUPPORTED, "%u spaces on axis %d exceed the supported %u", g.shape[a], a,
                        s->dim == 3 ? 1024u : 65535u);
        if (g.shape[a] == 2) g.any_two = 1;
    }
    g.n_cells = (uint32_t)cells;
    g.color_stride = (uint32_t)(cells >> s->dim);
    if (cells > s->cells_alloc) {
        Arrays& A = s->arr;
        dfree(s, &A.cell_count);
        dfree(s, &A.cell_start);
        dfree(s, &A.block_sums);
        dfree(s, &A.color_cells);
        const uint32_t scan_blocks = (uint32_t)((cells + 2047) / 2048);
        hmc_status st;
        if ((st = dalloc(s, &A.cell_count, cells)) || (st = dalloc(s, &A.cell_start, cells + 1)) ||
            (st = dalloc(s, &A.block_sums, (size_t)scan_blocks * 9)) || (st = dalloc(s, &A.color_cells, cells)))
            return st;
        if (s->soft() || s->oriented()) {  // the rounds' trial moves of the passes with lanes per trial
            dfree(s, &A.trial_t);
            dfree(s, &A.trial_o);
            dfree(s, &A.trial_k);
            dfree(s, &A.trial_q);
            if ((st = dalloc(s, &A.trial_t, cells)) || (st = dalloc(s, &A.trial_o, cells)) ||
                (st = dalloc(s, &A.trial_k, cells)))
                return st;
            if (s->interaction == HMC_HARD_CONVEX_POLYHEDRON && (st = dalloc(s, &A.trial_q, cells))) return st;
        }
        s->cells_alloc = cells;
    }
    s->geom = g;
    pair_setup(s);
    return HMC_OK;
}

hmc_status read_stats(hmc_system* s) {
    HMC_CUDA(cudaMemcpyAsync(s->host_stats, s->arr.stats, sizeof(DeviceStats), cudaMemcpyDeviceToHost, s->stream));
    HMC_CUDA(cudaStreamSynchronize(s->stream));
    return HMC_OK;
}

hmc_status check_flags(hmc_system* s) {
    uint32_t f = s->host_stats->error_flags;
    if (f & kErrNonFinite) return fail(HMC_NAN_STATE, "a body position is not finite");
    if (f & kErrOutsideCheckerboard) return fail(HMC_OUTSIDE_CHECKERBOARD, "a body maps to no checkerboard space");
    if (f & kErrAngleRange) return fail(HMC_INVALID_ARGUMENT, "a 2-D orientation angle reached 2^19 rad");
    if (f & kErrCellOverflow) return fail(HMC_CELL_OVERFLOW, "a cell of the serial sweep's grid is full");
    if (f & kErrIterationCap) return fail(HMC_ITERATION_CAP, "an approximate separation ran past its step bound");
    return HMC_OK;
}

// ---- launch variants -------------------------------------------------------------------------
// The colour-pass kernel family a system's sweep runs in a precision, and its variant table.
enum VariantFamily : uint32_t { kFamSphereDirect, kFamSphereCoop, kFamLj, kFamPoly3, kFamPoly2, kFamBatch, kFamBatchLj };

bool coop_of(const hmc_system* s, bool fp32);

uint32_t family_of(const hmc_system* s, bool fp32) {
    if (s->soft()) return kFamLj;
    if (s->interaction == HMC_HARD_CONVEX_POLYHEDRON) return kFamPoly3;
    if (s->polygon()) return kFamPoly2;
    return coop_of(s, fp32) ? kFamSphereCoop : kFamSphereDirect;
}

const LaunchShape* family_shapes(uint32_t fam, uint32_t* n) {
    switch (fam) {
        case kFamSphereDirect: *n = n_shapes(kSphereDirectShapes); return kSphereDirectShapes;
        case kFamSphereCoop: *n = n_shapes(kSphereCoopShapes); return kSphereCoopShapes;
        case kFamLj: *n = n_shapes(kLjShapes); return kLjShapes;
        case kFamPoly3: *n = n_shapes(kPolyShapes); return kPolyShapes;
        case kFamPoly2: *n = n_shapes(kPoly2Shapes); return kPoly2Shapes;
        case kFamBatch: *n = n_shapes(kBatchShapes); return kBatchShapes;
        default: *n = n_shapes(kBatchLjShapes); return kBatchLjShapes;
    }
}

// The density band of a workload: bodies per checkerboard space in quarter octaves.
int32_t density_band(double bodies, double spaces) {
    if (!(bodies > 0.0) || !(spaces > 0.0)) return -1000;
    return (int32_t)std::lround(4.0 * std::log2(bodies / spaces));
}

// Choices of hmc_autotune shared by every system and batch of the process, keyed by kernel
// family, dimension, precision and density band.
std::mutex g_variant_mutex;
std::map<std::tuple<uint32_t, uint32_t, uint32_t, int32_t>, uint32_t> g_variant_cache;

uint32_t cached_variant(uint32_t fam, uint32_t dim, bool fp32, int32_t band) {
    std::lock_guard<std::mutex> lock(g_variant_mutex);
    auto it = g_variant_cache.find(std::make_tuple(fam, dim, (uint32_t)fp32, band));
    return it == g_variant_cache.end() ? 0u : it->second;
}

void cache_variant(uint32_t fam, uint32_t dim, bool fp32, int32_t band, uint32_t v) {
    std::lock_guard<std::mutex> lock(g_variant_mutex);
    g_variant_cache[std::make_tuple(fam, dim, (uint32_t)fp32, band)] = v;
}

// Hard-sphere pass choices of hmc_autotune (true: the warp-cooperative pass), keyed by
// dimension, precision and density band; guarded by g_variant_mutex.
std::map<std::tuple<uint32_t, uint32_t, int32_t>, bool> g_pass_cache;

// Whether the next hard-sphere sweep of system s in this precision runs the warp-cooperative
// pass: the system's own choice, else the recorded one for its band, else the default.
bool coop_of(const hmc_system* s, bool fp32) {
    if (s->coop_set[fp32] || s->interaction != HMC_HARD_SPHERE) return s->coop[fp32];
    std::lock_guard<std::mutex> lock(g_variant_mutex);
    auto it = g_pass_cache.find(std::make_tuple((uint32_t)s->dim, (uint32_t)fp32,
                                                density_band((double)s->n, (double)s->geom.n_cells)));
    return it == g_pass_cache.end() ? s->coop[fp32] : it->second;
}

void cache_pass(uint32_t dim, bool fp32, int32_t band, bool coop) {
    std::lock_guard<std::mutex> lock(g_variant_mutex);
    g_pass_cache[std::make_tuple(dim, (uint32_t)fp32, band)] = coop;
}

// The variant the next sweep of system s runs in this precision.
uint32_t variant_of(const hmc_system* s, bool fp32) {
    if (s->variant[fp32] >= 0) return (uint32_t)s->variant[fp32];
    return cached_variant(family_of(s, fp32), (uint32_t)s->dim, fp32,
                          density_band((double)s->n, (double)s->geom.n_cells));
}

// Kernels of one cell-list rebuild: bin, 2 scan passes (3 for grids of more than 2048 scan
// blocks), scatter, space sort, gather.
uint32_t rebuild_kernels(const hmc_system* s) {
    return (s->n > 0 ? 6u : 2u) + ((s->geom.n_cells + 2047u) / 2048u > 2048u ? 1u : 0u);
}

// update_checkerboard (parallel_sweep.rs:176-201): origin shift from the counter's
// index u64::MAX stream, then the device counting sort into cell order.
hmc_status rebuild(hmc_system* s, bool write_s, bool write_slots = true) {
    Sfc64 rng = make_rng(s->step, s->substep, s->seed, UINT64_MAX);
    for (int a = 0; a < s->dim; ++a) {
        double off = uniform01(rng);
        s->geom.origin[a] = -s->geom.L[a] / 2.0 - off * s->geom.width[a];
    }
    HMC_CUDA(cudaMemsetAsync(s->arr.stats, 0, sizeof(DeviceStats), s->stream));
    HMC_CUDA(launch_rebuild(s->dim, s->geom, s->arr, (uint32_t)s->n, write_s, s->stream, write_slots));
    s->prof.kernel_launches += rebuild_kernels(s);
    return HMC_OK;
}

hmc_status validate_positions(const hmc_system* s, const double* pos) {
    for (uint64_t i = 0; i < s->n * (uint64_t)s->dim; ++i)
        if (!std::isfinite(pos[i])) return fail(HMC_NAN_STATE, "position %llu is not finite", (unsigned long long)(i / s->dim));
    return HMC_OK;
}

}  // namespace

namespace hmc {

hmc_status report_error(hmc_status st, const char* message) {
    g_last_error = message;
    return st;
}

// One FP32 frame of the state for a GSD file: one encoding kernel, one device-to-host copy.
hmc_status system_gsd_frame(hmc_system* s, GsdFrameView* out) {
    const uint64_t n = s->n;
    const bool ori = s->oriented();
    const uint64_t floats = n * (ori ? 7 : 3);
    HMC_CUDA(cudaSetDevice(s->ctx->device));
    if (n && !s->gsd_dev) {
        hmc_status st = dalloc(s, &s->gsd_dev, 7 * s->capacity);
        if (st != HMC_OK) return st;
        HMC_CUDA(cudaMallocHost((void**)&s->gsd_host, sizeof(float) * 7 * s->capacity));
    }
    if (n) {
        const int kind = !ori ? 0 : (s->dim == 3 ? 1 : 2);
        HMC_CUDA(launch_gsd_encode(s->dim, kind, s->geom, s->arr.body_pos, s->arr.body_ori, n, s->gsd_dev,
                                   s->gsd_dev + 3 * n, s->stream));  // versors follow the n positions
        s->prof.kernel_launches += 1;
        HMC_CUDA(cudaMemcpyAsync(s->gsd_host, s->gsd_dev, sizeof(float) * floats, cudaMemcpyDeviceToHost, s->stream));
        HMC_CUDA(cudaStreamSynchronize(s->stream));
    }
    if (n && s->tags_permuted) {
        // iter_sites_tag_order: rows in increasing tag order (tags are unique)
        std::vector<uint32_t> tag(n);
        HMC_CUDA(cudaMemcpy(tag.data(), s->tags, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost));
        std::vector<uint32_t> order(n);
        for (uint64_t i = 0; i < n; ++i) order[i] = (uint32_t)i;
        std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return tag[a] < tag[b]; });
        const int w[2] = {3, 4};
        float* base[2] = {s->gsd_host, s->gsd_host + 3 * n};
        for (int k = 0; k < (ori ? 2 : 1); ++k) {
            std::vector<float> tmp(base[k], base[k] + w[k] * n);
            for (uint64_t r = 0; r < n; ++r)
                std::memcpy(base[k] + w[k] * r, tmp.data() + (size_t)w[k] * order[r], sizeof(float) * w[k]);
        }
    }
    out->step = s->step;
    out->dim = s->dim;
    for (int a = 0; a < 3; ++a) out->L[a] = a < s->dim ? s->geom.L[a] : 0.0;
    out->n = n;
    out->position = s->gsd_host;
    out->orientation = ori ? s->gsd_host + 3 * n : nullptr;
    return HMC_OK;
}

}  // namespace hmc

extern "C" {

uint32_t hmc_abi_version(void) { return HMC_ABI_VERSION; }

const char* hmc_status_string(hmc_status st) {
    switch (st) {
        case HMC_OK: return "ok";
        case HMC_INVALID_ARGUMENT: return "invalid argument";
        case HMC_RANGE_TOO_LARGE: return "interaction range too large for the box";
        case HMC_OVERLAP_IN_INPUT: return "overlap in input";
        case HMC_CELL_OVERFLOW: return "cell overflow";
        case HMC_NAN_STATE: return "non-finite state";
        case HMC_ITERATION_CAP: return "iteration cap reached";
        case HMC_TIMEOUT: return "timeout";
        case HMC_CUDA_ERROR: return "CUDA error";
        case HMC_OUT_OF_MEMORY: return "out of device memory";
        case HMC_NOT_SUPPORTED: return "not supported";
        case HMC_OUTSIDE_CHECKERBOARD: return "body outside the checkerboard";
        case HMC_IO_ERROR: return "file I/O error or corrupt file";
    }
    return "unknown status";
}

const char* hmc_last_error_message(void) { return g_last_error.c_str(); }

hmc_status hmc_context_create(const hmc_device_opts* opts, hmc_context** out) {
    if (!out) return fail(HMC_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    int device = 0;
    if (opts) {
        if (opts->struct_size < sizeof(hmc_device_opts)) return fail(HMC_INVALID_ARGUMENT, "hmc_device_opts.struct_size");
        device = opts->device;
    }
    int count = 0;
    HMC_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) return fail(HMC_INVALID_ARGUMENT, "device %d of %d", device, count);
    HMC_CUDA(cudaSetDevice(device));
    hmc_context* c = new hmc_context();
    c->device = device;
    ZigTables t;
    zig_tables(t);
    cudaError_t e = cudaMalloc((void**)&c->zig, sizeof(double) * 2 * (kZigLayers + 1));
    if (e == cudaSuccess) e = cudaMemcpy(c->zig, t.x, sizeof(t.x), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(c->zig + kZigLayers + 1, t.f, sizeof(t.f), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        if (c->zig) cudaFree(c->zig);
        delete c;
        return fail(HMC_CUDA_ERROR, "context setup: %s", cudaGetErrorString(e));
    }
    *out = c;
    return HMC_OK;
}

static void context_release(hmc_context* c) {
    if (c->refs.fetch_sub(1) != 1) return;
    cudaSetDevice(c->device);
    if (c->zig) cudaFree(c->zig);
    cudaGetLastError();  // a destructor reports nothing: leave no sticky error behind
    delete c;
}

void hmc_context_destroy(hmc_context* c) {
    if (!c) return;
    context_release(c);
}

void hmc_system_destroy(hmc_system* s) {
    if (!s) return;
    cudaSetDevice(s->ctx->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (void* p : s->allocations) cudaFree(p);
    for (cudaEvent_t e : s->ev)
        if (e) cudaEventDestroy(e);
    if (s->host_stats) cudaFreeHost(s->host_stats);
    if (s->host_first_bad) cudaFreeHost(s->host_first_bad);
    if (s->host_slots) cudaFreeHost(s->host_slots);
    if (s->gsd_host) cudaFreeHost(s->gsd_host);
    if (s->own_stream) cudaStreamDestroy(s->own_stream);
    cudaGetLastError();  // a destructor reports nothing: leave no sticky error behind
    hmc_context* c = s->ctx;
    delete s;
    context_release(c);
}

hmc_status hmc_system_create(hmc_context* ctx, const hmc_system_desc* d, const double* positions,
                             const double* orientations, hmc_system** out) {
    if (!ctx || !d || !out) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    if (d->struct_size < sizeof(hmc_system_desc)) return fail(HMC_INVALID_ARGUMENT, "hmc_system_desc.struct_size");
    if (d->dim != 2 && d->dim != 3) return fail(HMC_INVALID_ARGUMENT, "dim must be 2 or 3 (got %u)", d->dim);
    if (d->n_bodies > 0 && !positions) return fail(HMC_INVALID_ARGUMENT, "positions is NULL");
    if (d->n_bodies >= (1ull << 31)) return fail(HMC_INVALID_ARGUMENT, "too many bodies");
    for (uint32_t a = 0; a < d->dim; ++a)
        if (!(d->edge_lengths[a] > 0.0) || !std::isfinite(d->edge_lengths[a]))
            return fail(HMC_INVALID_ARGUMENT, "edge length %u must be positive", a);
    if (d->capacity >= (1ull << 31)) return fail(HMC_INVALID_ARGUMENT, "capacity too large");
    if (d->interaction != HMC_HARD_SPHERE && d->interaction != HMC_LENNARD_JONES &&
        d->interaction != HMC_HARD_CONVEX_POLYHEDRON && d->interaction != HMC_HARD_CONVEX_POLYGON &&
        d->interaction != HMC_HARD_CONVEX_SURFACE_MESH_2D && d->interaction != HMC_OVERLAP_PENALTY &&
        d->interaction != HMC_ISOTROPIC)
        return fail(HMC_NOT_SUPPORTED, "interaction %u is not available in this build", d->interaction);
    if (d->interaction == HMC_ISOTROPIC) {
        if (d->univariate > HMC_UV_LENNARD_JONES_GAUSS || d->univariate_wrap > HMC_UVW_XPLOR)
            return fail(HMC_INVALID_ARGUMENT, "univariate %u / wrap %u", d->univariate, d->univariate_wrap);
        for (int k = 0; k < 4; ++k)
            if (!std::isfinite(d->univariate_params[k]))
                return fail(HMC_INVALID_ARGUMENT, "univariate parameters must be finite");
        for (int k = 0; k < 2; ++k)
            if (!std::isfinite(d->wrap_params[k])) return fail(HMC_INVALID_ARGUMENT, "wrap parameters must be finite");
        if (!(d->isotropic_r_cut > 0.0) || !std::isfinite(d->isotropic_r_cut))
            return fail(HMC_INVALID_ARGUMENT, "Isotropic r_cut must be positive");
        if ((d->univariate == HMC_UV_LENNARD_JONES || d->univariate == HMC_UV_WEEKS_CHANDLER_ANDERSON) &&
            !(d->univariate_params[1] > 0.0))
            return fail(HMC_INVALID_ARGUMENT, "sigma must be positive");
        if (d->univariate == HMC_UV_HARMONIC_REPULSION && !(d->univariate_params[1] > 0.0))
            return fail(HMC_INVALID_ARGUMENT, "HarmonicRepulsion r_cut must be positive");
        if (d->univariate == HMC_UV_LENNARD_JONES_GAUSS &&
            (!(d->univariate_params[1] > 0.0) || !(d->univariate_params[3] > 0.0)))
            return fail(HMC_INVALID_ARGUMENT, "LennardJonesGauss sigma_squared and scale must be positive");
    }
    const bool polygon = d->interaction == HMC_HARD_CONVEX_POLYGON || d->interaction == HMC_HARD_CONVEX_SURFACE_MESH_2D;
    if (polygon) {
        if (d->dim != 2) return fail(HMC_INVALID_ARGUMENT, "convex polygons are 2-D");
        // ConvexPolygon = ConvexPolytope<2, 32>; the separating-axis test needs a hull of >= 3
        if (d->n_vertices < 3 || d->n_vertices > 32 || !d->vertices)
            return fail(HMC_INVALID_ARGUMENT, "a convex polygon needs 3 to 32 vertices");
        for (uint32_t i = 0; i < 2 * d->n_vertices; ++i)
            if (!std::isfinite(d->vertices[i])) return fail(HMC_INVALID_ARGUMENT, "vertex coordinates must be finite");
        if (d->interaction == HMC_HARD_CONVEX_SURFACE_MESH_2D) {
            // ConvexSurfaceMesh2d keeps its hull counter-clockwise without collinear points
            // (convex_surface_mesh_2d.rs:166-260); its edge normals rely on that order.
            const uint32_t nv = d->n_vertices;
            for (uint32_t i = 0; i < nv; ++i) {
                const double* a = d->vertices + 2 * i;
                const double* b = d->vertices + 2 * ((i + 1) % nv);
                const double* c = d->vertices + 2 * ((i + 2) % nv);
                const double cross = (b[0] - a[0]) * (c[1] - b[1]) - (b[1] - a[1]) * (c[0] - b[0]);
                if (!(cross > 0.0))
                    return fail(HMC_INVALID_ARGUMENT,
                                "surface-mesh vertices must be a strictly convex counter-clockwise hull");
            }
        }
        if (d->n_bodies > 0 && orientations)
            for (uint64_t i = 0; i < d->n_bodies; ++i)
                if (!(std::fabs(orientations[i]) < 524288.0))
                    return fail(HMC_INVALID_ARGUMENT, "orientation angle %llu must be finite with |theta| < 2^19",
                                (unsigned long long)i);
    }
    if (d->interaction == HMC_HARD_CONVEX_POLYHEDRON) {
        if (d->dim != 3) return fail(HMC_INVALID_ARGUMENT, "convex polyhedra are 3-D");
        // ConvexPolytope::with_vertices: at least one vertex, at most 32 (ConvexPolyhedron)
        if (d->n_vertices < 1 || d->n_vertices > 32 || !d->vertices)
            return fail(HMC_INVALID_ARGUMENT, "a convex polyhedron needs 1 to 32 vertices");
        for (uint32_t i = 0; i < 3 * d->n_vertices; ++i)
            if (!std::isfinite(d->vertices[i])) return fail(HMC_INVALID_ARGUMENT, "vertex coordinates must be finite");
    }
    if ((d->interaction == HMC_HARD_SPHERE || d->interaction == HMC_OVERLAP_PENALTY) && !(d->diameter > 0.0))
        return fail(HMC_INVALID_ARGUMENT, "diameter must be positive");
    if (d->interaction == HMC_OVERLAP_PENALTY &&
        (!(d->penalty_k >= 0.0) || !std::isfinite(d->penalty_k) || !(d->penalty_maximum_overlap >= 0.0) ||
         !std::isfinite(d->penalty_maximum_overlap) || !std::isfinite(d->penalty_shoulder)))
        return fail(HMC_INVALID_ARGUMENT, "overlap penalty k and maximum overlap must be finite and >= 0");
    if (d->interaction == HMC_LENNARD_JONES &&
        (!(d->lj_sigma > 0.0) || !(d->lj_r_cut > 0.0) || !(d->lj_r_shift > 0.0) || !std::isfinite(d->lj_epsilon)))
        return fail(HMC_INVALID_ARGUMENT, "Lennard-Jones sigma, r_cut and r_shift must be positive");

    // maximum_interaction_range: HardSphere (hard_shape.rs:171-175) = diameter; Isotropic = r_cut;
    // HardShape (hard_shape.rs:111-118) = 2 x the bounding radius, where ConvexPolytope's
    // bounding radius (convex_polytope.rs:199-207) is sqrt(max |v|^2) with |v|^2 by mul_add.
    double bounding_radius = 0.0;
    if (d->interaction == HMC_HARD_CONVEX_POLYHEDRON || polygon) {
        double mx = 0.0;
        for (uint32_t i = 0; i < d->n_vertices; ++i) {
            const double* v = d->vertices + d->dim * i;
            double n2 = std::fma(v[1], v[1], std::fma(v[0], v[0], 0.0));
            if (d->dim == 3) n2 = std::fma(v[2], v[2], n2);
            mx = std::max(mx, n2);
        }
        bounding_radius = std::sqrt(mx);
        if (!(bounding_radius > 0.0)) return fail(HMC_INVALID_ARGUMENT, "the shape's bounding radius must be positive");
    }

    HMC_CUDA(cudaSetDevice(ctx->device));
    hmc_system* s = new hmc_system();
    ctx->refs.fetch_add(1);
    s->ctx = ctx;
    s->dim = (int)d->dim;
    s->n = d->n_bodies;
    s->capacity = std::max<uint64_t>(d->n_bodies, d->capacity);
    s->step = d->step;
    s->substep = d->substep;
    s->seed = d->seed;
    s->interaction = d->interaction;
    s->pair_range = d->interaction == HMC_ISOTROPIC       ? d->isotropic_r_cut
                    : d->interaction == HMC_LENNARD_JONES ? d->lj_r_cut
                    : (d->interaction == HMC_HARD_CONVEX_POLYHEDRON || polygon) ? bounding_radius * 2.0
                                                                  : d->diameter;
    s->boundary_range = d->boundary_range > 0.0 ? d->boundary_range : s->pair_range;
    s->body_range = d->body_interaction_range > 0.0 ? d->body_interaction_range : s->pair_range;
    auto destroy_fail = [&](hmc_status st) {
        std::string msg = g_last_error;
        hmc_system_destroy(s);
        g_last_error = msg;
        return st;
    };
    if (s->body_range < s->pair_range) {
        fail(HMC_INVALID_ARGUMENT, "body interaction range %g is below the pair range %g", s->body_range, s->pair_range);
        return destroy_fail(HMC_INVALID_ARGUMENT);
    }
    if (d->interaction == HMC_HARD_SPHERE) {
        s->pair.sigma2 = d->diameter * d->diameter;  // diameter.powi(2)
    } else if (d->interaction == HMC_HARD_CONVEX_POLYHEDRON || polygon) {
        // circumsphere rejection (convex.rs:162-165): r_cut = R + R, compared with r_cut.powi(2)
        const double rc = bounding_radius + bounding_radius;
        s->poly_rcut2 = rc * rc;
        s->n_vertices = d->n_vertices;
    } else if (d->interaction == HMC_ISOTROPIC) {
        Pair& P = s->pair;
        P.penalty = 2;
        P.uv_kind = d->univariate;
        P.uv_wrap = d->univariate_wrap;
        for (int k = 0; k < 4; ++k) P.uv_p[k] = d->univariate_params[k];
        for (int k = 0; k < 2; ++k) P.uv_w[k] = d->wrap_params[k];
        // WeeksChandlerAnderson's 2.0_f64.powf(1.0 / 6.0), from the platform's pow as in the reference
        if (P.uv_kind == HMC_UV_WEEKS_CHANDLER_ANDERSON) P.uv_p[2] = std::pow(2.0, 1.0 / 6.0);
        P.uv_shift = P.uv_wrap == HMC_UVW_SHIFTED ? univariate_host(P.uv_kind, P.uv_p, P.uv_w[0]) : 0.0;
        P.uv_rcut2 = d->isotropic_r_cut * d->isotropic_r_cut;
    } else if (d->interaction == HMC_OVERLAP_PENALTY) {
        Pair& P = s->pair;
        P.penalty = 1;
        P.sigma2 = d->diameter * d->diameter;  // pairs closer than delta overlap (energy > 0)
        P.op_rcut2 = d->diameter * d->diameter;
        P.op_delta = d->diameter;
        P.op_dmax = d->penalty_maximum_overlap;
        P.op_half_k = 0.5 * d->penalty_k;
        P.op_shoulder = d->penalty_shoulder;
    } else {
        s->lj_params[0] = d->lj_epsilon;
        s->lj_params[1] = d->lj_sigma;
        s->lj_params[2] = d->lj_r_cut;
        s->lj_params[3] = d->lj_r_shift;
    }
    {
        hmc_status st = setup_geometry(s, d->edge_lengths);
        if (st) return destroy_fail(st);
    }
    // The hard-sphere colour pass: per lane for FP32 (cheap pair tests), warp-cooperative for
    // FP64 (each pair test costs more than the coordination), as measured on B200;
    // HMC_B200_SWEEP_KERNEL=direct or =coop forces one of them for both precisions.
    // HMC_B200_PDL=0 launches every colour pass after the previous one has ended.
    if (const char* pdl = std::getenv("HMC_B200_PDL")) s->pdl = std::strcmp(pdl, "0") != 0;
    if (const char* kern = std::getenv("HMC_B200_SWEEP_KERNEL")) {
        const bool direct = std::strcmp(kern, "direct") == 0, coop = std::strcmp(kern, "coop") == 0;
        if (direct || coop) {
            s->coop[0] = s->coop[1] = coop;
            s->coop_set[0] = s->coop_set[1] = true;
        }
    }

    cudaError_t e = cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        fail(HMC_CUDA_ERROR, "cudaStreamCreate: %s", cudaGetErrorString(e));
        return destroy_fail(HMC_CUDA_ERROR);
    }
    s->stream = s->own_stream;
    e = cudaMallocHost((void**)&s->host_stats, sizeof(DeviceStats));
    if (e != cudaSuccess) {
        fail(HMC_CUDA_ERROR, "cudaMallocHost: %s", cudaGetErrorString(e));
        return destroy_fail(HMC_CUDA_ERROR);
    }
    uint64_t n = s->n;
    const uint64_t cap = s->capacity;
    hmc_status st = HMC_OK;
    Arrays& A = s->arr;
    if ((st = dalloc(s, &A.body_pos, cap)) || (st = dalloc(s, &A.sorted_b, cap)) || (st = dalloc(s, &A.sorted_s, cap)) ||
        (st = dalloc(s, &A.sorted_off, cap)) || (st = dalloc(s, &A.sorted_body, cap)) ||
        (st = dalloc(s, &A.slot_of_body, cap)) || (st = dalloc(s, &A.body_cell, cap)) ||
        (st = dalloc(s, &A.body_rank, cap)) || (st = dalloc(s, &A.body_m, cap)) || (st = dalloc(s, &A.stats, 1)) ||
        (st = dalloc(s, &A.abort_word, 1)) ||
        (st = dalloc(s, &s->stage, cap * (uint64_t)s->dim)) || (st = dalloc(s, &s->first_bad, 1)))
        return destroy_fail(st);
    e = cudaMallocHost((void**)&s->host_first_bad, sizeof(unsigned long long));
    if (e != cudaSuccess) {
        s->host_first_bad = nullptr;
        fail(HMC_OUT_OF_MEMORY, "cudaMallocHost: %s", cudaGetErrorString(e));
        return destroy_fail(HMC_OUT_OF_MEMORY);
    }
    e = cudaMemset(A.abort_word, 0, sizeof(uint32_t));
    if (e != cudaSuccess) {
        fail(HMC_CUDA_ERROR, "cudaMemset: %s", cudaGetErrorString(e));
        return destroy_fail(HMC_CUDA_ERROR);
    }
    A.body_ori = nullptr;
    A.sorted_q = nullptr;
    if (s->oriented()) {
        if ((st = dalloc(s, &A.body_ori, cap)) || (st = dalloc(s, &A.sorted_q, cap)) ||
            (st = dalloc(s, &s->verts, s->n_vertices)))
            return destroy_fail(st);
        std::vector<double4> hv(s->n_vertices);
        const uint32_t dv = (uint32_t)s->dim;
        for (uint32_t i = 0; i < s->n_vertices; ++i)
            hv[i] = make_double4(d->vertices[dv * i], d->vertices[dv * i + 1], dv == 3 ? d->vertices[dv * i + 2] : 0.0,
                                 0.0);
        e = cudaMemcpy(s->verts, hv.data(), sizeof(double4) * s->n_vertices, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && n > 0) {
            // versors (s, x, y, z) in 3-D, identity by default; angles in .x in 2-D, 0 by default
            std::vector<double4> hq(n);
            for (uint64_t i = 0; i < n; ++i) {
                if (s->dim == 3)
                    hq[i] = orientations ? make_double4(orientations[4 * i], orientations[4 * i + 1],
                                                        orientations[4 * i + 2], orientations[4 * i + 3])
                                         : make_double4(1.0, 0.0, 0.0, 0.0);
                else
                    hq[i] = make_double4(orientations ? orientations[i] : 0.0, 0.0, 0.0, 0.0);
            }
            e = cudaMemcpy(A.body_ori, hq.data(), sizeof(double4) * n, cudaMemcpyHostToDevice);
        }
        if (e != cudaSuccess) {
            fail(HMC_CUDA_ERROR, "upload: %s", cudaGetErrorString(e));
            return destroy_fail(HMC_CUDA_ERROR);
        }
    }
    A.zig_x = ctx->zig;
    A.zig_f = ctx->zig + kZigLayers + 1;
    if (n > 0) {
        if ((st = validate_positions(s, positions))) return destroy_fail(st);
        // Microstate::add_body (microstate.rs:777-835): the body keeps wrap(input).
        std::vector<double4> host(n);
        for (uint64_t i = 0; i < n; ++i) {
            double p[3] = {0.0, 0.0, 0.0};
            for (int a = 0; a < s->dim; ++a) p[a] = positions[i * s->dim + a];
            if (s->dim == 2)
                wrap<2>(s->geom.L, p);
            else
                wrap<3>(s->geom.L, p);
            host[i] = make_double4(p[0], p[1], p[2], 0.0);
        }
        e = cudaMemcpy(A.body_pos, host.data(), sizeof(double4) * n, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            fail(HMC_CUDA_ERROR, "upload: %s", cudaGetErrorString(e));
            return destroy_fail(HMC_CUDA_ERROR);
        }
    }
    *out = s;
    return HMC_OK;
}

hmc_status hmc_system_set_stream(hmc_system* s, void* stream) {
    if (!s) return fail(HMC_INVALID_ARGUMENT, "NULL system");
    HMC_CUDA(cudaStreamSynchronize(s->stream));
    s->stream = stream ? (cudaStream_t)stream : s->own_stream;
    return HMC_OK;
}

void* hmc_system_stream(hmc_system* s) { return s ? (void*)s->stream : nullptr; }

// The host arrays are copied with one cudaMemcpyAsync each (direct DMA when the caller's
// buffers are pinned) into the packed staging array, checked and unpacked on the device.
// The call returns after the copies complete, so the caller may reuse its buffers; on a
// non-finite coordinate it returns HMC_NAN_STATE and the device state is unchanged.
hmc_status hmc_set_state(hmc_system* s, const double* positions, const double* orientations, uint64_t step,
                         uint32_t substep) {
    if (!s || (s->n > 0 && !positions)) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    HMC_CUDA(cudaSetDevice(s->ctx->device));
    if (s->n) {
        const uint64_t count = s->n * (uint64_t)s->dim;
        HMC_CUDA(cudaMemcpyAsync(s->stage, positions, sizeof(double) * count, cudaMemcpyHostToDevice, s->stream));
        HMC_CUDA(cudaMemsetAsync(s->first_bad, 0xFF, sizeof(unsigned long long), s->stream));
        HMC_CUDA(launch_check_finite(s->stage, count, (uint32_t)s->dim, s->first_bad, s->stream));
        HMC_CUDA(cudaMemcpyAsync(s->host_first_bad, s->first_bad, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                 s->stream));
        HMC_CUDA(cudaStreamSynchronize(s->stream));
        if (*s->host_first_bad != ~0ull)
            return fail(HMC_NAN_STATE, "position %llu is not finite", (unsigned long long)*s->host_first_bad);
        // Positions are body positions as returned by hmc_get_state (already wrapped).
        HMC_CUDA(launch_unpack_positions(s->dim, s->stage, s->arr.body_pos, s->n, s->stream));
        if (s->oriented() && orientations && s->dim == 3)  // (s, x, y, z) per body: the double4 layout
            HMC_CUDA(cudaMemcpyAsync(s->arr.body_ori, orientations, sizeof(double4) * s->n, cudaMemcpyHostToDevice,
                                     s->stream));
        HMC_CUDA(cudaStreamSynchronize(s->stream));
        if (s->oriented() && orientations && s->dim == 2) {  // one angle per body, through the staging array
            HMC_CUDA(cudaMemcpyAsync(s->stage, orientations, sizeof(double) * s->n, cudaMemcpyHostToDevice, s->stream));
            HMC_CUDA(cudaMemsetAsync(s->first_bad, 0xFF, sizeof(unsigned long long), s->stream));
            HMC_CUDA(launch_check_angles(s->stage, s->n, s->first_bad, s->stream));
            HMC_CUDA(cudaMemcpyAsync(s->host_first_bad, s->first_bad, sizeof(unsigned long long),
                                     cudaMemcpyDeviceToHost, s->stream));
            HMC_CUDA(cudaStreamSynchronize(s->stream));
            if (*s->host_first_bad != ~0ull)
                return fail(HMC_INVALID_ARGUMENT, "orientation angle %llu must be finite with |theta| < 2^19 "
                            "(positions were set)", (unsigned long long)*s->host_first_bad);
            HMC_CUDA(launch_unpack_angles(s->stage, s->arr.body_ori, s->n, s->stream));
            HMC_CUDA(cudaStreamSynchronize(s->stream));
        }
    }
    s->step = step;
    s->substep = substep;
    return HMC_OK;
}

hmc_status hmc_get_state(hmc_system* s, double* positions, double* orientations, uint64_t* step,
                         uint32_t* substep) {
    if (!s) return fail(HMC_INVALID_ARGUMENT, "NULL system");
    if (s->n && (positions || (orientations && s->oriented()))) {
        HMC_CUDA(cudaSetDevice(s->ctx->device));
        if (positions) {
            HMC_CUDA(launch_pack_positions(s->dim, s->arr.body_pos, s->stage, s->n, s->stream));
            HMC_CUDA(cudaMemcpyAsync(positions, s->stage, sizeof(double) * s->n * s->dim, cudaMemcpyDeviceToHost,
                                     s->stream));
        }
        if (s->oriented() && orientations && s->dim == 3)
            HMC_CUDA(cudaMemcpyAsync(orientations, s->arr.body_ori, sizeof(double4) * s->n, cudaMemcpyDeviceToHost,
                                     s->stream));
        HMC_CUDA(cudaStreamSynchronize(s->stream));
        if (s->oriented() && orientations && s->dim == 2) {
            HMC_CUDA(launch_pack_angles(s->arr.body_ori, s->stage, s->n, s->stream));
            HMC_CUDA(cudaMemcpyAsync(orientations, s->stage, sizeof(double) * s->n, cudaMemcpyDeviceToHost, s->stream));
            HMC_CUDA(cudaStreamSynchronize(s->stream));
        }
    }
    if (step) *step = s->step;
    if (substep) *substep = s->substep;
    return HMC_OK;
}

hmc_status hmc_increment_step(hmc_system* s) {
    if (!s) return fail(HMC_INVALID_ARGUMENT, "NULL system");
    s->step += 1;
    s->substep = 0;
    return HMC_OK;
}

// How the sweeps of one call run: precision, launch variant and, for hard spheres, the pass.
struct SweepPlan {
    bool fp32, coop, poly2_fp32;
    uint32_t variant;
};

static SweepPlan sweep_plan(const hmc_system* s, const hmc_sweep_params* p) {
    SweepPlan sp{};
    sp.fp32 = p->precision == HMC_FP32_RECHECK;
    sp.variant = variant_of(s, sp.fp32);
    sp.coop = coop_of(s, sp.fp32);
    sp.poly2_fp32 = sp.fp32 && sp.variant == 0;  // polygon variant 1: the FP64 pass in both modes
    return sp;
}

// The cell-list rebuild of the current sweep; shapes read S in both modes, and the colour passes
// do not read slot_of_body.
static hmc_status sweep_rebuild(hmc_system* s, const SweepPlan& sp) {
    return rebuild(s, !sp.fp32 || s->oriented() || (s->soft() && !s->soft_fp32()), false);
}

static Launch sweep_launch(const hmc_system* s, const hmc_sweep_params* p) {
    Launch L{};
    L.step = s->step;
    L.seed = s->seed;
    L.max_move = p->maximum;
    L.kt = p->temperature;
    L.n_bodies = (uint32_t)s->n;
    L.n_active = s->geom.color_stride;  // grid bound; the kernels read the list lengths
    return L;
}

// Colour sets r0 .. r1-1 of the current sweep: per set the round's trial moves where a trial has
// several lanes (one thread each), then the 2^d colour passes.
static hmc_status enqueue_sets(hmc_system* s, const hmc_sweep_params* p, const SweepPlan& sp, Launch& L, uint32_t r0,
                               uint32_t r1) {
    const bool fp32 = sp.fp32;
    const uint32_t colors = 1u << s->dim;
    for (uint32_t r = r0; r < r1; ++r) {
        L.substep = s->substep + r;  // increment_substep after every full colour set
        L.round = r;
        if (s->soft()) {
            HMC_CUDA(launch_propose_lj(s->dim, fp32 && s->soft_fp32(), s->geom, s->arr, L, s->stream));
            s->prof.kernel_launches += 1;
        } else if (s->interaction == HMC_HARD_CONVEX_POLYHEDRON) {
            HMC_CUDA(launch_propose_poly(fp32 && !s->shape_soft, s->geom, s->arr, L, p->move == HMC_ROTATE,
                                         s->shape_soft, s->stream));
            s->prof.kernel_launches += 1;
        } else if (s->polygon()) {
            HMC_CUDA(launch_propose_poly2(sp.poly2_fp32 && !s->shape_soft, s->geom, s->arr, L, p->move == HMC_ROTATE,
                                          s->shape_soft, s->stream));
            s->prof.kernel_launches += 1;
        }
        for (uint32_t c = 0; c < colors; ++c) {
            L.color = c;
            L.overlap_previous = (r > 0 || c > 0) && s->pdl ? 1u : 0u;
            // the first pass after the rebuild (or after a round's proposals): launch early, wait
            // for it before reading anything
            L.early_wait = (r == 0 || s->soft() || s->oriented()) && c == 0 && s->pdl ? 1u : 0u;
            if (s->soft())  // the overlap penalty has no FP32 path: FP64 in both modes
                HMC_CUDA(launch_sweep_lj(s->dim, fp32 && s->soft_fp32(), !s->soft_fp32(), s->geom, s->arr, s->pair, L,
                                         s->stream, sp.variant));
            else if (s->shape_soft && s->dim == 3)  // FP64 in both modes
                HMC_CUDA(launch_sweep_poly3_soft(s->geom, s->arr, s->verts, s->n_vertices, s->so, L, s->stream));
            else if (s->shape_soft)
                HMC_CUDA(launch_sweep_poly2_soft(s->sat(), s->geom, s->arr, s->verts, s->n_vertices, s->so, L,
                                                 s->stream));
            else if (s->interaction == HMC_HARD_CONVEX_POLYHEDRON)
                HMC_CUDA(launch_sweep_poly(fp32, s->geom, s->arr, s->verts, s->n_vertices, s->poly_rcut2,
                                           s->poly_rcut2_hi32, L, p->move == HMC_ROTATE, s->stream, sp.variant));
            else if (s->polygon())
                HMC_CUDA(launch_sweep_poly2(sp.poly2_fp32, s->sat(), s->geom, s->arr, s->verts, s->n_vertices,
                                            s->poly_rcut2, s->poly_rcut2_hi32, L, p->move == HMC_ROTATE, s->stream));
            else
                HMC_CUDA(launch_sweep_sphere(s->dim, fp32, s->geom, s->arr, s->pair, L, sp.coop, s->stream,
                                             sp.variant));
            s->prof.kernel_launches += 1;
        }
    }
    return HMC_OK;
}

// A finished sweep into the call's Count and the system's Counter.
static void account_sweep(hmc_system* s, const hmc_sweep_params* p, const DeviceStats& d, hmc_count& total) {
    const uint32_t rounds = d.rounds;
    if (rounds > 0) s->rounds_guess = rounds;
    total.accepted += d.accepted;
    total.rejected += (uint64_t)rounds * d.nonempty - d.accepted;
    total.rechecks += d.rechecks;
    total.pair_checks += d.pair_checks;
    total.order_ambiguous += d.ambiguous;
    double me;
    unsigned long long bits = d.max_err_bits;
    std::memcpy(&me, &bits, 8);
    total.max_fp32_error = std::max(total.max_fp32_error, me);
    s->substep += rounds;
    if (p->increment_step) {
        s->step += 1;
        s->substep = 0;
    }
}

// Sweeps that increment the step, run without waiting for each one's count: every Counter of the
// call is known in advance (step + j, substep 0), so the host enqueues up to kPipelineSweeps
// sweeps back to back, each with the previous sweep's number of colour sets and its statistics
// copied to a pinned slot. After each sweep k_sweep_guard raises the abort word when the sweep
// needed more colour sets (or flagged an error); every later sweep then finds kErrAborted in its
// statistics (k_bin puts it there) and runs no colour pass. The host waits once, reads the slots,
// completes a sweep that needed more sets (the same origin gives the same spaces, since bodies
// do not leave their spaces within a sweep) and enqueues the sweeps after it again.
constexpr uint32_t kPipelineSweeps = 64;

static hmc_status sweep_pipelined(hmc_system* s, const hmc_sweep_params* p, hmc_count& total) {
    if (s->slots_cap < kPipelineSweeps) {
        if (s->host_slots) cudaFreeHost(s->host_slots);
        s->host_slots = nullptr;
        s->slots_cap = 0;
        HMC_CUDA(cudaMallocHost((void**)&s->host_slots, sizeof(DeviceStats) * kPipelineSweeps));
        s->slots_cap = kPipelineSweeps;
    }
    const SweepPlan sp = sweep_plan(s, p);
    uint32_t done = 0;
    while (done < p->n_sweeps) {
        const uint32_t chunk = std::min(p->n_sweeps - done, kPipelineSweeps);
        const uint32_t guess = std::max(1u, s->rounds_guess);
        const uint64_t step0 = s->step;
        const uint32_t substep0 = s->substep;
        hmc_status st = HMC_OK;
        for (uint32_t j = 0; j < chunk && !st; ++j) {
            s->step = step0 + j;
            s->substep = j == 0 ? substep0 : 0u;
            if ((st = sweep_rebuild(s, sp))) break;
            Launch L = sweep_launch(s, p);
            if ((st = enqueue_sets(s, p, sp, L, 0, guess))) break;
            cudaError_t e = launch_sweep_guard(s->arr.stats, guess, s->arr.abort_word, s->stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(s->host_slots + j, s->arr.stats, sizeof(DeviceStats), cudaMemcpyDeviceToHost,
                                    s->stream);
            if (e != cudaSuccess) st = fail(HMC_CUDA_ERROR, "pipelined sweep: %s", cudaGetErrorString(e));
            s->prof.kernel_launches += 1;
        }
        s->step = step0;
        s->substep = substep0;
        HMC_CUDA(cudaStreamSynchronize(s->stream));
        if (st) {
            cudaMemsetAsync(s->arr.abort_word, 0, sizeof(uint32_t), s->stream);
            return st;
        }
        for (uint32_t j = 0; j < chunk; ++j) {
            DeviceStats d = s->host_slots[j];
            if (d.error_flags & kErrAborted) break;  // a sweep before it stopped the chunk
            const bool short_sets = d.rounds > guess;
            if (short_sets || d.error_flags) HMC_CUDA(cudaMemsetAsync(s->arr.abort_word, 0, sizeof(uint32_t), s->stream));
            if (d.error_flags) {
                *s->host_stats = d;
                HMC_CUDA(cudaStreamSynchronize(s->stream));
                return check_flags(s);  // the colour passes left the state untouched
            }
            if (short_sets) {  // this sweep's missing colour sets, then the sweeps after it again
                if ((st = sweep_rebuild(s, sp))) return st;
                Launch L = sweep_launch(s, p);
                if ((st = enqueue_sets(s, p, sp, L, guess, d.rounds))) return st;
                if ((st = read_stats(s))) return st;
                if ((st = check_flags(s))) return st;
                const DeviceStats& x = *s->host_stats;
                d.accepted += x.accepted;
                d.rechecks += x.rechecks;
                d.pair_checks += x.pair_checks;
                d.ambiguous += x.ambiguous;
                d.max_err_bits = std::max(d.max_err_bits, x.max_err_bits);
            }
            account_sweep(s, p, d, total);
            done += 1;
            if (short_sets) break;
        }
    }
    return HMC_OK;
}

hmc_status hmc_sweep(hmc_system* s, const hmc_sweep_params* p, hmc_count* out) {
    if (!s || !p) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (p->struct_size < sizeof(hmc_sweep_params)) return fail(HMC_INVALID_ARGUMENT, "hmc_sweep_params.struct_size");
    if (p->move != HMC_TRANSLATE && !(p->move == HMC_ROTATE && s->oriented()))
        return fail(HMC_NOT_SUPPORTED, "rotation moves need oriented bodies (convex polyhedra)");
    if (!(p->maximum > 0.0) || !std::isfinite(p->maximum)) return fail(HMC_INVALID_ARGUMENT, "maximum must be positive");
    // The 2-D ball sampler squares the radius; keep it far from overflow. Moves longer
    // than the box are equivalent modulo wrapping, so this rejects no useful input.
    double lmax = 0.0;
    for (int a = 0; a < s->dim; ++a) lmax = std::max(lmax, s->geom.L[a]);
    if (p->maximum > 4.0 * lmax) return fail(HMC_INVALID_ARGUMENT, "maximum %g exceeds 4 box lengths", p->maximum);
    if (!(p->temperature > 0.0)) return fail(HMC_INVALID_ARGUMENT, "temperature must be positive");
    if (p->precision > HMC_FP32_RECHECK) return fail(HMC_INVALID_ARGUMENT, "precision");
    HMC_CUDA(cudaSetDevice(s->ctx->device));
    hmc_count total{};
    if (p->increment_step && p->n_sweeps > 1 && s->n > 0 && !s->profiling) {
        hmc_status st = sweep_pipelined(s, p, total);
        if (st) return st;
        if (out) *out = total;
        return HMC_OK;
    }
    const SweepPlan sp = sweep_plan(s, p);
    const uint32_t colors = 1u << s->dim;
    for (uint32_t sweep = 0; sweep < p->n_sweeps; ++sweep) {
        if (s->profiling) HMC_CUDA(cudaEventRecord(s->ev[0], s->stream));
        hmc_status st = sweep_rebuild(s, sp);
        if (st) return st;
        if (s->profiling) HMC_CUDA(cudaEventRecord(s->ev[1], s->stream));
        Launch L = sweep_launch(s, p);
        if (s->profiling) HMC_CUDA(cudaEventRecord(s->ev[2], s->stream));
        // The rounds (while count.total() < N, :402-418) are known on the device after the
        // rebuild; the host enqueues the previous sweep's number of colour sets without
        // waiting, the kernels skip sets beyond the true count, and any missing sets follow.
        const uint32_t guess = s->n == 0 ? 0u : s->rounds_guess;
        if ((st = enqueue_sets(s, p, sp, L, 0, guess))) return st;
        // the passes' end is recorded before the host waits for the counts, so that profiling adds
        // no host round trip to the sweep
        if (s->profiling) HMC_CUDA(cudaEventRecord(s->ev[3], s->stream));
        if ((st = read_stats(s))) return st;
        if ((st = check_flags(s))) return st;  // the kernels left the state untouched
        const uint32_t rounds = s->host_stats->rounds;
        if (rounds > guess) {
            if ((st = enqueue_sets(s, p, sp, L, guess, rounds))) return st;
            if (s->profiling) HMC_CUDA(cudaEventRecord(s->ev[3], s->stream));
            if ((st = read_stats(s))) return st;
        }
        if (s->profiling) {
            HMC_CUDA(cudaEventSynchronize(s->ev[3]));
            float t_rebuild = 0.f, t_sweep = 0.f;
            HMC_CUDA(cudaEventElapsedTime(&t_rebuild, s->ev[0], s->ev[1]));
            HMC_CUDA(cudaEventElapsedTime(&t_sweep, s->ev[2], s->ev[3]));
            s->prof.rebuild_ms += t_rebuild;
            s->prof.rebuild_launches += rebuild_kernels(s);
            s->prof.sweep_ms += t_sweep;
            s->prof.sweep_launches += (uint64_t)std::max(rounds, guess) * colors;
            s->prof.sweeps += 1;
        }
        account_sweep(s, p, *s->host_stats, total);
    }
    if (out) *out = total;
    return HMC_OK;
}

static void describe_variant(uint32_t fam, uint32_t index, hmc_launch_variant* out) {
    uint32_t n = 0;
    const LaunchShape* t = family_shapes(fam, &n);
    const LaunchShape& v = t[index < n ? index : 0];
    out->index = index < n ? index : 0;
    out->count = n;
    out->blocks_per_sm = v.blocks_per_sm;
    out->trials_per_warp = v.trials_per_warp;
    out->own_steps = v.own_steps;
}

hmc_status hmc_get_launch_variant(hmc_system* s, uint32_t precision, uint32_t index, hmc_launch_variant* out) {
    if (!s || !out) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (precision > HMC_FP32_RECHECK) return fail(HMC_INVALID_ARGUMENT, "precision");
    const bool fp32 = precision == HMC_FP32_RECHECK;
    const uint32_t fam = family_of(s, fp32);
    uint32_t n = 0;
    family_shapes(fam, &n);
    if (index != UINT32_MAX && index >= n) return fail(HMC_INVALID_ARGUMENT, "variant %u of %u", index, n);
    describe_variant(fam, index == UINT32_MAX ? variant_of(s, fp32) : index, out);
    return HMC_OK;
}

hmc_status hmc_set_cooperative_pass(hmc_system* s, uint32_t precision, uint32_t cooperative) {
    if (!s) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (precision > HMC_FP32_RECHECK) return fail(HMC_INVALID_ARGUMENT, "precision");
    if (s->interaction != HMC_HARD_SPHERE) return fail(HMC_NOT_SUPPORTED, "the cooperative pass is for hard spheres");
    const bool fp32 = precision == HMC_FP32_RECHECK;
    if (coop_of(s, fp32) != (cooperative != 0)) s->variant[fp32] = -1;  // the other pass has its own variants
    s->coop[fp32] = cooperative != 0;
    s->coop_set[fp32] = true;
    return HMC_OK;
}

hmc_status hmc_get_cooperative_pass(hmc_system* s, uint32_t precision, uint32_t* cooperative) {
    if (!s || !cooperative) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (precision > HMC_FP32_RECHECK) return fail(HMC_INVALID_ARGUMENT, "precision");
    if (s->interaction != HMC_HARD_SPHERE) return fail(HMC_NOT_SUPPORTED, "the cooperative pass is for hard spheres");
    *cooperative = coop_of(s, precision == HMC_FP32_RECHECK) ? 1u : 0u;
    return HMC_OK;
}

hmc_status hmc_set_launch_variant(hmc_system* s, uint32_t precision, uint32_t index) {
    if (!s) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (precision > HMC_FP32_RECHECK) return fail(HMC_INVALID_ARGUMENT, "precision");
    const bool fp32 = precision == HMC_FP32_RECHECK;
    uint32_t n = 0;
    family_shapes(family_of(s, fp32), &n);
    if (index != UINT32_MAX && index >= n) return fail(HMC_INVALID_ARGUMENT, "variant %u of %u", index, n);
    s->variant[fp32] = index == UINT32_MAX ? -1 : (int32_t)index;
    return HMC_OK;
}

}  // extern "C"

// Times `sweeps` sweeps (after one untimed) from the state saved in `save`, restoring it first;
// run(p) sweeps, restore() puts the saved state back. Returns the mean device time of a sweep
// (CUDA events on the stream around the host calls, so the host's share counts too).
template <typename Run, typename Restore>
static hmc_status time_variant(cudaStream_t stream, const hmc_sweep_params& p, uint32_t sweeps, Run&& run,
                               Restore&& restore, double* ms) {
    hmc_status st;
    if ((st = restore())) return st;
    hmc_sweep_params one = p;
    one.n_sweeps = 1;
    one.increment_step = 1;
    if ((st = run(one))) return st;  // warm-up (and the first rebuild's allocations)
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    HMC_CUDA(cudaEventCreate(&e0));
    cudaError_t e = cudaEventCreate(&e1);
    hmc_sweep_params many = one;
    many.n_sweeps = sweeps;
    if (e == cudaSuccess) e = cudaEventRecord(e0, stream);
    if (e == cudaSuccess && !(st = run(many))) e = cudaEventRecord(e1, stream);
    float t = 0.f;
    if (e == cudaSuccess && !st) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess && !st) e = cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) return st;
    if (e != cudaSuccess) return fail(HMC_CUDA_ERROR, "autotune timing: %s", cudaGetErrorString(e));
    *ms = (double)t / (double)sweeps;
    return HMC_OK;
}

extern "C" {

hmc_status hmc_autotune(hmc_system* s, const hmc_sweep_params* p, uint32_t sweeps, hmc_launch_variant* chosen,
                        double* ms_per_sweep) {
    if (!s || !p) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (s->shape_soft)
        return fail(HMC_NOT_SUPPORTED, "hmc_autotune runs under HardShape: hmc_set_shape_overlap(s, NULL) first");
    if (p->struct_size < sizeof(hmc_sweep_params)) return fail(HMC_INVALID_ARGUMENT, "hmc_sweep_params.struct_size");
    if (p->precision > HMC_FP32_RECHECK) return fail(HMC_INVALID_ARGUMENT, "precision");
    if (sweeps == 0 || sweeps > 1000) return fail(HMC_INVALID_ARGUMENT, "sweeps must be in [1, 1000]");
    HMC_CUDA(cudaSetDevice(s->ctx->device));
    const bool fp32 = p->precision == HMC_FP32_RECHECK;
    // hard spheres without a pass chosen for the system: both passes (a lane or a warp per
    // trial) and each one's variants, the current pass first
    const bool coop0 = coop_of(s, fp32), coop_set0 = s->coop_set[fp32], coop_own0 = s->coop[fp32];
    const bool both = s->interaction == HMC_HARD_SPHERE && !coop_set0;
    // the state to start every variant from
    const uint64_t n = s->n;
    const uint64_t step0 = s->step;
    const uint32_t substep0 = s->substep, guess0 = s->rounds_guess;
    const int32_t own0 = s->variant[fp32];
    double4 *bp = nullptr, *bq = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&bp, sizeof(double4) * (n ? n : 1), s->stream);
    if (e == cudaSuccess && n)
        e = cudaMemcpyAsync(bp, s->arr.body_pos, sizeof(double4) * n, cudaMemcpyDeviceToDevice, s->stream);
    if (e == cudaSuccess && s->arr.body_ori) {
        e = cudaMallocAsync((void**)&bq, sizeof(double4) * (n ? n : 1), s->stream);
        if (e == cudaSuccess && n)
            e = cudaMemcpyAsync(bq, s->arr.body_ori, sizeof(double4) * n, cudaMemcpyDeviceToDevice, s->stream);
    }
    auto restore = [&]() -> hmc_status {
        if (n) HMC_CUDA(cudaMemcpyAsync(s->arr.body_pos, bp, sizeof(double4) * n, cudaMemcpyDeviceToDevice, s->stream));
        if (bq && n)
            HMC_CUDA(cudaMemcpyAsync(s->arr.body_ori, bq, sizeof(double4) * n, cudaMemcpyDeviceToDevice, s->stream));
        s->step = step0;
        s->substep = substep0;
        s->rounds_guess = guess0;
        return HMC_OK;
    };
    auto run = [&](const hmc_sweep_params& q) -> hmc_status { return hmc_sweep(s, &q, nullptr); };
    hmc_status st = e == cudaSuccess ? HMC_OK : fail(HMC_CUDA_ERROR, "autotune: %s", cudaGetErrorString(e));
    std::vector<double> ms, best_ms;
    uint32_t best = 0, best_fam = family_of(s, fp32);
    bool best_coop = coop0, have = false;
    double best_t = 0.0;
    for (int k = 0; k < (both ? 2 : 1) && !st; ++k) {
        const bool coop = k == 0 ? coop0 : !coop0;
        if (both) {
            s->coop[fp32] = coop;
            s->coop_set[fp32] = true;
        }
        const uint32_t fam = family_of(s, fp32);
        uint32_t n_var = 0;
        family_shapes(fam, &n_var);
        ms.assign(n_var, 0.0);
        for (uint32_t v = 0; v < n_var && !st; ++v) {
            s->variant[fp32] = (int32_t)v;
            st = time_variant(s->stream, *p, sweeps, run, restore, &ms[v]);
            if (!st && (!have || ms[v] < best_t)) {
                have = true;
                best_t = ms[v];
                best = v;
                best_fam = fam;
                best_coop = coop;
            }
        }
        if (!st && best_fam == fam && best_coop == coop) best_ms = ms;  // the chosen pass's times
    }
    hmc_status st2 = restore();
    if (bp) cudaFreeAsync(bp, s->stream);
    if (bq) cudaFreeAsync(bq, s->stream);
    cudaStreamSynchronize(s->stream);
    if (st || st2) {
        s->variant[fp32] = own0;
        s->coop[fp32] = coop_own0;
        s->coop_set[fp32] = coop_set0;
        return st ? st : st2;
    }
    const int32_t band = density_band((double)s->n, (double)s->geom.n_cells);
    if (both) {  // the pass chosen becomes the system's own, and the recorded one for its band
        s->coop[fp32] = best_coop;
        s->coop_set[fp32] = true;
        cache_pass((uint32_t)s->dim, fp32, band, best_coop);
    }
    s->variant[fp32] = (int32_t)best;
    cache_variant(best_fam, (uint32_t)s->dim, fp32, band, best);
    if (chosen) describe_variant(best_fam, best, chosen);
    if (ms_per_sweep) std::memcpy(ms_per_sweep, best_ms.data(), sizeof(double) * best_ms.size());
    return HMC_OK;
}

hmc_status hmc_math_sincos(hmc_context* ctx, const double* x, uint64_t n, double* sn, double* cs) {
    if (!ctx || (n > 0 && (!x || !sn || !cs))) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (n == 0) return HMC_OK;
    HMC_CUDA(cudaSetDevice(ctx->device));
    double* d = nullptr;
    uint32_t* bad = nullptr;
    uint32_t hbad = 0;
    cudaError_t e = cudaMalloc((void**)&d, sizeof(double) * 3 * n);
    if (e == cudaSuccess) e = cudaMalloc((void**)&bad, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemcpy(d, x, sizeof(double) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(bad, 0, sizeof(uint32_t));
    if (e == cudaSuccess) e = launch_sincos(d, n, d + n, d + 2 * n, bad, nullptr);
    if (e == cudaSuccess) e = cudaMemcpy(sn, d + n, sizeof(double) * n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(cs, d + 2 * n, sizeof(double) * n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&hbad, bad, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (d) cudaFree(d);
    if (bad) cudaFree(bad);
    if (e != cudaSuccess) return fail(HMC_CUDA_ERROR, "sincos: %s", cudaGetErrorString(e));
    if (hbad) return fail(HMC_INVALID_ARGUMENT, "an argument has |x| >= 2^20");
    return HMC_OK;
}

hmc_status hmc_sample_moves(hmc_context* ctx, uint32_t dim, uint32_t kind, double maximum, uint64_t step,
                            uint32_t substep, uint32_t seed, uint64_t n, double* out) {
    if (!ctx || (n > 0 && !out)) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (dim != 2 && dim != 3) return fail(HMC_INVALID_ARGUMENT, "dim must be 2 or 3");
    if (kind > 2) return fail(HMC_INVALID_ARGUMENT, "kind: 0 translate, 1 rotate, 2 standard normal");
    if (kind != 2 && !(maximum > 0.0 && std::isfinite(maximum))) return fail(HMC_INVALID_ARGUMENT, "maximum");
    if (n == 0) return HMC_OK;
    if (n >= (1ull << 31)) return fail(HMC_INVALID_ARGUMENT, "too many samples");
    const uint64_t per = kind == 2 ? 1 : (kind == 0 ? dim : (dim == 3 ? 4 : 1));
    HMC_CUDA(cudaSetDevice(ctx->device));
    double* d = nullptr;
    cudaError_t e = cudaMalloc((void**)&d, sizeof(double) * per * n);
    if (e == cudaSuccess) e = launch_sample_moves((int)dim, kind, maximum, step, substep, seed, n, ctx->zig, d, nullptr);
    if (e == cudaSuccess) e = cudaMemcpy(out, d, sizeof(double) * per * n, cudaMemcpyDeviceToHost);
    if (d) cudaFree(d);
    if (e != cudaSuccess) return fail(HMC_CUDA_ERROR, "sample_moves: %s", cudaGetErrorString(e));
    return HMC_OK;
}

// Sweep::apply_with_filter (hoomd-mc/src/sweep.rs:159-224) for hard spheres: bodies in index
// order, one sequential stream Counter(step, substep, seed).make_rng(), then
// increment_substep. move_mask (n bytes, may be NULL) plays should_move_body.
// The serial grid (cells at least the pair range wide), laid out again when the box changed.
static hmc_status serial_grid(hmc_system* s) {
    bool same = s->serial_size != nullptr;
    for (int a = 0; a < s->dim; ++a) same = same && s->serial_L[a] == s->geom.L[a];
    if (same) return HMC_OK;
    dfree(s, &s->serial_size);
    dfree(s, &s->serial_items);
    uint64_t cells = 1;
    for (int a = 0; a < s->dim; ++a) {
        double f = std::floor(s->geom.L[a] / s->pair_range);
        s->serial_nc[a] = f >= 1.0 ? (uint32_t)std::min(f, 1024.0) : 1u;
        s->serial_w[a] = s->geom.L[a] / (double)s->serial_nc[a];
        s->serial_L[a] = s->geom.L[a];
        cells *= s->serial_nc[a];
    }
    s->serial_cap = (uint32_t)std::min<uint64_t>(4096, 4 * (s->capacity / cells + 1) + 64);
    hmc_status st;
    if ((st = dalloc(s, &s->serial_size, cells)) || (st = dalloc(s, &s->serial_items, cells * s->serial_cap)))
        return st;
    if (!s->serial_cell_of) {
        if ((st = dalloc(s, &s->serial_cell_of, s->capacity)) || (st = dalloc(s, &s->serial_site, s->capacity)) ||
            (st = dalloc(s, &s->serial_mask, s->capacity)))
            return st;
    }
    return HMC_OK;
}

hmc_status hmc_serial_sweep(hmc_system* s, const hmc_sweep_params* p, const uint8_t* move_mask, hmc_count* out) {
    if (!s || !p) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (s->shape_soft)
        return fail(HMC_NOT_SUPPORTED, "hmc_serial_sweep runs under HardShape: hmc_set_shape_overlap(s, NULL) first");
    if (p->struct_size < sizeof(hmc_sweep_params)) return fail(HMC_INVALID_ARGUMENT, "hmc_sweep_params.struct_size");
    if (p->move != HMC_TRANSLATE && !(p->move == HMC_ROTATE && s->oriented()))
        return fail(HMC_NOT_SUPPORTED, "rotation moves need oriented bodies (convex polyhedra or polygons)");
    if (!(p->temperature > 0.0)) return fail(HMC_INVALID_ARGUMENT, "temperature must be positive");
    double lmax = 0.0;
    for (int a = 0; a < s->dim; ++a) lmax = std::max(lmax, s->geom.L[a]);
    if (!(p->maximum > 0.0) || !(p->maximum <= 4.0 * lmax))
        return fail(HMC_INVALID_ARGUMENT, "maximum must be in (0, 4 box lengths]");
    HMC_CUDA(cudaSetDevice(s->ctx->device));
    {
        hmc_status st = serial_grid(s);
        if (st) return st;
    }
    uint64_t moving = s->n;
    if (move_mask) {
        moving = 0;
        for (uint64_t i = 0; i < s->n; ++i) moving += move_mask[i] ? 1 : 0;
        if (s->n) HMC_CUDA(cudaMemcpyAsync(s->serial_mask, move_mask, s->n, cudaMemcpyHostToDevice, s->stream));
    }
    hmc_count total{};
    for (uint32_t sweep = 0; sweep < p->n_sweeps; ++sweep) {
        Launch L{};
        L.step = s->step;
        L.substep = s->substep;
        L.seed = s->seed;
        L.max_move = p->maximum;
        L.kt = p->temperature;
        L.n_bodies = (uint32_t)s->n;
        HMC_CUDA(cudaMemsetAsync(s->arr.stats, 0, sizeof(DeviceStats), s->stream));
        const uint8_t* mask = move_mask ? s->serial_mask : nullptr;
        const bool rot = p->move == HMC_ROTATE;
        if (s->polygon())
            HMC_CUDA(launch_serial_poly2(s->sat(), s->geom, s->arr, s->verts, s->n_vertices, s->poly_rcut2, L, rot,
                                         s->serial_nc, s->serial_w, s->serial_cap, s->serial_size, s->serial_items,
                                         s->serial_cell_of, s->serial_site, mask, s->stream));
        else if (s->oriented())
            HMC_CUDA(launch_serial_poly(s->geom, s->arr, s->verts, s->n_vertices, s->poly_rcut2, L, rot, s->serial_nc,
                                        s->serial_w, s->serial_cap, s->serial_size, s->serial_items,
                                        s->serial_cell_of, s->serial_site, mask, s->stream));
        else
            HMC_CUDA(launch_serial_sphere(s->dim, s->soft(), s->geom, s->arr, s->pair, L, s->serial_nc, s->serial_w,
                                          s->serial_cap, s->serial_size, s->serial_items, s->serial_cell_of,
                                          s->serial_site, mask, s->stream));
        s->prof.kernel_launches += 2;
        hmc_status st;
        if ((st = read_stats(s))) return st;
        if ((st = check_flags(s))) return st;
        total.accepted += s->host_stats->accepted;
        total.rejected += moving - s->host_stats->accepted;
        total.order_ambiguous += s->host_stats->ambiguous;
        s->substep += 1;  // increment_substep (sweep.rs:222)
        if (p->increment_step) {
            s->step += 1;
            s->substep = 0;
        }
    }
    if (out) *out = total;
    return HMC_OK;
}

hmc_status hmc_profile_enable(hmc_system* s, int enable) {
    if (!s) return fail(HMC_INVALID_ARGUMENT, "NULL system");
    HMC_CUDA(cudaSetDevice(s->ctx->device));
    for (cudaEvent_t& e : s->ev)
        if (!e) HMC_CUDA(cudaEventCreate(&e));
    s->profiling = enable != 0;
    return HMC_OK;
}

hmc_status hmc_profile_read(hmc_system* s, hmc_profile* out, int reset) {
    if (!s || !out) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    *out = s->prof;
    if (reset) s->prof = hmc_profile{};
    return HMC_OK;
}

// Tune::tune_with_options for ParallelSweep (hoomd-mc/src/lib.rs:430-449, tune_local.rs:21-89):
// `steps` rounds of `samples` trial moves of random bodies against the unchanged state, each
// round scaling the move size by (acceptance + 1.5) / (target + 1.5) (tune_by_scaling,
// lib.rs:514-524). The state and its counters are not modified.
hmc_status hmc_tune(hmc_system* s, hmc_sweep_params* p, double target, uint32_t samples, uint32_t steps) {
    if (!s || !p) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (s->shape_soft)
        return fail(HMC_NOT_SUPPORTED, "hmc_tune runs under HardShape: hmc_set_shape_overlap(s, NULL) first");
    if (p->struct_size < sizeof(hmc_sweep_params)) return fail(HMC_INVALID_ARGUMENT, "hmc_sweep_params.struct_size");
    if (!(target > 0.0 && target < 1.0)) return fail(HMC_INVALID_ARGUMENT, "target acceptance must be in (0, 1)");
    if (p->move != HMC_TRANSLATE && !(p->move == HMC_ROTATE && s->oriented()))
        return fail(HMC_NOT_SUPPORTED, "rotation moves need oriented bodies (convex polyhedra)");
    if (!(p->maximum > 0.0) || !std::isfinite(p->maximum)) return fail(HMC_INVALID_ARGUMENT, "maximum must be positive");
    if (!(p->temperature > 0.0)) return fail(HMC_INVALID_ARGUMENT, "temperature must be positive");
    if (samples == 0 || samples >= (1u << 31)) return fail(HMC_INVALID_ARGUMENT, "samples must be in [1, 2^31)");
    if (p->flags & ~HMC_TUNE_PER_SAMPLE_STREAMS) return fail(HMC_INVALID_ARGUMENT, "unknown tune flags");
    if (s->n == 0 || steps == 0) return HMC_OK;
    HMC_CUDA(cudaSetDevice(s->ctx->device));
    hmc_status st = rebuild(s, true);
    if (st) return st;
    if (!(p->flags & HMC_TUNE_PER_SAMPLE_STREAMS)) {
        // the reference's single stream, one warp (tune_stream_run)
        TuneJob job{};
        job.g = s->geom;
        job.a = s->arr;
        job.p = s->pair;
        job.step = s->step;
        job.substep = s->substep;
        job.seed = s->seed;
        job.n_bodies = (uint32_t)s->n;
        job.samples = samples;
        job.steps = steps;
        job.rotate = p->move == HMC_ROTATE ? 1u : 0u;
        job.maximum = p->maximum;
        job.kt = p->temperature;
        job.target = target;
        const double pi = 3.141592653589793;
        job.cap = p->move == HMC_ROTATE ? (s->dim == 3 ? pi / 2.0 : pi) : 0.0;
        TuneJob* dj = nullptr;
        cudaError_t e = cudaMallocAsync((void**)&dj, sizeof(TuneJob), s->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dj, &job, sizeof(TuneJob), cudaMemcpyHostToDevice, s->stream);
        if (e == cudaSuccess) {
            if (s->soft())
                e = launch_tune_stream_lj(s->dim, dj, 1, s->stream);
            else if (s->polygon())
                e = launch_tune_stream_poly2(s->sat(), dj, 1, s->verts, s->n_vertices, s->poly_rcut2, s->stream);
            else if (s->oriented())
                e = launch_tune_stream_poly(dj, 1, s->verts, s->n_vertices, s->poly_rcut2, s->stream);
            else
                e = launch_tune_stream_sphere(s->dim, dj, 1, s->stream);
            s->prof.kernel_launches += 1;
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(&job, dj, sizeof(TuneJob), cudaMemcpyDeviceToHost, s->stream);
        if (dj) cudaFreeAsync(dj, s->stream);
        cudaError_t e2 = cudaStreamSynchronize(s->stream);
        if (e == cudaSuccess) e = e2;
        if (e != cudaSuccess) return fail(HMC_CUDA_ERROR, "tune: %s", cudaGetErrorString(e));
        if ((st = read_stats(s))) return st;
        if ((st = check_flags(s))) return st;
        p->maximum = job.maximum;
        return HMC_OK;
    }
    double lmax = 0.0;
    for (int a = 0; a < s->dim; ++a) lmax = std::max(lmax, s->geom.L[a]);
    uint64_t* db = nullptr;
    double4 *dt = nullptr, *dq = nullptr;
    double *du = nullptr, *dh = nullptr;
    uint8_t* dd = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&db, sizeof(uint64_t) * samples, s->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dt, sizeof(double4) * samples, s->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dq, sizeof(double4) * samples, s->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&du, sizeof(double) * samples, s->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dh, sizeof(double) * samples, s->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dd, 2 * (size_t)samples, s->stream);
    std::vector<uint8_t> hd(samples);
    const bool fp32 = p->precision == HMC_FP32_RECHECK;
    for (uint32_t step = 0; step < steps && e == cudaSuccess; ++step) {
        if (p->maximum > 4.0 * lmax) p->maximum = 4.0 * lmax;  // the samplers' bound (see hmc_sweep)
        Launch L{};
        L.step = s->step;
        L.substep = s->substep;
        L.seed = s->seed;
        L.max_move = p->maximum;
        L.kt = p->temperature;
        L.n_bodies = (uint32_t)s->n;
        e = launch_tune_moves(s->dim, s->geom, s->arr, L, step, samples, p->move == HMC_ROTATE, db, dt, dq, du, s->stream);
        if (e != cudaSuccess) break;
        if (s->soft())
            e = launch_eval_lj(s->dim, fp32 && s->soft_fp32(), s->geom, s->arr, s->pair, db, dt, du, p->temperature,
                               samples, dd, dd + samples, dh, s->stream);
        else if (s->polygon())
            e = launch_eval_poly2(fp32, s->sat(), s->geom, s->arr, s->verts, s->n_vertices, s->poly_rcut2,
                                  s->poly_rcut2_hi32, db, dt, dq, samples, dd, s->stream);
        else if (s->oriented())
            e = launch_eval_poly(fp32, s->geom, s->arr, s->verts, s->n_vertices, s->poly_rcut2, s->poly_rcut2_hi32, db,
                                 dt, dq, samples, dd, s->stream);
        else
            e = launch_eval_sphere(s->dim, fp32, s->geom, s->arr, s->pair, db, dt, samples, dd, dd + samples, s->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hd.data(), dd, samples, cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) break;
        s->prof.kernel_launches += 2;
        uint64_t acc = 0;
        for (uint32_t j = 0; j < samples; ++j) acc += hd[j];
        const double ratio = (double)acc / (double)samples;
        p->maximum *= (ratio + 1.5) / (target + 1.5);
    }
    if (db) cudaFreeAsync(db, s->stream);
    if (dt) cudaFreeAsync(dt, s->stream);
    if (dq) cudaFreeAsync(dq, s->stream);
    if (du) cudaFreeAsync(du, s->stream);
    if (dh) cudaFreeAsync(dh, s->stream);
    if (dd) cudaFreeAsync(dd, s->stream);
    cudaError_t e2 = cudaStreamSynchronize(s->stream);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return fail(HMC_CUDA_ERROR, "tune: %s", cudaGetErrorString(e));
    if ((st = read_stats(s))) return st;
    return check_flags(s);
}

hmc_status hmc_overlap_check(hmc_system* s, uint64_t* n_overlaps) {
    if (!s || !n_overlaps) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (s->interaction == HMC_LENNARD_JONES || s->interaction == HMC_ISOTROPIC)
        return fail(HMC_NOT_SUPPORTED, "overlap check of a soft potential");
    // overlap penalty: pairs closer than delta (those with a positive pair energy)
    HMC_CUDA(cudaSetDevice(s->ctx->device));
    hmc_status st = rebuild(s, true);
    if (st) return st;
    if (s->interaction == HMC_HARD_CONVEX_POLYHEDRON)
        HMC_CUDA(launch_overlap_poly(s->geom, s->arr, s->verts, s->n_vertices, s->poly_rcut2, (uint32_t)s->n, s->stream));
    else if (s->polygon())
        HMC_CUDA(launch_overlap_poly2(s->sat(), s->geom, s->arr, s->verts, s->n_vertices, s->poly_rcut2, (uint32_t)s->n,
                                      s->stream));
    else
        HMC_CUDA(launch_overlap_sphere(s->dim, s->geom, s->arr, s->pair, (uint32_t)s->n, s->stream));
    s->prof.kernel_launches += 1;
    if ((st = read_stats(s))) return st;
    if ((st = check_flags(s))) return st;
    *n_overlaps = s->host_stats->overlaps;
    return HMC_OK;
}

// Pair histogram on a checkerboard at least `reach` wide (so the 3^d stencil holds every pair
// binned); the next sweep rebuilds its own checkerboard.
static hmc_status pair_histogram(hmc_system* s, bool sdf, double sigma, double limit, double reach, uint32_t n_bins,
                                 uint64_t* counts) {
    if (!counts || n_bins == 0 || n_bins > 8192) return fail(HMC_INVALID_ARGUMENT, "1 to 8192 bins");
    if (!(limit > 0.0) || !std::isfinite(limit)) return fail(HMC_INVALID_ARGUMENT, "the histogram range must be positive");
    HMC_CUDA(cudaSetDevice(s->ctx->device));
    Geometry g = s->geom;
    const double range = std::max(reach, s->body_range);
    if (!compute_dimensions(s->dim, g.L, range, g.width, g.shape))
        return fail(HMC_RANGE_TOO_LARGE, "a histogram reaching %g needs at least two spaces of that width per axis", range);
    uint64_t cells = 1;
    g.any_two = 0;
    for (int a = 0; a < s->dim; ++a) {
        g.w32[a] = (float)g.width[a];
        g.invW[a] = 1.0 / g.width[a];
        g.half_shape[a] = g.shape[a] / 2;
        if (g.shape[a] == 2) g.any_two = 1;
        g.origin[a] = -g.L[a] / 2.0;
        cells *= g.shape[a];
    }
    g.n_cells = (uint32_t)cells;  // no more than the system's own spaces: these are wider
    g.color_stride = (uint32_t)(cells >> s->dim);
    HMC_CUDA(cudaMemsetAsync(s->arr.stats, 0, sizeof(DeviceStats), s->stream));
    HMC_CUDA(launch_rebuild(s->dim, g, s->arr, (uint32_t)s->n, true, s->stream));
    unsigned long long* d = nullptr;
    HMC_CUDA(cudaMallocAsync((void**)&d, sizeof(unsigned long long) * n_bins, s->stream));
    cudaError_t e = launch_pair_histogram(s->dim, sdf, g, s->arr, (uint32_t)s->n, sigma, limit, (double)n_bins / limit,
                                          n_bins, d, s->stream);
    std::vector<unsigned long long> h(n_bins);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), d, sizeof(unsigned long long) * n_bins, cudaMemcpyDeviceToHost, s->stream);
    cudaFreeAsync(d, s->stream);
    cudaError_t e2 = cudaStreamSynchronize(s->stream);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return fail(HMC_CUDA_ERROR, "pair histogram: %s", cudaGetErrorString(e));
    s->prof.kernel_launches += s->n > 0 ? 7 : 2;  // the rebuild and the histogram
    hmc_status st;
    if ((st = read_stats(s))) return st;
    if ((st = check_flags(s))) return st;
    for (uint32_t b = 0; b < n_bins; ++b) counts[b] = h[b];
    return HMC_OK;
}

hmc_status hmc_sdf(hmc_system* s, double x_max, uint32_t n_bins, uint64_t* counts) {
    if (!s) return fail(HMC_INVALID_ARGUMENT, "NULL system");
    if (s->interaction != HMC_HARD_SPHERE) return fail(HMC_NOT_SUPPORTED, "the scale distribution is for hard spheres");
    if (!(x_max > 0.0 && x_max < 0.5)) return fail(HMC_INVALID_ARGUMENT, "x_max must be in (0, 0.5)");
    const double sigma = std::sqrt(s->pair.sigma2);
    return pair_histogram(s, true, sigma, x_max, sigma / (1.0 - x_max), n_bins, counts);
}

hmc_status hmc_gr(hmc_system* s, double r_max, uint32_t n_bins, uint64_t* counts) {
    if (!s) return fail(HMC_INVALID_ARGUMENT, "NULL system");
    return pair_histogram(s, false, 0.0, r_max, r_max, n_bins, counts);
}

hmc_status hmc_total_energy(hmc_system* s, double* energy) {
    if (!s || !energy) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (s->shape_soft) {
        HMC_CUDA(cudaSetDevice(s->ctx->device));
        hmc_status st = rebuild(s, true);
        if (st) return st;
        double* d = reinterpret_cast<double*>(&s->arr.stats->overlaps);  // 8 zeroed bytes after the rebuild
        if (s->dim == 3)
            HMC_CUDA(launch_energy_poly3_soft(s->geom, s->arr, s->verts, s->n_vertices, s->so, (uint32_t)s->n, d,
                                              s->stream));
        else
            HMC_CUDA(launch_energy_poly2_soft(s->sat(), s->geom, s->arr, s->verts, s->n_vertices, s->so,
                                              (uint32_t)s->n, d, s->stream));
        s->prof.kernel_launches += 1;
        if ((st = read_stats(s))) return st;
        if ((st = check_flags(s))) return st;
        std::memcpy(energy, &s->host_stats->overlaps, sizeof(double));
        return HMC_OK;
    }
    if (!s->soft()) {
        uint64_t n = 0;
        hmc_status st = hmc_overlap_check(s, &n);
        if (st) return st;
        *energy = n > 0 ? INFINITY : 0.0;
        return HMC_OK;
    }
    HMC_CUDA(cudaSetDevice(s->ctx->device));
    hmc_status st = rebuild(s, true);
    if (st) return st;
    double* d = reinterpret_cast<double*>(&s->arr.stats->overlaps);  // 8 zeroed bytes after the rebuild
    HMC_CUDA(launch_energy_lj(s->dim, s->geom, s->arr, s->pair, (uint32_t)s->n, d, s->stream));
    s->prof.kernel_launches += 1;
    if ((st = read_stats(s))) return st;
    if ((st = check_flags(s))) return st;
    std::memcpy(energy, &s->host_stats->overlaps, sizeof(double));
    return HMC_OK;
}

hmc_status hmc_get_box(hmc_system* s, double* edge_lengths) {
    if (!s || !edge_lengths) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    for (int a = 0; a < s->dim; ++a) edge_lengths[a] = s->geom.L[a];
    return HMC_OK;
}

hmc_status hmc_get_n_bodies(hmc_system* s, uint64_t* n_bodies) {
    if (!s || !n_bodies) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    *n_bodies = s->n;
    return HMC_OK;
}

// clone_with_boundary onto the box L: the positions are kept in `backup` (restore_box puts
// them and the old box back), mapped on the device, and the checkerboard is laid out again.
static hmc_status restore_box(hmc_system* s, const double* L_old) {
    if (s->n)
        HMC_CUDA(cudaMemcpyAsync(s->arr.body_pos, s->backup, sizeof(double4) * s->n, cudaMemcpyDeviceToDevice,
                                 s->stream));
    return setup_geometry(s, L_old);
}

static hmc_status map_into_box(hmc_system* s, const double* L) {
    double L_old[3] = {s->geom.L[0], s->geom.L[1], s->geom.L[2]};
    if (!s->backup) {
        hmc_status st = dalloc(s, &s->backup, s->capacity);
        if (st) return st;
    }
    if (s->n)
        HMC_CUDA(cudaMemcpyAsync(s->backup, s->arr.body_pos, sizeof(double4) * s->n, cudaMemcpyDeviceToDevice,
                                 s->stream));
    double old_half[3] = {0, 0, 0}, scale[3] = {1, 1, 1}, lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int a = 0; a < s->dim; ++a) {
        old_half[a] = L_old[a] / 2.0;
        scale[a] = L[a] / L_old[a];
        lo[a] = -L[a] / 2.0;
        hi[a] = std::nextafter(L[a] / 2.0, -INFINITY);  // f64::next_down
    }
    hmc_status st = setup_geometry(s, L);
    if (st) return st;
    const unsigned long long none = ~0ull;
    HMC_CUDA(cudaMemcpyAsync(s->first_bad, &none, sizeof(none), cudaMemcpyHostToDevice, s->stream));
    HMC_CUDA(launch_map_bodies(s->dim, s->geom, old_half, scale, lo, hi, s->arr.body_pos, s->n, s->first_bad,
                               s->stream));
    s->prof.kernel_launches += 1;
    HMC_CUDA(cudaMemcpyAsync(s->host_first_bad, s->first_bad, sizeof(none), cudaMemcpyDeviceToHost, s->stream));
    HMC_CUDA(cudaStreamSynchronize(s->stream));
    if (*s->host_first_bad != none) {
        const unsigned long long bad = *s->host_first_bad;
        restore_box(s, L_old);
        return fail(HMC_INVALID_ARGUMENT, "body %llu is outside the box (map_point)", bad);
    }
    return HMC_OK;
}

hmc_status hmc_set_shape_overlap(hmc_system* s, const hmc_shape_overlap_params* p) {
    if (!s) return fail(HMC_INVALID_ARGUMENT, "NULL system");
    if (!p) {
        s->shape_soft = false;
        return HMC_OK;
    }
    if (p->struct_size < sizeof(hmc_shape_overlap_params))
        return fail(HMC_INVALID_ARGUMENT, "hmc_shape_overlap_params.struct_size");
    if (!s->oriented())
        return fail(HMC_NOT_SUPPORTED, "the approximate shape overlap is for convex polyhedra and polygons");
    if (!(p->resolution > 0.0) || !std::isfinite(p->resolution))
        return fail(HMC_INVALID_ARGUMENT, "resolution must be positive");
    if (!(p->penalty_k >= 0.0) || !std::isfinite(p->penalty_k) || !(p->penalty_maximum_overlap >= 0.0) ||
        !std::isfinite(p->penalty_maximum_overlap) || !std::isfinite(p->penalty_shoulder))
        return fail(HMC_INVALID_ARGUMENT, "overlap penalty k and maximum overlap must be finite and >= 0");
    const double range = s->pair_range;  // R + R of the shape's bounding sphere
    const double rcut = p->r_cut > 0.0 ? p->r_cut : range;
    // every candidate lies in the 3^d spaces around the site only up to the pair range
    if (!(rcut <= range)) return fail(HMC_NOT_SUPPORTED, "r_cut %g beyond the shape's range %g", rcut, range);
    // A pair closer than r_cut <= R + R separates within (R + R) / resolution steps, since
    // |v + direction * d| = |v| + d up to rounding; the device loop stops at this bound.
    const double steps = std::ceil(range / p->resolution) + 8.0;
    if (!(steps <= 4194304.0))
        return fail(HMC_INVALID_ARGUMENT, "resolution %g takes more than 2^22 steps over the range %g", p->resolution,
                    range);
    ShapeOverlap& so = s->so;
    so.resolution = p->resolution;
    so.rcut = rcut;
    so.rr = s->poly_rcut2;
    so.dmax = p->penalty_maximum_overlap;
    so.half_k = 0.5 * p->penalty_k;
    so.shoulder = p->penalty_shoulder;
    so.max_steps = (uint32_t)steps;
    s->shape_soft = true;
    return HMC_OK;
}

hmc_status hmc_set_box(hmc_system* s, const double* edge_lengths) {
    if (!s || !edge_lengths) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    HMC_CUDA(cudaSetDevice(s->ctx->device));
    return map_into_box(s, edge_lengths);
}

// Body tags on the device: identity for the bodies present when first needed.
static hmc_status body_tags(hmc_system* s, BodyTags* out) {
    if (!s->tags) {
        hmc_status st;
        if ((st = dalloc(s, &s->tags, s->capacity)) || (st = dalloc(s, &s->tag_heap, s->capacity)) ||
            (st = dalloc(s, &s->tag_meta, 2)))
            return st;
        std::vector<uint32_t> id(std::max<uint64_t>(s->n, 1));
        for (uint64_t i = 0; i < s->n; ++i) id[i] = (uint32_t)i;
        if (s->n) HMC_CUDA(cudaMemcpy(s->tags, id.data(), sizeof(uint32_t) * s->n, cudaMemcpyHostToDevice));
        const uint32_t meta[2] = {0u, (uint32_t)s->n};
        HMC_CUDA(cudaMemcpy(s->tag_meta, meta, sizeof(meta), cudaMemcpyHostToDevice));
    }
    *out = BodyTags{s->tags, s->tag_heap, s->tag_meta};
    return HMC_OK;
}

hmc_status hmc_quick_insert_apply(hmc_system* s, hmc_quick_insert* qi, hmc_count* out) {
    if (!s || !qi) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (s->interaction != HMC_HARD_SPHERE && !s->penalty() && !s->shape_soft)
        return fail(HMC_NOT_SUPPORTED, "QuickInsert places hard or overlap-penalty spheres, or convex shapes "
                                       "under the approximate shape overlap");
    if (qi->allowed_overlaps == 0) return fail(HMC_INVALID_ARGUMENT, "allowed_overlaps must be >= 1");
    if (qi->inserted > qi->target) return fail(HMC_INVALID_ARGUMENT, "inserted exceeds target");
    if (s->n + (qi->target - qi->inserted) > s->capacity)
        return fail(HMC_INVALID_ARGUMENT, "the system holds %llu bodies; %llu more do not fit",
                    (unsigned long long)s->capacity, (unsigned long long)(qi->target - qi->inserted));
    hmc_count count{};
    if (out) *out = count;
    if (qi->complete) return HMC_OK;
    HMC_CUDA(cudaSetDevice(s->ctx->device));
    double energy = 0.0;
    hmc_status st = hmc_total_energy(s, &energy);
    if (st) return st;
    if (energy <= 0.0 && qi->inserted >= qi->target) {
        qi->complete = 1;
        return HMC_OK;
    }
    if (energy <= 0.0) {
        if ((st = serial_grid(s))) return st;
        if (!s->qi_out && (st = dalloc(s, &s->qi_out, 8))) return st;
        Launch L{};
        L.step = s->step;
        L.substep = s->substep;
        L.seed = s->seed;
        L.n_bodies = (uint32_t)s->n;
        QuickInsertArgs q{};
        q.n0 = (uint32_t)s->n;
        q.capacity = (uint32_t)s->capacity;
        q.attempts = qi->target;
        q.to_insert = qi->target - qi->inserted;
        q.allowed = qi->allowed_overlaps;
        q.soft = s->penalty() ? 1u : 0u;
        for (int a = 0; a < 3; ++a) {
            // Uniform::new(minimal, maximal extent): low = -L/2, scale = L/2 - (-L/2)
            const double low = a < s->dim ? -s->geom.L[a] / 2.0 : 0.0, high = a < s->dim ? s->geom.L[a] / 2.0 : 0.0;
            q.low[a] = low;
            q.scale[a] = high - low;
        }
        HMC_CUDA(cudaMemsetAsync(s->arr.stats, 0, sizeof(DeviceStats), s->stream));
        BodyTags tags;
        if ((st = body_tags(s, &tags))) return st;
        if (s->shape_soft && s->dim == 3)
            HMC_CUDA(launch_quick_insert_poly3(s->geom, s->arr, s->verts, s->n_vertices, s->so, L, q, tags,
                                               s->serial_nc, s->serial_w, s->serial_cap, s->serial_size,
                                               s->serial_items, s->serial_cell_of, s->serial_site, s->qi_out,
                                               s->stream));
        else if (s->shape_soft)
            HMC_CUDA(launch_quick_insert_poly2(s->sat(), s->geom, s->arr, s->verts, s->n_vertices, s->so, L, q, tags,
                                               s->serial_nc, s->serial_w, s->serial_cap, s->serial_size,
                                               s->serial_items, s->serial_cell_of, s->serial_site, s->qi_out,
                                               s->stream));
        else
            HMC_CUDA(launch_quick_insert(s->dim, s->geom, s->arr, s->pair, L, q, tags, s->serial_nc, s->serial_w,
                                         s->serial_cap, s->serial_size, s->serial_items, s->serial_cell_of,
                                         s->serial_site, s->qi_out, s->stream));
        s->prof.kernel_launches += 2;
        unsigned long long r[4] = {0, 0, 0, 0};
        HMC_CUDA(cudaMemcpyAsync(r, s->qi_out, sizeof(r), cudaMemcpyDeviceToHost, s->stream));
        if ((st = read_stats(s))) return st;
        if ((st = check_flags(s))) return st;
        s->n = r[3];
        qi->inserted += r[0];
        count.accepted = r[0];
        count.rejected = r[2];
    }
    s->substep += 1;  // increment_substep (quick_insert.rs:278)
    if (out) *out = count;
    return HMC_OK;
}

hmc_status hmc_grand_canonical_apply(hmc_system* s, const hmc_grand_canonical_params* p,
                                     hmc_insert_remove_count* out) {
    if (!s || !p) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (s->interaction != HMC_HARD_SPHERE && !s->penalty())
        return fail(HMC_NOT_SUPPORTED, "GrandCanonical inserts and removes hard or overlap-penalty spheres");
    if (!(p->temperature > 0.0)) return fail(HMC_INVALID_ARGUMENT, "temperature must be positive");
    if (!std::isfinite(p->fugacity)) return fail(HMC_INVALID_ARGUMENT, "fugacity must be finite");
    hmc_insert_remove_count count{};
    if (out) *out = count;
    if (p->n_trials == 0) return HMC_OK;
    HMC_CUDA(cudaSetDevice(s->ctx->device));
    hmc_status st;
    if ((st = serial_grid(s))) return st;
    if (!s->qi_out && (st = dalloc(s, &s->qi_out, 8))) return st;
    BodyTags tags;
    if ((st = body_tags(s, &tags))) return st;
    GrandCanonicalArgs q{};
    q.step = s->step;
    q.substep = s->substep;
    q.seed = s->seed;
    q.n_trials = p->n_trials;
    q.n0 = (uint32_t)s->n;
    q.capacity = (uint32_t)s->capacity;
    q.soft = s->penalty() ? 1u : 0u;
    q.temperature = p->temperature;
    q.fugacity = p->fugacity;
    double volume = s->geom.L[0];
    for (int a = 1; a < s->dim; ++a) volume = volume * s->geom.L[a];  // Hypercuboid::volume
    q.volume = volume;
    for (int a = 0; a < 3; ++a) {
        const double low = a < s->dim ? -s->geom.L[a] / 2.0 : 0.0, high = a < s->dim ? s->geom.L[a] / 2.0 : 0.0;
        q.low[a] = low;
        q.scale[a] = high - low;
    }
    HMC_CUDA(cudaMemsetAsync(s->arr.stats, 0, sizeof(DeviceStats), s->stream));
    HMC_CUDA(launch_grand_canonical(s->dim, s->geom, s->arr, s->pair, q, tags, s->serial_nc, s->serial_w, s->serial_cap,
                                    s->serial_size, s->serial_items, s->serial_cell_of, s->serial_site, s->qi_out,
                                    s->stream));
    s->prof.kernel_launches += 2;
    unsigned long long r[5] = {0, 0, 0, 0, 0};
    HMC_CUDA(cudaMemcpyAsync(r, s->qi_out, sizeof(r), cudaMemcpyDeviceToHost, s->stream));
    if ((st = read_stats(s))) return st;
    if ((st = check_flags(s))) return st;
    s->n = r[4];
    if (r[2]) s->tags_permuted = true;
    s->substep += p->n_trials;  // one increment_substep per apply
    count.insert_accepted = r[0];
    count.insert_rejected = r[1];
    count.remove_accepted = r[2];
    count.remove_rejected = r[3];
    if (out) *out = count;
    return HMC_OK;
}

hmc_status hmc_quick_compress_apply(hmc_system* s, hmc_quick_compress* qc) {
    if (!s || !qc) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (!(qc->target_volume > 0.0) || !std::isfinite(qc->target_volume))
        return fail(HMC_INVALID_ARGUMENT, "target volume must be positive");
    if (!(qc->maximum_delta > 0.0 && qc->maximum_delta < 1.0))
        return fail(HMC_INVALID_ARGUMENT, "maximum_delta must be in (0, 1)");
    if (qc->state > HMC_QC_COMPLETE) return fail(HMC_INVALID_ARGUMENT, "state");
    HMC_CUDA(cudaSetDevice(s->ctx->device));
    Sfc64 rng = make_rng(s->step, s->substep, s->seed, 0);  // microstate.counter().make_rng()
    s->substep += 1;
    double L[3] = {s->geom.L[0], s->geom.L[1], s->geom.L[2]};
    auto same_box = [&](const double* b) {
        for (int a = 0; a < s->dim; ++a)
            if (b[a] != L[a]) return false;
        return true;
    };
    auto wait_on = [&](bool is_final, const double* b) {
        qc->state = HMC_QC_WAITING;
        qc->is_final = is_final ? 1u : 0u;
        for (int a = 0; a < 3; ++a) qc->boundary[a] = a < s->dim ? b[a] : 0.0;
    };
    hmc_status st = HMC_OK;
    switch (qc->state) {
        case HMC_QC_STARTUP:
            wait_on(false, L);
            break;
        case HMC_QC_COMPLETE:
            if (!same_box(qc->boundary)) wait_on(false, L);
            break;
        case HMC_QC_COMPRESSING: {
            // Uniform::new(0.0, maximum_delta).sample(rng)
            const double u = as_double(0x3FF0000000000000ULL | (rng.next_u64() >> 12)) - 1.0;
            const double delta = u * (qc->maximum_delta - 0.0) + 0.0;
            double volume = L[0];
            for (int a = 1; a < s->dim; ++a) volume = volume * L[a];  // Hypercuboid::volume
            const double trial_volume = qc->target_volume > volume ? std::min(volume * (1.0 + delta), qc->target_volume)
                                                                   : std::max(volume * (1.0 - delta), qc->target_volume);
            // scale_volume: edge lengths times (V'/V)^(1/N) (cuboid.rs:483-517)
            const double v = std::pow(trial_volume / volume, 1.0 / (double)s->dim);
            double L_new[3] = {L[0], L[1], L[2]};
            for (int a = 0; a < s->dim; ++a) L_new[a] = L[a] * v;
            double e0 = 0.0, e1 = 0.0;
            if ((st = hmc_total_energy(s, &e0))) return st;
            if ((st = map_into_box(s, L_new))) return st;
            if ((st = hmc_total_energy(s, &e1))) return st;
            const double delta_energy = e1 - e0;  // delta_energy_total
            if (delta_energy > qc->maximum_energy_per_site * (double)s->n) {
                if ((st = restore_box(s, L))) return st;  // too strained: stay Compressing
            } else {
                wait_on(trial_volume == qc->target_volume, L_new);
            }
            break;
        }
        case HMC_QC_WAITING: {
            double e = 0.0;
            if ((st = hmc_total_energy(s, &e))) return st;
            if (e <= 0.0) {
                if (qc->is_final && same_box(qc->boundary)) {
                    qc->state = HMC_QC_COMPLETE;
                    for (int a = 0; a < 3; ++a) qc->boundary[a] = a < s->dim ? L[a] : 0.0;
                } else {
                    qc->state = HMC_QC_COMPRESSING;
                }
            }
            break;
        }
    }
    return HMC_OK;
}

hmc_status hmc_eval_moves(hmc_system* s, const hmc_injected_move* moves, uint64_t n, double temperature,
                          uint32_t precision, uint8_t* decisions, uint8_t* rechecked, double* delta_h) {
    if (!s || (n && (!moves || !decisions))) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (s->shape_soft)
        return fail(HMC_NOT_SUPPORTED, "hmc_eval_moves runs under HardShape: hmc_set_shape_overlap(s, NULL) first");
    if (precision > HMC_FP32_RECHECK) return fail(HMC_INVALID_ARGUMENT, "precision");
    if (s->soft() && !(temperature > 0.0))
        return fail(HMC_INVALID_ARGUMENT, "temperature must be positive");
    if (n == 0) return HMC_OK;
    if (n >= (1ull << 31)) return fail(HMC_INVALID_ARGUMENT, "too many moves");
    HMC_CUDA(cudaSetDevice(s->ctx->device));
    for (uint64_t i = 0; i < n; ++i)
        if (moves[i].body >= s->n) return fail(HMC_INVALID_ARGUMENT, "move %llu names body %llu of %llu",
                                                (unsigned long long)i, (unsigned long long)moves[i].body,
                                                (unsigned long long)s->n);
    hmc_status st = rebuild(s, true);
    if (st) return st;
    std::vector<uint64_t> hb(n);
    std::vector<double4> ht(n);
    std::vector<double> hu(n);
    std::vector<double4> hq(n);
    for (uint64_t i = 0; i < n; ++i) {
        hb[i] = moves[i].body;
        ht[i] = make_double4(moves[i].position[0], moves[i].position[1], s->dim == 3 ? moves[i].position[2] : 0.0, 0.0);
        hu[i] = moves[i].u;
        hq[i] = make_double4(moves[i].orientation[0], moves[i].orientation[1], moves[i].orientation[2],
                             moves[i].orientation[3]);
    }
    const bool lj = s->soft();
    uint64_t* db = nullptr;
    double4* dt = nullptr;
    double* du = nullptr;
    double* dh = nullptr;
    uint8_t* dd = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&db, sizeof(uint64_t) * n, s->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dt, sizeof(double4) * n, s->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&du, sizeof(double) * n, s->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dh, sizeof(double) * n, s->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dd, 2 * n, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(db, hb.data(), sizeof(uint64_t) * n, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dt, ht.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(du, hu.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s->stream);
    double4* dq = nullptr;
    if (e == cudaSuccess && s->oriented()) {
        e = cudaMallocAsync((void**)&dq, sizeof(double4) * n, s->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dq, hq.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, s->stream);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(dh, 0, sizeof(double) * n, s->stream);
    if (e == cudaSuccess) {
        if (lj)
            e = launch_eval_lj(s->dim, precision == HMC_FP32_RECHECK && s->soft_fp32(), s->geom, s->arr, s->pair, db, dt, du, temperature,
                               (uint32_t)n, dd, dd + n, dh, s->stream);
        else if (s->polygon())
            e = launch_eval_poly2(precision == HMC_FP32_RECHECK, s->sat(), s->geom, s->arr, s->verts, s->n_vertices,
                                  s->poly_rcut2, s->poly_rcut2_hi32, db, dt, dq, (uint32_t)n, dd, s->stream);
        else if (s->oriented())
            e = launch_eval_poly(precision == HMC_FP32_RECHECK, s->geom, s->arr, s->verts, s->n_vertices, s->poly_rcut2,
                                 s->poly_rcut2_hi32, db, dt, dq, (uint32_t)n, dd, s->stream);
        else
            e = launch_eval_sphere(s->dim, precision == HMC_FP32_RECHECK, s->geom, s->arr, s->pair, db, dt,
                                   (uint32_t)n, dd, dd + n, s->stream);
    }
    std::vector<uint8_t> hd(2 * n);
    std::vector<double> hh(n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hd.data(), dd, 2 * n, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hh.data(), dh, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream);
    if (db) cudaFreeAsync(db, s->stream);
    if (dt) cudaFreeAsync(dt, s->stream);
    if (du) cudaFreeAsync(du, s->stream);
    if (dh) cudaFreeAsync(dh, s->stream);
    if (dd) cudaFreeAsync(dd, s->stream);
    if (dq) cudaFreeAsync(dq, s->stream);
    cudaError_t e2 = cudaStreamSynchronize(s->stream);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return fail(HMC_CUDA_ERROR, "eval_moves: %s", cudaGetErrorString(e));
    if ((st = read_stats(s))) return st;
    if ((st = check_flags(s))) return st;
    std::memcpy(decisions, hd.data(), n);
    if (rechecked) std::memcpy(rechecked, hd.data() + n, n);
    if (delta_h) {
        if (lj) {
            std::memcpy(delta_h, hh.data(), sizeof(double) * n);
        } else {
            for (uint64_t i = 0; i < n; ++i) delta_h[i] = hd[i] ? 0.0 : INFINITY;
        }
    }
    return HMC_OK;
}

hmc_status hmc_eval_trials(hmc_system* s, const hmc_injected_move* moves, uint64_t n, double temperature,
                           uint32_t precision, uint8_t* decisions, uint8_t* flags) {
    if (!s || (n && (!moves || !decisions))) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (s->shape_soft)
        return fail(HMC_NOT_SUPPORTED, "hmc_eval_trials runs under HardShape: hmc_set_shape_overlap(s, NULL) first");
    if (precision > HMC_FP32_RECHECK) return fail(HMC_INVALID_ARGUMENT, "precision");
    if (s->polygon()) return fail(HMC_NOT_SUPPORTED, "eval_trials: convex polygons");
    if (s->soft() && !(temperature > 0.0)) return fail(HMC_INVALID_ARGUMENT, "temperature must be positive");
    if (n == 0) return HMC_OK;
    if (n >= (1ull << 31)) return fail(HMC_INVALID_ARGUMENT, "too many moves");
    HMC_CUDA(cudaSetDevice(s->ctx->device));
    for (uint64_t i = 0; i < n; ++i)
        if (moves[i].body >= s->n) return fail(HMC_INVALID_ARGUMENT, "move %llu names body %llu of %llu",
                                                (unsigned long long)i, (unsigned long long)moves[i].body,
                                                (unsigned long long)s->n);
    hmc_status st = rebuild(s, true);
    if (st) return st;
    std::vector<uint64_t> hb(n);
    std::vector<double4> ht(n), hq(n);
    std::vector<double> hu(n);
    for (uint64_t i = 0; i < n; ++i) {
        hb[i] = moves[i].body;
        ht[i] = make_double4(moves[i].position[0], moves[i].position[1], s->dim == 3 ? moves[i].position[2] : 0.0, 0.0);
        hq[i] = make_double4(moves[i].orientation[0], moves[i].orientation[1], moves[i].orientation[2],
                             moves[i].orientation[3]);
        hu[i] = moves[i].u;
    }
    const bool fp32 = precision == HMC_FP32_RECHECK;
    uint64_t* db = nullptr;
    double4* dt = nullptr;
    double4* dq = nullptr;
    double* du = nullptr;
    uint8_t* dd = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&db, sizeof(uint64_t) * n, s->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dt, sizeof(double4) * n, s->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dq, sizeof(double4) * n, s->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&du, sizeof(double) * n, s->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dd, 2 * n, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(db, hb.data(), sizeof(uint64_t) * n, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dt, ht.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dq, hq.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(du, hu.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(dd, 0, 2 * n, s->stream);
    if (e == cudaSuccess) {
        Injected j;
        j.bodies = db;
        j.trial = dt;
        j.trial_q = dq;
        j.u = du;
        j.decisions = dd;
        j.flags = dd + n;
        j.n = (uint32_t)n;
        if (s->soft())
            e = launch_trials_lj(s->dim, fp32 && s->soft_fp32(), s->geom, s->arr, s->pair, temperature, j, s->stream);
        else if (s->oriented())
            e = launch_trials_poly(fp32, s->geom, s->arr, s->verts, s->n_vertices, s->poly_rcut2, s->poly_rcut2_hi32, j,
                                   s->stream);
        else
            e = launch_trials_sphere(s->dim, fp32, coop_of(s, fp32), s->geom, s->arr, s->pair, j, s->stream);
        s->prof.kernel_launches++;
    }
    std::vector<uint8_t> hd(2 * n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hd.data(), dd, 2 * n, cudaMemcpyDeviceToHost, s->stream);
    for (void* p : {(void*)db, (void*)dt, (void*)dq, (void*)du, (void*)dd})
        if (p) cudaFreeAsync(p, s->stream);
    cudaError_t e2 = cudaStreamSynchronize(s->stream);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return fail(HMC_CUDA_ERROR, "eval_trials: %s", cudaGetErrorString(e));
    if ((st = read_stats(s))) return st;
    if ((st = check_flags(s))) return st;
    std::memcpy(decisions, hd.data(), n);
    if (flags) std::memcpy(flags, hd.data() + n, n);
    return HMC_OK;
}

}  // extern "C"

// ---- batches of independent hard-sphere replicas ------------------------------------------
// Every replica is a full system of its own (box, checkerboard, Counter); the batch only
// shares the device arrays and the launches, so each replica's trajectory equals that of an
// hmc_system built from the same description.
struct hmc_batch {
    hmc_context* ctx = nullptr;
    int dim = 3;
    uint32_t n_rep = 0;
    uint64_t n = 0;
    uint32_t cells = 0;
    std::vector<Replica> rep;          // host copies; uploaded through rep_pinned
    Replica* rep_pinned = nullptr;
    std::vector<uint32_t> cell_base;   // [R + 1]
    std::vector<uint32_t> body_base;   // [R + 1]
    Arrays arr{};
    Batch b{};
    double* stage = nullptr;
    unsigned long long* first_bad = nullptr;
    cudaStream_t stream = nullptr;
    DeviceStats* host_stats = nullptr;  // pinned
    unsigned long long* host_rep_u64 = nullptr;  // pinned [R]: accepted or overlaps
    unsigned int* host_nonempty = nullptr;       // pinned [R]
    unsigned long long* host_first_bad = nullptr;
    std::vector<void*> allocations;
    uint64_t kernel_launches = 0;
    int32_t variant[2] = {-1, -1};  // launch variant of the hard-sphere replica pass per precision
    uint32_t rounds_guess = 2;
    uint32_t interaction = HMC_HARD_SPHERE;  // the same for every replica
    std::vector<double> body_range;          // [R] ParallelSweep range of each replica
    // captured sweeps (hmc_batch_set_captured_sweeps): one sweep as a CUDA graph, built for a
    // precision, launch variant and increment_step (graph_key), launched once per sweep
    bool captured = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    uint32_t graph_key = UINT32_MAX;
    cudaStream_t body_stream = nullptr;             // captures the rounds loop's body
    uint32_t* round_dev = nullptr;                  // the colour set the captured passes run
    unsigned long long* rep_counts = nullptr;       // [2R] accepted, rejected per replica
    BatchSweepTotals* totals = nullptr;
    unsigned long long* host_rep_counts = nullptr;  // pinned [2R]
    BatchSweepTotals* host_totals = nullptr;        // pinned
};

namespace {

template <typename T>
hmc_status balloc(hmc_batch* bt, T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * count);
    if (e != cudaSuccess)
        return fail(e == cudaErrorMemoryAllocation ? HMC_OUT_OF_MEMORY : HMC_CUDA_ERROR, "cudaMalloc(%zu bytes): %s",
                    sizeof(T) * count, cudaGetErrorString(e));
    bt->allocations.push_back((void*)*p);
    return HMC_OK;
}

hmc_status batch_upload_replicas(hmc_batch* bt) {
    std::memcpy(bt->rep_pinned, bt->rep.data(), sizeof(Replica) * bt->n_rep);
    HMC_CUDA(cudaMemcpyAsync((void*)bt->b.rep, bt->rep_pinned, sizeof(Replica) * bt->n_rep, cudaMemcpyHostToDevice,
                             bt->stream));
    return HMC_OK;
}

// update_checkerboard for every replica (its own Counter), then the batched counting sort.
hmc_status batch_rebuild(hmc_batch* bt, bool write_s) {
    for (Replica& r : bt->rep) {
        Sfc64 rng = make_rng(r.step, r.substep, r.seed, UINT64_MAX);
        for (int a = 0; a < bt->dim; ++a) {
            double off = uniform01(rng);
            r.g.origin[a] = -r.g.L[a] / 2.0 - off * r.g.width[a];
        }
    }
    hmc_status st = batch_upload_replicas(bt);
    if (st) return st;
    HMC_CUDA(cudaMemsetAsync(bt->arr.stats, 0, sizeof(DeviceStats), bt->stream));
    HMC_CUDA(launch_rebuild_batch(bt->dim, bt->b, bt->arr, (uint32_t)bt->n, write_s, bt->stream));
    bt->kernel_launches += bt->n > 0 ? 6 : 2;  // bin, 2 scan passes, scatter, space sort, gather
    return HMC_OK;
}

// Stats, per-replica non-empty spaces and accepted moves to the host (one synchronisation).
hmc_status batch_read(hmc_batch* bt) {
    HMC_CUDA(cudaMemcpyAsync(bt->host_stats, bt->arr.stats, sizeof(DeviceStats), cudaMemcpyDeviceToHost, bt->stream));
    HMC_CUDA(cudaMemcpyAsync(bt->host_nonempty, bt->b.nonempty, sizeof(unsigned int) * bt->n_rep,
                             cudaMemcpyDeviceToHost, bt->stream));
    HMC_CUDA(cudaMemcpyAsync(bt->host_rep_u64, bt->b.accepted, sizeof(unsigned long long) * bt->n_rep,
                             cudaMemcpyDeviceToHost, bt->stream));
    HMC_CUDA(cudaStreamSynchronize(bt->stream));
    const uint32_t f = bt->host_stats->error_flags;
    if (f & kErrNonFinite) return fail(HMC_NAN_STATE, "a body position is not finite");
    if (f & kErrOutsideCheckerboard) return fail(HMC_OUTSIDE_CHECKERBOARD, "a body maps to no checkerboard space");
    return HMC_OK;
}

// The colour passes of one set of a batch sweep, every colour, on stream s.
hmc_status batch_enqueue_colours(hmc_batch* bt, bool fp32, uint32_t round, bool first, uint32_t variant,
                                 cudaStream_t s) {
    const uint32_t colors = 1u << bt->dim;
    for (uint32_t c = 0; c < colors; ++c) {
        const bool overlap = !first || c > 0, early = first && c == 0;
        if (bt->interaction == HMC_LENNARD_JONES)
            HMC_CUDA(launch_sweep_batch_lj(bt->dim, fp32, bt->b, bt->arr, c, round, bt->b.color_stride, overlap, early,
                                           s, variant));
        else
            HMC_CUDA(launch_sweep_batch(bt->dim, fp32, bt->b, bt->arr, c, round, bt->b.color_stride, overlap, early, s,
                                        variant));
    }
    return HMC_OK;
}

void batch_drop_graph(hmc_batch* bt) {
    if (bt->graph_exec) cudaGraphExecDestroy(bt->graph_exec);
    if (bt->graph) cudaGraphDestroy(bt->graph);
    bt->graph_exec = nullptr;
    bt->graph = nullptr;
    bt->graph_key = UINT32_MAX;
}

// One batch sweep as a CUDA graph, built by stream capture: every replica's origin from its
// Counter (k_batch_origins), the batched rebuild, the per-replica rounds, a while node whose body
// is one colour set (the passes read the set from round_dev; k_batch_round_next advances it and
// sets the condition), and the bookkeeping (k_batch_sweep_end). The graph reads and writes device
// memory only, so the sweeps of a call are launched back to back and the host waits once.
hmc_status batch_build_graph(hmc_batch* bt, bool fp32, uint32_t variant, bool increment_step) {
    batch_drop_graph(bt);
    if (!bt->body_stream) HMC_CUDA(cudaStreamCreateWithFlags(&bt->body_stream, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    HMC_CUDA(cudaGraphCreate(&g, 0));
    bt->graph = g;
    cudaGraphConditionalHandle h;
    HMC_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
    cudaStream_t cs = bt->stream;
    Replica* rep = const_cast<Replica*>(bt->b.rep);
    // an error inside a capture leaves the stream capturing: end it before returning
    auto capture = [&](cudaStream_t st, auto&& body) -> hmc_status {
        hmc_status r = body();
        cudaGraph_t out = nullptr;
        const cudaError_t e = cudaStreamEndCapture(st, &out);
        if (r != HMC_OK) return r;
        if (e != cudaSuccess) return fail(HMC_CUDA_ERROR, "captured sweep: %s", cudaGetErrorString(e));
        return HMC_OK;
    };
    HMC_CUDA(cudaStreamBeginCaptureToGraph(cs, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    hmc_status st = capture(cs, [&]() -> hmc_status {
        HMC_CUDA(cudaMemsetAsync(bt->arr.stats, 0, sizeof(DeviceStats), cs));
        HMC_CUDA(launch_batch_origins(bt->dim, bt->b, rep, cs));
        HMC_CUDA(launch_rebuild_batch(bt->dim, bt->b, bt->arr, (uint32_t)bt->n, !fp32, cs));
        HMC_CUDA(launch_batch_rounds(bt->b, rep, bt->arr.stats, cs));
        HMC_CUDA(cudaMemsetAsync(bt->b.accepted, 0, sizeof(unsigned long long) * bt->n_rep, cs));
        HMC_CUDA(launch_batch_round_first(h, bt->arr.stats, bt->round_dev, bt->totals, cs));
        // the rounds loop
        cudaStreamCaptureStatus cst;
        cudaGraph_t cg = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t n_deps = 0;
        HMC_CUDA(cudaStreamGetCaptureInfo(cs, &cst, nullptr, &cg, &deps, &n_deps));
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t loop;
        HMC_CUDA(cudaGraphAddNode(&loop, cg, deps, n_deps, &cp));
        HMC_CUDA(cudaStreamUpdateCaptureDependencies(cs, &loop, 1, cudaStreamSetCaptureDependencies));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        HMC_CUDA(cudaStreamBeginCaptureToGraph(bt->body_stream, body, nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal));
        hmc_status sb = capture(bt->body_stream, [&]() -> hmc_status {
            hmc_status r = batch_enqueue_colours(bt, fp32, kRoundFromDevice, true, variant, bt->body_stream);
            if (r) return r;
            HMC_CUDA(launch_batch_round_next(h, bt->arr.stats, bt->round_dev, bt->body_stream));
            return HMC_OK;
        });
        if (sb) return sb;
        HMC_CUDA(launch_batch_sweep_end(bt->b, rep, bt->arr.stats, bt->rep_counts, bt->totals, increment_step, cs));
        return HMC_OK;
    });
    if (st) {
        batch_drop_graph(bt);
        return st;
    }
    cudaGraphExec_t x = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&x, g, 0);
    if (e != cudaSuccess) {
        batch_drop_graph(bt);
        return fail(HMC_CUDA_ERROR, "captured sweep: cudaGraphInstantiate: %s", cudaGetErrorString(e));
    }
    bt->graph_exec = x;
    bt->graph_key = (fp32 ? 1u : 0u) | (increment_step ? 2u : 0u) | (variant << 2);
    return HMC_OK;
}

// n_sweeps batch sweeps through the captured graph: the replica table up, one graph launch per
// sweep, then the counts, the statistics and the replica table (Counters, rounds) down with one
// wait. Decisions, counts and Counters equal the launched sweep's.
hmc_status batch_sweep_captured(hmc_batch* bt, const hmc_sweep_params& p0, bool fp32, uint32_t variant,
                                hmc_count* counts, hmc_count* total) {
    const uint32_t key = (fp32 ? 1u : 0u) | (p0.increment_step ? 2u : 0u) | (variant << 2);
    if (!bt->graph_exec || bt->graph_key != key) {
        hmc_status st = batch_build_graph(bt, fp32, variant, p0.increment_step != 0);
        if (st) return st;
    }
    hmc_status st = batch_upload_replicas(bt);
    if (st) return st;
    HMC_CUDA(cudaMemsetAsync(bt->rep_counts, 0, sizeof(unsigned long long) * 2 * bt->n_rep, bt->stream));
    HMC_CUDA(cudaMemsetAsync(bt->totals, 0, sizeof(BatchSweepTotals), bt->stream));
    for (uint32_t sweep = 0; sweep < p0.n_sweeps; ++sweep) HMC_CUDA(cudaGraphLaunch(bt->graph_exec, bt->stream));
    HMC_CUDA(cudaMemcpyAsync(bt->host_totals, bt->totals, sizeof(BatchSweepTotals), cudaMemcpyDeviceToHost,
                             bt->stream));
    HMC_CUDA(cudaMemcpyAsync(bt->host_rep_counts, bt->rep_counts, sizeof(unsigned long long) * 2 * bt->n_rep,
                             cudaMemcpyDeviceToHost, bt->stream));
    HMC_CUDA(cudaMemcpyAsync(bt->rep_pinned, bt->b.rep, sizeof(Replica) * bt->n_rep, cudaMemcpyDeviceToHost,
                             bt->stream));
    HMC_CUDA(cudaStreamSynchronize(bt->stream));
    std::memcpy(bt->rep.data(), bt->rep_pinned, sizeof(Replica) * bt->n_rep);
    const BatchSweepTotals& t = *bt->host_totals;
    // kernels: origins, the rebuild's six, rounds, the first test and the end per sweep; the
    // colour passes and the step per colour set
    const uint64_t per_sweep = bt->n > 0 ? 10 : 6;
    bt->kernel_launches += per_sweep * p0.n_sweeps + t.colour_sets * ((1u << bt->dim) + 1);
    const uint32_t f = t.error_flags;
    if (f & kErrNonFinite) return fail(HMC_NAN_STATE, "a body position is not finite");
    if (f & kErrOutsideCheckerboard) return fail(HMC_OUTSIDE_CHECKERBOARD, "a body maps to no checkerboard space");
    hmc_count tot{};
    for (uint32_t k = 0; k < bt->n_rep; ++k) {
        const uint64_t acc = bt->host_rep_counts[2 * k], rej = bt->host_rep_counts[2 * k + 1];
        if (counts) {
            counts[k].accepted += acc;
            counts[k].rejected += rej;
        }
        tot.accepted += acc;
        tot.rejected += rej;
    }
    tot.rechecks = t.rechecks;
    tot.pair_checks = t.pair_checks;
    tot.order_ambiguous = t.ambiguous;
    double me;
    unsigned long long bits = t.max_err_bits;
    std::memcpy(&me, &bits, 8);
    tot.max_fp32_error = me;
    if (total) *total = tot;
    return HMC_OK;
}

}  // namespace

extern "C" {

void hmc_batch_destroy(hmc_batch* bt) {
    if (!bt) return;
    cudaSetDevice(bt->ctx->device);
    if (bt->stream) cudaStreamSynchronize(bt->stream);
    for (void* p : bt->allocations) cudaFree(p);
    if (bt->rep_pinned) cudaFreeHost(bt->rep_pinned);
    if (bt->host_stats) cudaFreeHost(bt->host_stats);
    if (bt->host_rep_u64) cudaFreeHost(bt->host_rep_u64);
    if (bt->host_nonempty) cudaFreeHost(bt->host_nonempty);
    if (bt->host_first_bad) cudaFreeHost(bt->host_first_bad);
    if (bt->host_rep_counts) cudaFreeHost(bt->host_rep_counts);
    if (bt->host_totals) cudaFreeHost(bt->host_totals);
    if (bt->graph_exec) cudaGraphExecDestroy(bt->graph_exec);
    if (bt->graph) cudaGraphDestroy(bt->graph);
    if (bt->body_stream) cudaStreamDestroy(bt->body_stream);
    if (bt->stream) cudaStreamDestroy(bt->stream);
    cudaGetLastError();
    hmc_context* c = bt->ctx;
    delete bt;
    context_release(c);
}

hmc_status hmc_batch_create(hmc_context* ctx, uint32_t n_replicas, const hmc_system_desc* descs,
                            const double* const* positions, hmc_batch** out) {
    if (!ctx || !descs || !positions || !out) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    if (n_replicas == 0 || n_replicas > 65535) return fail(HMC_INVALID_ARGUMENT, "1 to 65535 replicas");
    const uint32_t dim = descs[0].dim;
    const uint32_t interaction = descs[0].interaction;
    const bool lj = interaction == HMC_LENNARD_JONES;
    uint64_t n_total = 0, cells_total = 0;
    std::vector<Replica> reps(n_replicas);
    for (uint32_t k = 0; k < n_replicas; ++k) {
        const hmc_system_desc* d = descs + k;
        if (d->struct_size < sizeof(hmc_system_desc)) return fail(HMC_INVALID_ARGUMENT, "replica %u: struct_size", k);
        if (d->dim != dim || (dim != 2 && dim != 3))
            return fail(HMC_INVALID_ARGUMENT, "replica %u: all replicas need the same dim, 2 or 3", k);
        if (d->interaction != HMC_HARD_SPHERE && d->interaction != HMC_LENNARD_JONES)
            return fail(HMC_NOT_SUPPORTED, "replica %u: batches hold hard spheres or Lennard-Jones bodies", k);
        if (d->interaction != interaction)
            return fail(HMC_INVALID_ARGUMENT, "replica %u: all replicas need the same interaction", k);
        if (!lj && !(d->diameter > 0.0)) return fail(HMC_INVALID_ARGUMENT, "replica %u: diameter must be positive", k);
        if (lj && (!(d->lj_sigma > 0.0) || !(d->lj_r_cut > 0.0) || !(d->lj_r_shift > 0.0) ||
                   !std::isfinite(d->lj_epsilon) || !std::isfinite(d->lj_sigma) || !std::isfinite(d->lj_r_cut) ||
                   !std::isfinite(d->lj_r_shift)))
            return fail(HMC_INVALID_ARGUMENT, "replica %u: Lennard-Jones sigma, r_cut and r_shift must be positive", k);
        if (d->n_bodies > 0 && !positions[k]) return fail(HMC_INVALID_ARGUMENT, "replica %u: positions is NULL", k);
        for (uint32_t a = 0; a < dim; ++a)
            if (!(d->edge_lengths[a] > 0.0) || !std::isfinite(d->edge_lengths[a]))
                return fail(HMC_INVALID_ARGUMENT, "replica %u: edge length %u must be positive", k, a);
        for (uint64_t i = 0; i < d->n_bodies * dim; ++i)
            if (!std::isfinite(positions[k][i]))
                return fail(HMC_NAN_STATE, "replica %u: position %llu is not finite", k, (unsigned long long)(i / dim));
        Replica& r = reps[k];
        std::memset(&r, 0, sizeof(Replica));
        const double pair_range = lj ? d->lj_r_cut : d->diameter;  // maximum_interaction_range
        const double boundary_range = d->boundary_range > 0.0 ? d->boundary_range : pair_range;
        const double body_range = d->body_interaction_range > 0.0 ? d->body_interaction_range : pair_range;
        double min_l = d->edge_lengths[0];
        for (uint32_t a = 0; a < dim; ++a) {
            r.g.L[a] = d->edge_lengths[a];
            min_l = std::min(min_l, d->edge_lengths[a]);
        }
        for (uint32_t a = dim; a < 3; ++a) r.g.L[a] = 1.0;
        if (boundary_range > min_l / 2.0)
            return fail(HMC_RANGE_TOO_LARGE, "replica %u: boundary range %g exceeds L/2", k, boundary_range);
        if (body_range < pair_range) return fail(HMC_INVALID_ARGUMENT, "replica %u: body range below the pair range", k);
        if (!compute_dimensions((int)dim, r.g.L, body_range, r.g.width, r.g.shape))
            return fail(HMC_RANGE_TOO_LARGE, "replica %u: fewer than 2 spaces per axis", k);
        uint64_t cells = 1;
        for (uint32_t a = 0; a < dim; ++a) {
            if (r.g.shape[a] > (dim == 3 ? 1024u : 65535u))
                return fail(HMC_NOT_SUPPORTED, "replica %u: too many spaces on axis %u", k, a);
            r.g.half[a] = r.g.L[a] / 2.0;
            r.g.ghost_hi[a] = r.g.half[a] - boundary_range;
            r.g.ghost_lo[a] = -r.g.half[a] + boundary_range;
            r.g.w32[a] = (float)r.g.width[a];
            r.g.invL[a] = 1.0 / r.g.L[a];
            r.g.invW[a] = 1.0 / r.g.width[a];
            r.g.half_shape[a] = r.g.shape[a] / 2;
            if (r.g.shape[a] == 2) r.g.any_two = 1;
            cells *= r.g.shape[a];
        }
        r.g.n_cells = (uint32_t)cells;
        r.g.color_stride = (uint32_t)(cells >> dim);
        if (lj) {
            lj_setup_for((int)dim, r.g, r.p, d->lj_epsilon, d->lj_sigma, d->lj_r_cut, d->lj_r_shift);
        } else {
            r.p.sigma2 = d->diameter * d->diameter;
            sphere_bound_for((int)dim, r.g, r.p);
        }
        r.kt = 1.0;
        r.cell_base = (uint32_t)cells_total;
        r.body_base = (uint32_t)n_total;
        r.n_bodies = (uint32_t)d->n_bodies;
        r.step = d->step;
        r.substep = d->substep;
        r.seed = d->seed;
        n_total += d->n_bodies;
        cells_total += cells;
        if (n_total >= (1ull << 31)) return fail(HMC_INVALID_ARGUMENT, "too many bodies");
        if (cells_total > (1ull << 31)) return fail(HMC_NOT_SUPPORTED, "more than 2^31 spaces in the batch");
    }
    HMC_CUDA(cudaSetDevice(ctx->device));
    hmc_batch* bt = new hmc_batch();
    ctx->refs.fetch_add(1);
    bt->ctx = ctx;
    bt->dim = (int)dim;
    bt->n_rep = n_replicas;
    bt->n = n_total;
    bt->cells = (uint32_t)cells_total;
    bt->rep = reps;
    bt->interaction = interaction;
    bt->body_range.resize(n_replicas);
    for (uint32_t k = 0; k < n_replicas; ++k) {
        const hmc_system_desc* d = descs + k;
        const double pr = lj ? d->lj_r_cut : d->diameter;
        bt->body_range[k] = d->body_interaction_range > 0.0 ? d->body_interaction_range : pr;
    }
    auto destroy_fail = [&](hmc_status st) {
        std::string msg = g_last_error;
        hmc_batch_destroy(bt);
        g_last_error = msg;
        return st;
    };
    bt->cell_base.resize(n_replicas + 1);
    bt->body_base.resize(n_replicas + 1);
    for (uint32_t k = 0; k < n_replicas; ++k) {
        bt->cell_base[k] = reps[k].cell_base;
        bt->body_base[k] = reps[k].body_base;
    }
    bt->cell_base[n_replicas] = bt->cells;
    bt->body_base[n_replicas] = (uint32_t)n_total;
    cudaError_t e = cudaStreamCreateWithFlags(&bt->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&bt->rep_pinned, sizeof(Replica) * n_replicas);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&bt->host_stats, sizeof(DeviceStats));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&bt->host_rep_u64, sizeof(unsigned long long) * n_replicas);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&bt->host_nonempty, sizeof(unsigned int) * n_replicas);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&bt->host_first_bad, sizeof(unsigned long long));
    if (e == cudaSuccess)
        e = cudaMallocHost((void**)&bt->host_rep_counts, sizeof(unsigned long long) * 2 * (size_t)n_replicas);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&bt->host_totals, sizeof(BatchSweepTotals));
    if (e != cudaSuccess) {
        fail(HMC_CUDA_ERROR, "batch setup: %s", cudaGetErrorString(e));
        return destroy_fail(HMC_CUDA_ERROR);
    }
    const uint64_t n = n_total;
    const uint32_t cells = bt->cells;
    const uint32_t scan_blocks = (cells + 2047) / 2048;
    Arrays& A = bt->arr;
    Replica* d_rep = nullptr;
    uint32_t *d_cell_base = nullptr, *d_body_rep = nullptr;
    hmc_status st;
    if ((st = balloc(bt, &A.body_pos, n)) || (st = balloc(bt, &A.sorted_b, n)) || (st = balloc(bt, &A.sorted_s, n)) ||
        (st = balloc(bt, &A.sorted_off, n)) || (st = balloc(bt, &A.sorted_body, n)) ||
        (st = balloc(bt, &A.slot_of_body, n)) || (st = balloc(bt, &A.body_cell, n)) ||
        (st = balloc(bt, &A.body_rank, n)) || (st = balloc(bt, &A.body_m, n)) || (st = balloc(bt, &A.cell_count, cells)) ||
        (st = balloc(bt, &A.cell_start, (size_t)cells + 1)) || (st = balloc(bt, &A.block_sums, (size_t)scan_blocks * 9)) ||
        (st = balloc(bt, &A.color_cells, cells)) || (st = balloc(bt, &A.stats, 1)) ||
        (st = balloc(bt, &d_rep, n_replicas)) || (st = balloc(bt, &d_cell_base, (size_t)n_replicas + 1)) ||
        (st = balloc(bt, &d_body_rep, n)) || (st = balloc(bt, &bt->b.color_rep, cells)) ||
        (st = balloc(bt, &bt->b.accepted, n_replicas)) || (st = balloc(bt, &bt->b.nonempty, n_replicas)) ||
        (st = balloc(bt, &bt->b.overlaps, n_replicas)) || (st = balloc(bt, &bt->stage, n * dim)) ||
        (st = balloc(bt, &bt->first_bad, 1)) || (st = balloc(bt, &bt->round_dev, 1)) ||
        (st = balloc(bt, &bt->rep_counts, 2 * (size_t)n_replicas)) || (st = balloc(bt, &bt->totals, 1)))
        return destroy_fail(st);
    bt->b.round_dev = bt->round_dev;
    A.body_ori = nullptr;
    A.sorted_q = nullptr;
    A.zig_x = ctx->zig;
    A.zig_f = ctx->zig + kZigLayers + 1;
    bt->b.rep = d_rep;
    bt->b.cell_base = d_cell_base;
    bt->b.body_rep = d_body_rep;
    bt->b.n_replicas = n_replicas;
    bt->b.n_cells = cells;
    bt->b.color_stride = cells >> dim;
    // Microstate::add_body (microstate.rs:777-835): each body keeps wrap(input).
    std::vector<double4> host(n);
    std::vector<uint32_t> host_rep(n);
    for (uint32_t k = 0; k < n_replicas; ++k) {
        for (uint32_t i = 0; i < reps[k].n_bodies; ++i) {
            double pnt[3] = {0.0, 0.0, 0.0};
            for (uint32_t a = 0; a < dim; ++a) pnt[a] = positions[k][(size_t)i * dim + a];
            if (dim == 2)
                wrap<2>(reps[k].g.L, pnt);
            else
                wrap<3>(reps[k].g.L, pnt);
            host[reps[k].body_base + i] = make_double4(pnt[0], pnt[1], pnt[2], 0.0);
            host_rep[reps[k].body_base + i] = k;
        }
    }
    e = cudaMemcpy(A.body_pos, host.data(), sizeof(double4) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_body_rep, host_rep.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(d_cell_base, bt->cell_base.data(), sizeof(uint32_t) * (n_replicas + 1), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        fail(HMC_CUDA_ERROR, "upload: %s", cudaGetErrorString(e));
        return destroy_fail(HMC_CUDA_ERROR);
    }
    *out = bt;
    return HMC_OK;
}

static uint32_t batch_family(const hmc_batch* bt) {
    return bt->interaction == HMC_LENNARD_JONES ? kFamBatchLj : kFamBatch;
}

// The variant the batch's next sweep runs: its own choice, else the cached one for its family,
// dimension, precision and density band (all replicas' bodies over all their spaces), else 0.
static uint32_t batch_variant_of(const hmc_batch* bt, bool fp32) {
    if (bt->variant[fp32] >= 0) return (uint32_t)bt->variant[fp32];
    return cached_variant(batch_family(bt), (uint32_t)bt->dim, fp32, density_band((double)bt->n, (double)bt->cells));
}

hmc_status hmc_batch_sweep(hmc_batch* bt, const hmc_sweep_params* params, hmc_count* counts, hmc_count* total) {
    if (!bt || !params) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    const hmc_sweep_params& p0 = params[0];
    if (p0.struct_size < sizeof(hmc_sweep_params)) return fail(HMC_INVALID_ARGUMENT, "hmc_sweep_params.struct_size");
    if (p0.move != HMC_TRANSLATE) return fail(HMC_NOT_SUPPORTED, "batch replicas take translation moves");
    if (p0.precision > HMC_FP32_RECHECK) return fail(HMC_INVALID_ARGUMENT, "precision");
    for (uint32_t k = 0; k < bt->n_rep; ++k) {
        const hmc_sweep_params& p = params[k];
        if (p.move != p0.move || p.precision != p0.precision || p.n_sweeps != p0.n_sweeps ||
            p.increment_step != p0.increment_step)
            return fail(HMC_INVALID_ARGUMENT, "replica %u: move, precision, n_sweeps and increment_step must agree", k);
        double lmax = 0.0;
        for (int a = 0; a < bt->dim; ++a) lmax = std::max(lmax, bt->rep[k].g.L[a]);
        if (!(p.maximum > 0.0) || !(p.maximum <= 4.0 * lmax))
            return fail(HMC_INVALID_ARGUMENT, "replica %u: maximum must be in (0, 4 box lengths]", k);
        if (!(p.temperature > 0.0) || !std::isfinite(p.temperature))
            return fail(HMC_INVALID_ARGUMENT, "replica %u: temperature must be positive", k);
    }
    for (uint32_t k = 0; k < bt->n_rep; ++k) {
        bt->rep[k].max_move = params[k].maximum;
        bt->rep[k].kt = params[k].temperature;  // Isothermal kT of replica k (hard spheres ignore it)
    }
    HMC_CUDA(cudaSetDevice(bt->ctx->device));
    const bool fp32 = p0.precision == HMC_FP32_RECHECK;
    const uint32_t colors = 1u << bt->dim;
    const uint32_t variant = batch_variant_of(bt, fp32);
    if (counts) std::memset(counts, 0, sizeof(hmc_count) * bt->n_rep);
    if (bt->captured) return batch_sweep_captured(bt, p0, fp32, variant, counts, total);
    hmc_count tot{};
    for (uint32_t sweep = 0; sweep < p0.n_sweeps; ++sweep) {
        hmc_status st = batch_rebuild(bt, !fp32);
        if (st) return st;
        HMC_CUDA(launch_batch_rounds(bt->b, const_cast<Replica*>(bt->b.rep), bt->arr.stats, bt->stream));
        bt->kernel_launches += 1;
        HMC_CUDA(cudaMemsetAsync(bt->b.accepted, 0, sizeof(unsigned long long) * bt->n_rep, bt->stream));
        auto enqueue = [&](uint32_t r0, uint32_t r1) -> hmc_status {
            for (uint32_t round = r0; round < r1; ++round)
                for (uint32_t c = 0; c < colors; ++c) {
                    if (bt->interaction == HMC_LENNARD_JONES)
                        HMC_CUDA(launch_sweep_batch_lj(bt->dim, fp32, bt->b, bt->arr, c, round, bt->b.color_stride,
                                                       round > 0 || c > 0, round == 0 && c == 0, bt->stream,
                                                       variant));
                    else
                        HMC_CUDA(launch_sweep_batch(bt->dim, fp32, bt->b, bt->arr, c, round, bt->b.color_stride,
                                                    round > 0 || c > 0, round == 0 && c == 0, bt->stream, variant));
                    bt->kernel_launches += 1;
                }
            return HMC_OK;
        };
        const uint32_t guess = bt->rounds_guess;
        if ((st = enqueue(0, guess))) return st;
        if ((st = batch_read(bt))) return st;
        const uint32_t max_rounds = bt->host_stats->rounds;
        if (max_rounds > guess) {
            if ((st = enqueue(guess, max_rounds))) return st;
            if ((st = batch_read(bt))) return st;
        }
        if (max_rounds > 0) bt->rounds_guess = max_rounds;
        for (uint32_t k = 0; k < bt->n_rep; ++k) {
            Replica& r = bt->rep[k];
            const uint32_t ne = bt->host_nonempty[k];
            r.rounds = (r.n_bodies == 0 || ne == 0) ? 0u : (r.n_bodies + ne - 1) / ne;
            const uint64_t acc = bt->host_rep_u64[k];
            const uint64_t trials = (uint64_t)r.rounds * ne;
            if (counts) {
                counts[k].accepted += acc;
                counts[k].rejected += trials - acc;
            }
            tot.accepted += acc;
            tot.rejected += trials - acc;
            r.substep += r.rounds;  // increment_substep after every full colour set
            if (p0.increment_step) {
                r.step += 1;
                r.substep = 0;
            }
        }
        tot.rechecks += bt->host_stats->rechecks;
        tot.pair_checks += bt->host_stats->pair_checks;
        tot.order_ambiguous += bt->host_stats->ambiguous;
        double me;
        unsigned long long bits = bt->host_stats->max_err_bits;
        std::memcpy(&me, &bits, 8);
        tot.max_fp32_error = std::max(tot.max_fp32_error, me);
    }
    if (total) *total = tot;
    return HMC_OK;
}

hmc_status hmc_batch_set_captured_sweeps(hmc_batch* bt, uint32_t enable) {
    if (!bt) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    bt->captured = enable != 0;
    return HMC_OK;
}

hmc_status hmc_batch_set_launch_variant(hmc_batch* bt, uint32_t precision, uint32_t index) {
    if (!bt) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (precision > HMC_FP32_RECHECK) return fail(HMC_INVALID_ARGUMENT, "precision");
    uint32_t n = 0;
    family_shapes(batch_family(bt), &n);
    if (index != UINT32_MAX && index >= n) return fail(HMC_INVALID_ARGUMENT, "variant %u of %u", index, n);
    bt->variant[precision == HMC_FP32_RECHECK] = index == UINT32_MAX ? -1 : (int32_t)index;
    return HMC_OK;
}

}  // extern "C"

hmc_status hmc_batch_autotune(hmc_batch* bt, const hmc_sweep_params* params, uint32_t sweeps,
                              hmc_launch_variant* chosen, double* ms_per_sweep) {
    if (!bt || !params) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (params[0].precision > HMC_FP32_RECHECK) return fail(HMC_INVALID_ARGUMENT, "precision");
    if (sweeps == 0 || sweeps > 1000) return fail(HMC_INVALID_ARGUMENT, "sweeps must be in [1, 1000]");
    HMC_CUDA(cudaSetDevice(bt->ctx->device));
    const bool fp32 = params[0].precision == HMC_FP32_RECHECK;
    const uint32_t fam = batch_family(bt);
    uint32_t n_var = 0;
    family_shapes(fam, &n_var);
    const uint64_t n = bt->n;
    std::vector<std::pair<uint64_t, uint32_t>> counters(bt->n_rep);
    for (uint32_t k = 0; k < bt->n_rep; ++k) counters[k] = {bt->rep[k].step, bt->rep[k].substep};
    const uint32_t guess0 = bt->rounds_guess;
    const int32_t own0 = bt->variant[fp32];
    double4* bp = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&bp, sizeof(double4) * (n ? n : 1), bt->stream);
    if (e == cudaSuccess && n)
        e = cudaMemcpyAsync(bp, bt->arr.body_pos, sizeof(double4) * n, cudaMemcpyDeviceToDevice, bt->stream);
    auto restore = [&]() -> hmc_status {
        if (n) HMC_CUDA(cudaMemcpyAsync(bt->arr.body_pos, bp, sizeof(double4) * n, cudaMemcpyDeviceToDevice, bt->stream));
        for (uint32_t k = 0; k < bt->n_rep; ++k) {
            bt->rep[k].step = counters[k].first;
            bt->rep[k].substep = counters[k].second;
        }
        bt->rounds_guess = guess0;
        return HMC_OK;
    };
    std::vector<hmc_sweep_params> ps(params, params + bt->n_rep);
    auto run = [&](const hmc_sweep_params& q) -> hmc_status {
        for (auto& x : ps) {
            x.n_sweeps = q.n_sweeps;
            x.increment_step = q.increment_step;
        }
        return hmc_batch_sweep(bt, ps.data(), nullptr, nullptr);
    };
    hmc_status st = e == cudaSuccess ? HMC_OK : fail(HMC_CUDA_ERROR, "batch autotune: %s", cudaGetErrorString(e));
    std::vector<double> ms(n_var, 0.0);
    uint32_t best = 0;
    for (uint32_t v = 0; v < n_var && !st; ++v) {
        bt->variant[fp32] = (int32_t)v;
        st = time_variant(bt->stream, params[0], sweeps, run, restore, &ms[v]);
        if (!st && ms[v] < ms[best]) best = v;
    }
    hmc_status st2 = restore();
    if (bp) cudaFreeAsync(bp, bt->stream);
    cudaStreamSynchronize(bt->stream);
    if (st || st2) {
        bt->variant[fp32] = own0;
        return st ? st : st2;
    }
    bt->variant[fp32] = (int32_t)best;
    cache_variant(fam, (uint32_t)bt->dim, fp32, density_band((double)bt->n, (double)bt->cells), best);
    if (chosen) describe_variant(fam, best, chosen);
    if (ms_per_sweep) std::memcpy(ms_per_sweep, ms.data(), sizeof(double) * n_var);
    return HMC_OK;
}

extern "C" {

hmc_status hmc_batch_get_state(hmc_batch* bt, uint32_t replica, double* positions, uint64_t* step, uint32_t* substep) {
    if (!bt || replica >= bt->n_rep) return fail(HMC_INVALID_ARGUMENT, "no such replica");
    const Replica& r = bt->rep[replica];
    if (positions && r.n_bodies) {
        HMC_CUDA(cudaSetDevice(bt->ctx->device));
        HMC_CUDA(launch_pack_positions(bt->dim, bt->arr.body_pos + r.body_base, bt->stage, r.n_bodies, bt->stream));
        HMC_CUDA(cudaMemcpyAsync(positions, bt->stage, sizeof(double) * r.n_bodies * bt->dim, cudaMemcpyDeviceToHost,
                                 bt->stream));
        HMC_CUDA(cudaStreamSynchronize(bt->stream));
    }
    if (step) *step = r.step;
    if (substep) *substep = r.substep;
    return HMC_OK;
}

hmc_status hmc_batch_set_state(hmc_batch* bt, uint32_t replica, const double* positions, uint64_t step,
                               uint32_t substep) {
    if (!bt || replica >= bt->n_rep) return fail(HMC_INVALID_ARGUMENT, "no such replica");
    Replica& r = bt->rep[replica];
    if (r.n_bodies && !positions) return fail(HMC_INVALID_ARGUMENT, "positions is NULL");
    if (r.n_bodies) {
        HMC_CUDA(cudaSetDevice(bt->ctx->device));
        const uint64_t count = (uint64_t)r.n_bodies * bt->dim;
        HMC_CUDA(cudaMemcpyAsync(bt->stage, positions, sizeof(double) * count, cudaMemcpyHostToDevice, bt->stream));
        HMC_CUDA(cudaMemsetAsync(bt->first_bad, 0xFF, sizeof(unsigned long long), bt->stream));
        HMC_CUDA(launch_check_finite(bt->stage, count, (uint32_t)bt->dim, bt->first_bad, bt->stream));
        HMC_CUDA(cudaMemcpyAsync(bt->host_first_bad, bt->first_bad, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                 bt->stream));
        HMC_CUDA(cudaStreamSynchronize(bt->stream));
        if (*bt->host_first_bad != ~0ull)
            return fail(HMC_NAN_STATE, "position %llu is not finite", (unsigned long long)*bt->host_first_bad);
        HMC_CUDA(launch_unpack_positions(bt->dim, bt->stage, bt->arr.body_pos + r.body_base, r.n_bodies, bt->stream));
        HMC_CUDA(cudaStreamSynchronize(bt->stream));
    }
    r.step = step;
    r.substep = substep;
    return HMC_OK;
}

// Arrays of replica k inside the batch's arrays: its bodies at its offset, the space arrays
// from their start (a replica's own checkerboard has no more spaces than the batch).
static Arrays replica_view(const hmc_batch* bt, uint32_t k) {
    Arrays v = bt->arr;
    const uint32_t o = bt->rep[k].body_base;
    v.body_pos += o;
    v.sorted_b += o;
    v.sorted_s += o;
    v.sorted_off += o;
    v.sorted_body += o;
    v.slot_of_body += o;
    v.body_cell += o;
    v.body_rank += o;
    v.body_m += o;
    v.body_ori = nullptr;
    v.sorted_q = nullptr;
    return v;
}

hmc_status hmc_batch_tune(hmc_batch* bt, hmc_sweep_params* params, double target, uint32_t samples, uint32_t steps) {
    if (!bt || !params) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (!(target > 0.0 && target < 1.0)) return fail(HMC_INVALID_ARGUMENT, "target acceptance must be in (0, 1)");
    if (samples == 0 || samples >= (1u << 31)) return fail(HMC_INVALID_ARGUMENT, "samples must be in [1, 2^31)");
    for (uint32_t k = 0; k < bt->n_rep; ++k) {
        const hmc_sweep_params& p = params[k];
        if (p.struct_size < sizeof(hmc_sweep_params)) return fail(HMC_INVALID_ARGUMENT, "hmc_sweep_params.struct_size");
        if (p.move != HMC_TRANSLATE) return fail(HMC_NOT_SUPPORTED, "batch replicas take translation moves");
        if (p.precision > HMC_FP32_RECHECK) return fail(HMC_INVALID_ARGUMENT, "precision");
        if (!(p.maximum > 0.0) || !std::isfinite(p.maximum))
            return fail(HMC_INVALID_ARGUMENT, "replica %u: maximum must be positive", k);
        if (!(p.temperature > 0.0)) return fail(HMC_INVALID_ARGUMENT, "replica %u: temperature must be positive", k);
    }
    for (uint32_t k = 0; k < bt->n_rep; ++k)
        if ((params[k].flags & ~HMC_TUNE_PER_SAMPLE_STREAMS) || params[k].flags != params[0].flags)
            return fail(HMC_INVALID_ARGUMENT, "tune flags must be known and the same for every replica");
    if (steps == 0 || bt->n == 0) return HMC_OK;
    HMC_CUDA(cudaSetDevice(bt->ctx->device));
    const bool lj = bt->interaction == HMC_LENNARD_JONES;
    if (!(params[0].flags & HMC_TUNE_PER_SAMPLE_STREAMS)) {
        // the reference's single stream per replica, one warp per replica in one launch: each
        // replica's cell list is built (with its own Counter's checkerboard) into its own part of
        // temporary space-count and space-start arrays, as hmc_tune builds a system's
        std::vector<TuneJob> jobs;
        std::vector<uint32_t> which;
        uint64_t cells_total = 0;
        for (uint32_t k = 0; k < bt->n_rep; ++k) cells_total += bt->cell_base[k + 1] - bt->cell_base[k] + 1;
        uint32_t *cc = nullptr, *cs = nullptr;
        TuneJob* dj = nullptr;
        cudaError_t e = cudaMallocAsync((void**)&cc, sizeof(uint32_t) * cells_total, bt->stream);
        if (e == cudaSuccess) e = cudaMallocAsync((void**)&cs, sizeof(uint32_t) * cells_total, bt->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(bt->arr.stats, 0, sizeof(DeviceStats), bt->stream);
        uint64_t off = 0;
        for (uint32_t k = 0; k < bt->n_rep && e == cudaSuccess; ++k) {
            const Replica& r = bt->rep[k];
            const uint32_t cells_k = bt->cell_base[k + 1] - bt->cell_base[k];
            const uint64_t o = off;
            off += cells_k + 1;
            if (r.n_bodies == 0) continue;
            Geometry g = r.g;
            Sfc64 rng = make_rng(r.step, r.substep, r.seed, UINT64_MAX);  // the origin of rebuild()
            for (int a = 0; a < bt->dim; ++a) {
                const double u0 = uniform01(rng);
                g.origin[a] = -g.L[a] / 2.0 - u0 * g.width[a];
            }
            Arrays v = replica_view(bt, k);
            v.cell_count = cc + o;
            v.cell_start = cs + o;
            // each rebuild appends to the colour lists from zero; the error flags of all of them
            // (and of the tuner) accumulate
            e = cudaMemsetAsync(&v.stats->nonempty, 0, sizeof(unsigned int), bt->stream);
            if (e == cudaSuccess) e = cudaMemsetAsync(v.stats->color_count, 0, sizeof(unsigned int) * 8, bt->stream);
            if (e == cudaSuccess) e = launch_rebuild(bt->dim, g, v, r.n_bodies, true, bt->stream);
            bt->kernel_launches += 6;
            TuneJob job{};
            job.g = g;
            job.a = v;
            job.p = r.p;
            job.step = r.step;
            job.substep = r.substep;
            job.seed = r.seed;
            job.n_bodies = r.n_bodies;
            job.samples = samples;
            job.steps = steps;
            job.maximum = params[k].maximum;
            job.kt = params[k].temperature;
            job.target = target;
            jobs.push_back(job);
            which.push_back(k);
        }
        const uint32_t nj = (uint32_t)jobs.size();
        if (e == cudaSuccess && nj) e = cudaMallocAsync((void**)&dj, sizeof(TuneJob) * nj, bt->stream);
        if (e == cudaSuccess && nj)
            e = cudaMemcpyAsync(dj, jobs.data(), sizeof(TuneJob) * nj, cudaMemcpyHostToDevice, bt->stream);
        if (e == cudaSuccess && nj) {
            e = lj ? launch_tune_stream_lj(bt->dim, dj, nj, bt->stream)
                   : launch_tune_stream_sphere(bt->dim, dj, nj, bt->stream);
            bt->kernel_launches += 1;
        }
        if (e == cudaSuccess && nj)
            e = cudaMemcpyAsync(jobs.data(), dj, sizeof(TuneJob) * nj, cudaMemcpyDeviceToHost, bt->stream);
        for (void* ptr : {(void*)cc, (void*)cs, (void*)dj})
            if (ptr) cudaFreeAsync(ptr, bt->stream);
        cudaError_t e2 = cudaStreamSynchronize(bt->stream);
        if (e == cudaSuccess) e = e2;
        if (e != cudaSuccess) return fail(HMC_CUDA_ERROR, "batch tune: %s", cudaGetErrorString(e));
        HMC_CUDA(cudaMemcpy(bt->host_stats, bt->arr.stats, sizeof(DeviceStats), cudaMemcpyDeviceToHost));
        if (bt->host_stats->error_flags) return fail(HMC_OUTSIDE_CHECKERBOARD, "batch tune: a body maps to no space");
        for (uint32_t j = 0; j < nj; ++j) params[which[j]].maximum = jobs[j].maximum;
        return HMC_OK;
    }
    uint64_t* db = nullptr;
    double4 *dt = nullptr, *dq = nullptr;
    double *du = nullptr, *dh = nullptr;
    uint8_t* dd = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&db, sizeof(uint64_t) * samples, bt->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dt, sizeof(double4) * samples, bt->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dq, sizeof(double4) * samples, bt->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&du, sizeof(double) * samples, bt->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dh, sizeof(double) * samples, bt->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dd, 2 * (size_t)samples, bt->stream);
    std::vector<uint8_t> hd(samples);
    hmc_status st = HMC_OK;
    // Replica by replica, hmc_tune on a view of the batch's arrays: the checkerboard of the
    // replica's Counter, the same samples and the same scaling, so replica k's maximum equals
    // hmc_tune of the same state in its own system. The next sweep rebuilds the batch.
    for (uint32_t k = 0; k < bt->n_rep && e == cudaSuccess && st == HMC_OK; ++k) {
        Replica& r = bt->rep[k];
        hmc_sweep_params& p = params[k];
        if (r.n_bodies == 0) continue;
        Geometry g = r.g;
        Sfc64 rng = make_rng(r.step, r.substep, r.seed, UINT64_MAX);  // the origin of rebuild()
        for (int a = 0; a < bt->dim; ++a) {
            const double off = uniform01(rng);
            g.origin[a] = -g.L[a] / 2.0 - off * g.width[a];
        }
        const Arrays v = replica_view(bt, k);
        e = cudaMemsetAsync(v.stats, 0, sizeof(DeviceStats), bt->stream);
        if (e == cudaSuccess) e = launch_rebuild(bt->dim, g, v, r.n_bodies, true, bt->stream);
        if (e != cudaSuccess) break;
        bt->kernel_launches += 6;  // the rebuild
        double lmax = 0.0;
        for (int a = 0; a < bt->dim; ++a) lmax = std::max(lmax, g.L[a]);
        const bool fp32 = p.precision == HMC_FP32_RECHECK;
        for (uint32_t step = 0; step < steps && e == cudaSuccess; ++step) {
            if (p.maximum > 4.0 * lmax) p.maximum = 4.0 * lmax;  // the samplers' bound (see hmc_sweep)
            Launch L{};
            L.step = r.step;
            L.substep = r.substep;
            L.seed = r.seed;
            L.max_move = p.maximum;
            L.kt = p.temperature;
            L.n_bodies = r.n_bodies;
            e = launch_tune_moves(bt->dim, g, v, L, step, samples, false, db, dt, dq, du, bt->stream);
            if (e == cudaSuccess) {
                if (lj)
                    e = launch_eval_lj(bt->dim, fp32, g, v, r.p, db, dt, du, p.temperature, samples, dd, dd + samples,
                                       dh, bt->stream);
                else
                    e = launch_eval_sphere(bt->dim, fp32, g, v, r.p, db, dt, samples, dd, dd + samples, bt->stream);
            }
            if (e == cudaSuccess) e = cudaMemcpyAsync(hd.data(), dd, samples, cudaMemcpyDeviceToHost, bt->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(bt->stream);
            if (e != cudaSuccess) break;
            bt->kernel_launches += 2;
            uint64_t acc = 0;
            for (uint32_t j = 0; j < samples; ++j) acc += hd[j];
            p.maximum *= ((double)acc / (double)samples + 1.5) / (target + 1.5);  // tune_by_scaling
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(bt->host_stats, v.stats, sizeof(DeviceStats), cudaMemcpyDeviceToHost,
                                                  bt->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(bt->stream);
        if (e == cudaSuccess) {
            const uint32_t f = bt->host_stats->error_flags;
            if (f & kErrNonFinite) st = fail(HMC_NAN_STATE, "replica %u: a body position is not finite", k);
            else if (f & kErrOutsideCheckerboard) st = fail(HMC_OUTSIDE_CHECKERBOARD, "replica %u: a body maps to no space", k);
        }
    }
    if (db) cudaFreeAsync(db, bt->stream);
    if (dt) cudaFreeAsync(dt, bt->stream);
    if (dq) cudaFreeAsync(dq, bt->stream);
    if (du) cudaFreeAsync(du, bt->stream);
    if (dh) cudaFreeAsync(dh, bt->stream);
    if (dd) cudaFreeAsync(dd, bt->stream);
    cudaError_t e2 = cudaStreamSynchronize(bt->stream);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return fail(HMC_CUDA_ERROR, "batch tune: %s", cudaGetErrorString(e));
    return st;
}

hmc_status hmc_batch_sdf(hmc_batch* bt, double x_max, uint32_t n_bins, uint64_t* counts) {
    if (!bt || !counts) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (bt->interaction != HMC_HARD_SPHERE) return fail(HMC_NOT_SUPPORTED, "the scale distribution is for hard spheres");
    if (!(x_max > 0.0 && x_max < 0.5)) return fail(HMC_INVALID_ARGUMENT, "x_max must be in (0, 0.5)");
    if (n_bins == 0 || n_bins > 8192) return fail(HMC_INVALID_ARGUMENT, "1 to 8192 bins");
    HMC_CUDA(cudaSetDevice(bt->ctx->device));
    // Replica by replica, hmc_sdf's histogram on a view of the batch's arrays: the replica's
    // bodies at its offset, the (wider, so fewer) spaces of its histogram grid at the start of
    // the batch's space arrays. The next sweep rebuilds the batch's cell order from scratch.
    unsigned long long* d = nullptr;
    HMC_CUDA(cudaMallocAsync((void**)&d, sizeof(unsigned long long) * n_bins, bt->stream));
    std::vector<unsigned long long> h((size_t)n_bins * bt->n_rep);
    hmc_status st = HMC_OK;
    for (uint32_t k = 0; k < bt->n_rep && st == HMC_OK; ++k) {
        const Replica& r = bt->rep[k];
        const double sigma = std::sqrt(r.p.sigma2);
        Geometry g = r.g;
        const double range = std::max(sigma / (1.0 - x_max), bt->body_range[k]);
        if (!compute_dimensions(bt->dim, g.L, range, g.width, g.shape)) {
            st = fail(HMC_RANGE_TOO_LARGE, "replica %u: a histogram reaching %g needs two spaces per axis", k, range);
            break;
        }
        uint64_t cells = 1;
        g.any_two = 0;
        for (int a = 0; a < bt->dim; ++a) {
            g.w32[a] = (float)g.width[a];
            g.invW[a] = 1.0 / g.width[a];
            g.half_shape[a] = g.shape[a] / 2;
            if (g.shape[a] == 2) g.any_two = 1;
            g.origin[a] = -g.L[a] / 2.0;
            cells *= g.shape[a];
        }
        g.n_cells = (uint32_t)cells;  // no more than the replica's own spaces: these are wider
        g.color_stride = (uint32_t)(cells >> bt->dim);
        const Arrays v = replica_view(bt, k);
        cudaError_t e = cudaMemsetAsync(v.stats, 0, sizeof(DeviceStats), bt->stream);
        if (e == cudaSuccess) e = launch_rebuild(bt->dim, g, v, r.n_bodies, true, bt->stream);
        if (e == cudaSuccess)
            e = launch_pair_histogram(bt->dim, true, g, v, r.n_bodies, sigma, x_max, (double)n_bins / x_max, n_bins, d,
                                      bt->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(h.data() + (size_t)k * n_bins, d, sizeof(unsigned long long) * n_bins,
                                cudaMemcpyDeviceToHost, bt->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(bt->host_stats, v.stats, sizeof(DeviceStats), cudaMemcpyDeviceToHost, bt->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(bt->stream);
        if (e != cudaSuccess) {
            st = fail(HMC_CUDA_ERROR, "replica %u: scale distribution: %s", k, cudaGetErrorString(e));
            break;
        }
        bt->kernel_launches += r.n_bodies > 0 ? 7 : 2;  // the rebuild and the histogram
        const uint32_t f = bt->host_stats->error_flags;
        if (f & kErrNonFinite) st = fail(HMC_NAN_STATE, "replica %u: a body position is not finite", k);
        else if (f & kErrOutsideCheckerboard) st = fail(HMC_OUTSIDE_CHECKERBOARD, "replica %u: a body maps to no space", k);
    }
    cudaFreeAsync(d, bt->stream);
    cudaError_t e2 = cudaStreamSynchronize(bt->stream);
    if (st) return st;
    if (e2 != cudaSuccess) return fail(HMC_CUDA_ERROR, "scale distribution: %s", cudaGetErrorString(e2));
    for (size_t i = 0; i < h.size(); ++i) counts[i] = h[i];
    return HMC_OK;
}

hmc_status hmc_batch_overlap_check(hmc_batch* bt, uint64_t* n_overlaps) {
    if (!bt || !n_overlaps) return fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (bt->interaction == HMC_LENNARD_JONES) return fail(HMC_NOT_SUPPORTED, "overlap check of a soft potential");
    HMC_CUDA(cudaSetDevice(bt->ctx->device));
    hmc_status st = batch_rebuild(bt, true);
    if (st) return st;
    if ((st = batch_read(bt))) return st;
    HMC_CUDA(launch_overlap_batch(bt->dim, bt->b, bt->arr, (uint32_t)bt->n, bt->stream));
    bt->kernel_launches += 1;
    HMC_CUDA(cudaMemcpyAsync(bt->host_rep_u64, bt->b.overlaps, sizeof(unsigned long long) * bt->n_rep,
                             cudaMemcpyDeviceToHost, bt->stream));
    HMC_CUDA(cudaStreamSynchronize(bt->stream));
    for (uint32_t k = 0; k < bt->n_rep; ++k) n_overlaps[k] = bt->host_rep_u64[k];
    return HMC_OK;
}

uint64_t hmc_batch_kernel_launches(hmc_batch* bt) { return bt ? bt->kernel_launches : 0; }

}  // extern "C"
