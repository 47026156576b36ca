// hmc_overlap_count_noalloc: the hard-sphere overlap count with no device allocation.
//
// Who needs this: a caller that cannot call cudaMalloc at the point where it wants the
// check. Examples are a host framework whose device memory all comes from its own
// pre-reserved pool (a stray cudaMalloc would fragment or exceed its budget), code that
// runs between allocation-free phases of a long job, or a plugin that must not grow the
// process's device footprint after start-up. hmc_overlap_check needs an hmc_system, whose
// creation allocates the cell list; this entry point instead keeps its cell list in one
// fixed-size array in the library's own device memory and writes only to buffers the
// caller passes.
//
// The scratch array (kScratchBytes, about 3.4 MB) is a file-scope __device__ array, so
// every GPU that loads the library holds it until the process exits. Its capacity caps
// the input at kMaxBodies bodies; larger inputs are rejected with HMC_INVALID_ARGUMENT.
// Every call uses the same array and leaves its contents behind; the kernels clear what
// must start at zero. Two calls whose work overlaps on the GPU (for example on two
// streams) race on the array and give wrong counts; serialise them.
//
// In host code the array's name is only a host-side handle, not a device address. The
// device address comes from cudaGetSymbolAddress, taken once per device with that device
// current, on the first call that runs on it. CUDA loads a library's device code lazily by
// default (unless CUDA_MODULE_LOADING=EAGER), so that first call is also the one that creates
// the array on the device: it grows the device footprint once. A caller that must not grow it
// later makes one call at start-up (n_bodies = 0 is enough), before capturing any stream into a
// CUDA graph. The address is kept together with the identity of the device's context; after a
// cudaDeviceReset the context is a new one and the next call looks the address up again.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <utility>

#include "../../include/hmc.h"
#include "hmc_math.cuh"

namespace {

constexpr uint32_t kMaxBodies = HMC_NOALLOC_MAX_BODIES;
constexpr uint32_t kMaxCells = HMC_NOALLOC_MAX_CELLS;
constexpr int kScanThreadsNA = 1024;
constexpr int kScanItemsNA = (kMaxCells + kScanThreadsNA - 1) / kScanThreadsNA;

// Layout of the scratch array (all offsets multiples of 256 bytes).
struct ScratchLayout {
    static constexpr size_t sites = 0;                                       // double4[kMaxBodies]
    static constexpr size_t cell_count = sites + sizeof(double4) * kMaxBodies;  // u32[kMaxCells]
    static constexpr size_t cell_start = cell_count + 4ull * kMaxCells;       // u32[kMaxCells + 64]
    static constexpr size_t body_cell = cell_start + 4ull * (kMaxCells + 64);  // u32[kMaxBodies]
    static constexpr size_t body_rank = body_cell + 4ull * kMaxBodies;        // u32[kMaxBodies]
    static constexpr size_t sorted = body_rank + 4ull * kMaxBodies;           // u32[kMaxBodies]
    static constexpr size_t total = sorted + 4ull * kMaxBodies;
};
constexpr size_t kScratchBytes = ScratchLayout::total;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct NaGeom {
    double L[3], half[3], ghost_hi[3], ghost_lo[3];
    uint32_t nc[3];  // cells per axis
    uint32_t n_cells;
    double sigma2;
};

struct NaPtrs {
    double4* sites;
    uint32_t* cell_count;
    uint32_t* cell_start;
    uint32_t* body_cell;
    uint32_t* body_rank;
    uint32_t* sorted;
};

NaPtrs carve(unsigned char* base) {
    NaPtrs p;
    p.sites = reinterpret_cast<double4*>(base + ScratchLayout::sites);
    p.cell_count = reinterpret_cast<uint32_t*>(base + ScratchLayout::cell_count);
    p.cell_start = reinterpret_cast<uint32_t*>(base + ScratchLayout::cell_start);
    p.body_cell = reinterpret_cast<uint32_t*>(base + ScratchLayout::body_cell);
    p.body_rank = reinterpret_cast<uint32_t*>(base + ScratchLayout::body_rank);
    p.sorted = reinterpret_cast<uint32_t*>(base + ScratchLayout::sorted);
    return p;
}

template <int DIM>
__device__ __forceinline__ uint32_t na_cell(const NaGeom& g, const double* x, uint32_t* m) {
    uint32_t idx = 0;
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
        double f = (x[a] + g.half[a]) / g.L[a];
        f = f - floor(f);
        double c = floor(f * (double)g.nc[a]);
        uint32_t ci = c >= 0.0 ? (uint32_t)c : 0u;
        if (ci >= g.nc[a]) ci = g.nc[a] - 1;
        m[a] = ci;
        idx = idx * g.nc[a] + ci;
    }
    return idx;
}

// Squared distance of sites t and s over s's primary and ghost images, with the image
// rule of the periodic boundary (the same arithmetic as hmc_overlap_check).
template <int DIM>
__device__ __forceinline__ double na_dist2(const NaGeom& g, const double* t, const double* s) {
    bool inside = true;
#pragma unroll
    for (int a = 0; a < DIM; ++a) inside = inside && (s[a] >= -g.half[a]) && (s[a] < g.half[a]);
    double p = 0.0;
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
        double d = hmc::dsub(t[a], s[a]);
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
                double d2 = hmc::dsub(t[a], hmc::dadd(s[a], tr));
                if (fabs(d2) < fabs(d)) d = d2;
            }
        }
        p = hmc::dadd(p, hmc::dmul(d, d));
    }
    return p;
}

__global__ void k_na_zero(NaPtrs p, uint32_t n_cells, unsigned long long* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_cells) p.cell_count[i] = 0;
    if (i == 0) *out = 0ull;
}

// Body positions B (as hmc_get_state returns them) -> sites S = wrap(B), binned.
template <int DIM>
__global__ void k_na_bin(NaGeom g, NaPtrs p, const double* pos, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s[3] = {pos[(size_t)i * DIM], pos[(size_t)i * DIM + 1], DIM == 3 ? pos[(size_t)i * DIM + 2] : 0.0};
    hmc::wrap<DIM>(g.L, s);
    p.sites[i] = make_double4(s[0], s[1], s[2], 0.0);
    uint32_t m[3];
    uint32_t c = na_cell<DIM>(g, s, m);
    p.body_cell[i] = c;
    p.body_rank[i] = atomicAdd(&p.cell_count[c], 1u);
}

__global__ void __launch_bounds__(kScanThreadsNA) k_na_scan(NaPtrs p, uint32_t n_cells) {
    __shared__ uint32_t warp_sums[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t base = threadIdx.x * kScanItemsNA;
    uint32_t sum = 0;
    for (int k = 0; k < kScanItemsNA; ++k) sum += base + k < n_cells ? p.cell_count[base + k] : 0u;
    uint32_t x = sum;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_sums[lane];
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        warp_sums[lane] = w;
    }
    __syncthreads();
    uint32_t run = (warp > 0 ? warp_sums[warp - 1] : 0u) + x - sum;
    for (int k = 0; k < kScanItemsNA; ++k) {
        uint32_t c = base + k;
        if (c < n_cells) {
            p.cell_start[c] = run;
            run += p.cell_count[c];
            if (c + 1 == n_cells) p.cell_start[n_cells] = run;
        }
    }
}

__global__ void k_na_scatter(NaPtrs p, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    p.sorted[p.cell_start[p.body_cell[i]] + p.body_rank[i]] = i;
}

// Pairs (i < j) whose sites overlap through any image: PairwiseCutoff::total_energy
// (hoomd-interaction/src/pairwise_cutoff.rs:720-745) as a count.
template <int DIM>
__global__ void k_na_count(NaGeom g, NaPtrs p, uint32_t n, unsigned long long* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t found = 0;
    if (i < n) {
        double4 s4 = p.sites[i];
        double t[3] = {s4.x, s4.y, s4.z};
        uint32_t m[3];
        na_cell<DIM>(g, t, m);
        int lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
            lo[a] = 0;
            hi[a] = 0;
        }
        for (int a = 0; a < DIM; ++a) {
            if (g.nc[a] >= 3) {
                lo[a] = -1;
                hi[a] = 1;
            } else {
                lo[a] = -(int)m[a];
                hi[a] = (int)g.nc[a] - 1 - (int)m[a];
            }
        }
        for (int o0 = lo[0]; o0 <= hi[0]; ++o0)
            for (int o1 = lo[1]; o1 <= hi[1]; ++o1)
                for (int o2 = (DIM == 3 ? lo[2] : 0); o2 <= (DIM == 3 ? hi[2] : 0); ++o2) {
                    int off[3] = {o0, o1, o2};
                    uint32_t c = 0;
                    for (int a = 0; a < DIM; ++a) {
                        int v = (int)m[a] + off[a];
                        if (v < 0) v += (int)g.nc[a];
                        if (v >= (int)g.nc[a]) v -= (int)g.nc[a];
                        c = c * g.nc[a] + (uint32_t)v;
                    }
                    for (uint32_t q = p.cell_start[c]; q < p.cell_start[c + 1]; ++q) {
                        uint32_t j = p.sorted[q];
                        if (j <= i) continue;
                        double4 o4 = p.sites[j];
                        double sv[3] = {o4.x, o4.y, o4.z};
                        if (na_dist2<DIM>(g, t, sv) < g.sigma2) found++;
                    }
                }
    }
    unsigned tot = __reduce_add_sync(0xffffffffu, found);
    if ((threadIdx.x & 31) == 0 && tot) atomicAdd(out, (unsigned long long)tot);
}

std::mutex g_setup_mutex;
constexpr int kMaxDevices = 64;
unsigned char* g_scratch_ptr[kMaxDevices] = {nullptr};
unsigned long long g_scratch_ctx[kMaxDevices] = {0};  // context the address belongs to (0: unknown)

hmc_status na_fail(hmc_status st, const char*) { return st; }

// The unique id of the calling thread's current context (cuCtxGetId through the runtime's
// driver entry point; ids are never reused within a process), or 0 when it cannot be read.
unsigned long long current_context_id() {
    using CtxGetId = int (*)(void*, unsigned long long*);
    static const CtxGetId fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<CtxGetId>(f);
    }();
    unsigned long long id = 0;
    if (!fn || fn(nullptr, &id) != 0) return 0;
    return id;
}

// One launch; its own status (no reliance on the thread's last-error state, which may hold an
// unrelated earlier error).
template <typename... K, typename... A>
cudaError_t launch(void (*kernel)(K...), uint32_t grid, uint32_t block, cudaStream_t s, A&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.stream = s;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

}  // namespace

extern "C" hmc_status hmc_overlap_count_noalloc(const double* positions, uint64_t n_bodies, uint32_t dim,
                                                const double* edge_lengths, double diameter, double boundary_range,
                                                uint64_t* overlaps_out, void* cuda_stream) {
    unsigned long long* overlaps = reinterpret_cast<unsigned long long*>(overlaps_out);
    if (dim != 2 && dim != 3) return na_fail(HMC_INVALID_ARGUMENT, "dim must be 2 or 3");
    if (!overlaps || !edge_lengths || (n_bodies > 0 && !positions))
        return na_fail(HMC_INVALID_ARGUMENT, "NULL argument");
    if (n_bodies > kMaxBodies)
        return na_fail(HMC_INVALID_ARGUMENT, "n_bodies exceeds the fixed scratch capacity (HMC_NOALLOC_MAX_BODIES)");
    if (!(diameter > 0.0)) return na_fail(HMC_INVALID_ARGUMENT, "diameter must be positive");
    double range = boundary_range > 0.0 ? boundary_range : diameter;
    NaGeom g{};
    uint64_t cells = 1;
    for (uint32_t a = 0; a < dim; ++a) {
        double L = edge_lengths[a];
        if (!(L > 0.0) || !std::isfinite(L)) return na_fail(HMC_INVALID_ARGUMENT, "edge lengths must be positive");
        if (range > L / 2.0) return na_fail(HMC_RANGE_TOO_LARGE, "interaction range exceeds L/2");
        g.L[a] = L;
        g.half[a] = L / 2.0;
        g.ghost_hi[a] = g.half[a] - range;
        g.ghost_lo[a] = -g.half[a] + range;
        // cells at least one diameter wide (with margin), so the 3^d stencil sees every pair
        double f = std::floor(L / (diameter * (1.0 + 1e-9)));
        g.nc[a] = f >= 1.0 ? (uint32_t)std::fmin(f, 65535.0) : 1u;
    }
    for (;;) {
        cells = 1;
        for (uint32_t a = 0; a < dim; ++a) cells *= g.nc[a];
        if (cells <= kMaxCells) break;
        uint32_t big = 0;
        for (uint32_t a = 1; a < dim; ++a)
            if (g.nc[a] > g.nc[big]) big = a;
        g.nc[big] -= 1;  // wider cells stay correct, only slower
    }
    for (uint32_t a = dim; a < 3; ++a) {
        g.L[a] = 1.0;
        g.nc[a] = 1;
    }
    g.n_cells = (uint32_t)cells;
    g.sigma2 = diameter * diameter;

    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices)
        return na_fail(HMC_CUDA_ERROR, "no current CUDA device");
    unsigned char* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        const unsigned long long ctx = current_context_id();
        if (!g_scratch_ptr[device] || ctx == 0 || ctx != g_scratch_ctx[device]) {
            // first call on this device, or its context was reset: (re)load the address
            void* ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess || !ptr) return na_fail(HMC_CUDA_ERROR, "cudaGetSymbolAddress failed");
            g_scratch_ptr[device] = static_cast<unsigned char*>(ptr);
            g_scratch_ctx[device] = current_context_id();
        }
        base = g_scratch_ptr[device];
    }
    NaPtrs p = carve(base);
    cudaStream_t s = (cudaStream_t)cuda_stream;
    const uint32_t n = (uint32_t)n_bodies;
    cudaError_t e = launch(k_na_zero, (g.n_cells + 255) / 256, 256, s, p, g.n_cells, overlaps);
    if (e == cudaSuccess && n > 0)
        e = dim == 2 ? launch(k_na_bin<2>, (n + 255) / 256, 256, s, g, p, positions, n)
                     : launch(k_na_bin<3>, (n + 255) / 256, 256, s, g, p, positions, n);
    if (e == cudaSuccess) e = launch(k_na_scan, 1, kScanThreadsNA, s, p, g.n_cells);
    if (e == cudaSuccess && n > 0) e = launch(k_na_scatter, (n + 255) / 256, 256, s, p, n);
    if (e == cudaSuccess && n > 0)
        e = dim == 2 ? launch(k_na_count<2>, (n + 127) / 128, 128, s, g, p, n, overlaps)
                     : launch(k_na_count<3>, (n + 127) / 128, 128, s, g, p, n, overlaps);
    return e == cudaSuccess ? HMC_OK : na_fail(HMC_CUDA_ERROR, "kernel launch failed");
}
