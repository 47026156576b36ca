// The serial sweep's cell grid (Sweep::apply_with_filter, hoomd-mc/src/sweep.rs:159-224, and
// QuickInsert / GrandCanonical): cells at least the pair range wide, each holding the bodies whose
// site lies in it, kept current after every accepted move; one warp walks the 3^d stencil with
// one lane per cell. Shared by the sphere, Lennard-Jones and shape kernels of the serial chain.
#pragma once

#include "hmc_device.cuh"

namespace hmc {
namespace {

struct SerialGrid {
    uint32_t nc[3];      // cells per axis (>= 1)
    double w[3];         // cell width L / nc (>= the diameter when nc >= 3 on that axis)
    uint32_t n_cells;
    uint32_t cap;        // bodies a cell holds
    uint32_t* size;      // [n_cells]
    uint32_t* items;     // [n_cells * cap]
    uint32_t* cell_of;   // [n] cell of each body's site
    double4* site;       // [n] S = wrap(B)
};

template <int DIM>
__device__ __forceinline__ void serial_cell(const Geometry& g, const SerialGrid& G, const double* s, uint32_t* m) {
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
        double f = floor(ddiv(dadd(s[a], g.half[a]), G.w[a]));
        uint32_t i = f > 0.0 ? (uint32_t)f : 0u;
        m[a] = i < G.nc[a] ? i : G.nc[a] - 1u;
    }
}
template <int DIM>
__device__ __forceinline__ uint32_t serial_index(const SerialGrid& G, const uint32_t* m) {
    uint32_t c = 0;
#pragma unroll
    for (int a = 0; a < DIM; ++a) c = c * G.nc[a] + m[a];
    return c;
}

// This lane's stencil cell around multi-index m (radix decomposition over the distinct cells of
// each axis); false when the lane has none.
template <int DIM>
__device__ __forceinline__ bool lane_cell(const SerialGrid& G, const uint32_t* m, uint32_t lane, uint32_t* cell) {
    uint32_t len[3] = {1, 1, 1}, off[3] = {0, 0, 0}, rem = lane;
#pragma unroll
    for (int a = 0; a < DIM; ++a) len[a] = G.nc[a] >= 3 ? 3u : G.nc[a];
#pragma unroll
    for (int a = DIM - 1; a >= 0; --a) {
        off[a] = rem % len[a];
        rem /= len[a];
    }
    uint32_t c[3] = {0, 0, 0};
#pragma unroll
    for (int a = 0; a < DIM; ++a) c[a] = G.nc[a] >= 3 ? wrap_index((int)m[a] + (int)off[a] - 1, G.nc[a]) : off[a];
    *cell = serial_index<DIM>(G, c);
    return rem == 0;
}

// Move body b's site into the cell of sv (lane 0 only): the last item of the old cell takes
// b's slot there (swap_remove), b is appended to the new cell.
template <int DIM>
__device__ __forceinline__ void serial_move(const Geometry& g, const SerialGrid& G, const Arrays& A, uint32_t b,
                                            const double* sv) {
    uint32_t ms[3] = {0, 0, 0};
    serial_cell<DIM>(g, G, sv, ms);
    const uint32_t nc = serial_index<DIM>(G, ms), oc = G.cell_of[b];
    if (nc == oc) return;
    const uint32_t osz = G.size[oc];
    for (uint32_t k = 0; k < osz; ++k)
        if (G.items[(size_t)oc * G.cap + k] == b) {
            G.items[(size_t)oc * G.cap + k] = G.items[(size_t)oc * G.cap + osz - 1];
            break;
        }
    G.size[oc] = osz - 1;
    const uint32_t nsz = G.size[nc];
    if (nsz < G.cap) {
        G.items[(size_t)nc * G.cap + nsz] = b;
        G.size[nc] = nsz + 1;
    } else {
        atomicOr(&A.stats->error_flags, kErrCellOverflow);
    }
    G.cell_of[b] = nc;
}

// Body tags (the tagged container of hoomd-microstate/src/microstate.rs:60-123): a new body
// takes the smallest free tag (a min-heap of freed tags), else the next unused one; removal
// frees the tag and swap_removes. Lane 0 only.
__device__ uint32_t tag_take(const BodyTags& T) {
    uint32_t& size = T.meta[0];
    if (size == 0) return T.meta[1]++;
    const uint32_t top = T.heap[0];
    const uint32_t last = T.heap[--size];
    uint32_t i = 0;
    for (;;) {
        const uint32_t l = 2 * i + 1, r = l + 1;
        uint32_t m = i;
        uint32_t vm = last;
        if (l < size && T.heap[l] < vm) {
            m = l;
            vm = T.heap[l];
        }
        if (r < size && T.heap[r] < vm) m = r;
        if (m == i) break;
        T.heap[i] = T.heap[m];
        i = m;
    }
    if (size) T.heap[i] = last;
    return top;
}
__device__ void tag_free(const BodyTags& T, uint32_t tag) {
    uint32_t i = T.meta[0]++;
    while (i > 0) {
        const uint32_t parent = (i - 1) / 2;
        if (T.heap[parent] <= tag) break;
        T.heap[i] = T.heap[parent];
        i = parent;
    }
    T.heap[i] = tag;
}

// Append body n at B = wrap(x), S = wrap(B) (Microstate::add_body) to the arrays and the grid.
template <int DIM>
__device__ void grid_append(const Geometry& g, const Arrays& A, const SerialGrid& G, const BodyTags& T, uint32_t n,
                            const double* x) {
    double b[3] = {x[0], x[1], x[2]};
    wrap_inv<DIM>(g.L, g.invL, b);
    double sv[3] = {b[0], b[1], b[2]};
    wrap_inv<DIM>(g.L, g.invL, sv);
    A.body_pos[n] = make_double4(b[0], b[1], DIM == 3 ? b[2] : 0.0, 0.0);
    G.site[n] = make_double4(sv[0], sv[1], DIM == 3 ? sv[2] : 0.0, 0.0);
    uint32_t ms[3] = {0, 0, 0};
    serial_cell<DIM>(g, G, sv, ms);
    const uint32_t c = serial_index<DIM>(G, ms);
    const uint32_t sz = G.size[c];
    if (sz < G.cap) {
        G.items[(size_t)c * G.cap + sz] = n;
        G.size[c] = sz + 1;
    } else {
        atomicOr(&A.stats->error_flags, kErrCellOverflow);
    }
    G.cell_of[n] = c;
    if (T.tag) T.tag[n] = tag_take(T);
}

// Sites and cell lists from the body positions (one thread per body).
template <int DIM>
__global__ void k_serial_build(Geometry g, Arrays A, SerialGrid G, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 b = A.body_pos[i];
    double s[3] = {b.x, b.y, b.z};
    wrap_inv<DIM>(g.L, g.invL, s);
    G.site[i] = make_double4(s[0], s[1], s[2], 0.0);
    uint32_t m[3] = {0, 0, 0};
    serial_cell<DIM>(g, G, s, m);
    const uint32_t c = serial_index<DIM>(G, m);
    G.cell_of[i] = c;
    const uint32_t k = atomicAdd(G.size + c, 1u);
    if (k < G.cap)
        G.items[(size_t)c * G.cap + k] = i;
    else
        atomicOr(&A.stats->error_flags, kErrCellOverflow);
}

// The grid's description from the host's arrays, and its contents from the body positions.
SerialGrid make_grid(int dim, const uint32_t* nc, const double* w, uint32_t cap, uint32_t* size, uint32_t* items,
                     uint32_t* cell_of, double4* site) {
    SerialGrid G{};
    uint64_t cells = 1;
    for (int k = 0; k < 3; ++k) {
        G.nc[k] = k < dim ? nc[k] : 1u;
        G.w[k] = k < dim ? w[k] : 1.0;
        cells *= G.nc[k];
    }
    G.n_cells = (uint32_t)cells;
    G.cap = cap;
    G.size = size;
    G.items = items;
    G.cell_of = cell_of;
    G.site = site;
    return G;
}

cudaError_t build_grid(int dim, const Geometry& g, const Arrays& a, const SerialGrid& G, uint32_t n, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(G.size, 0, sizeof(uint32_t) * G.n_cells, s);
    if (e != cudaSuccess || n == 0) return e;
    if (dim == 2)
        k_serial_build<2><<<(n + 255) / 256, 256, 0, s>>>(g, a, G, n);
    else
        k_serial_build<3><<<(n + 255) / 256, 256, 0, s>>>(g, a, G, n);
    return cudaGetLastError();
}
}  // namespace
}  // namespace hmc
