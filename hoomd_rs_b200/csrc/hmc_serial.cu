// Sweep::apply_with_filter (hoomd-mc/src/sweep.rs:159-224) for hard disks and spheres: one
// trial per body in index order, all from ONE sequential random stream
// Counter(step, substep, seed).make_rng() (index 0), each trial seeing every earlier accepted
// move. The chain is sequential by definition, so one warp runs it: the 32 lanes keep the same
// stream and trial, and each lane tests the sites of one cell of the 3^d stencil around the
// trial site (cells at least one diameter wide, kept current after every accepted move). This
// is the exact serial Markov chain on the device, not a fast path: the checkerboard sweep is.
#include <cuda_runtime.h>

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

template <int DIM>
__global__ void __launch_bounds__(32) k_serial_sphere(Geometry g, Arrays A, SerialGrid G, Pair P, Launch L,
                                                      const uint8_t* __restrict__ mask) {
    const uint32_t lane = threadIdx.x;
    if (A.stats->error_flags) return;
    Sfc64 rng = make_rng(L.step, L.substep, L.seed, 0);
    // this lane's stencil cell: radix decomposition over the distinct cells of each axis
    uint32_t len[3] = {1, 1, 1};
#pragma unroll
    for (int a = 0; a < DIM; ++a) len[a] = G.nc[a] >= 3 ? 3u : G.nc[a];
    uint32_t off[3] = {0, 0, 0}, rem = lane;
#pragma unroll
    for (int a = DIM - 1; a >= 0; --a) {
        off[a] = rem % len[a];
        rem /= len[a];
    }
    const bool lane_used = rem == 0;  // lane < prod(len)
    uint64_t accepted = 0;
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
        uint32_t m[3] = {0, 0, 0};
        serial_cell<DIM>(g, G, t, m);
        bool overlap = false;
        if (lane_used) {
            uint32_t c[3] = {0, 0, 0};
#pragma unroll
            for (int a = 0; a < DIM; ++a)
                c[a] = G.nc[a] >= 3 ? wrap_index((int)m[a] + (int)off[a] - 1, G.nc[a]) : off[a];
            const uint32_t cell = serial_index<DIM>(G, c);
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
        accepted++;
        if (lane == 0) {
            // update_body_properties: body = wrap(W1) = T, site = wrap(body)
            double sv[3] = {t[0], t[1], t[2]};
            wrap_inv<DIM>(g.L, g.invL, sv);
            A.body_pos[b] = make_double4(t[0], t[1], t[2], 0.0);
            G.site[b] = make_double4(sv[0], sv[1], sv[2], 0.0);
            uint32_t ms[3] = {0, 0, 0};
            serial_cell<DIM>(g, G, sv, ms);
            const uint32_t nc = serial_index<DIM>(G, ms), oc = G.cell_of[b];
            if (nc != oc) {
                // remove b from its old cell (last item takes its slot), append to the new one
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
        }
        __syncwarp();
        if (A.stats->error_flags) break;
    }
    if (lane == 0) {
        A.stats->accepted = accepted;
        A.stats->rechecks = 0;
    }
}

}  // namespace

cudaError_t launch_serial_sphere(int dim, const Geometry& g, const Arrays& a, const Pair& p, const Launch& l,
                                 const uint32_t* nc, const double* w, uint32_t cap, uint32_t* size, uint32_t* items,
                                 uint32_t* cell_of, double4* site, const uint8_t* mask, cudaStream_t s) {
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
    cudaError_t e = cudaMemsetAsync(size, 0, sizeof(uint32_t) * cells, s);
    if (e != cudaSuccess) return e;
    const uint32_t n = l.n_bodies;
    if (n == 0) return cudaSuccess;
    if (dim == 2) {
        k_serial_build<2><<<(n + 255) / 256, 256, 0, s>>>(g, a, G, n);
        k_serial_sphere<2><<<1, 32, 0, s>>>(g, a, G, p, l, mask);
    } else {
        k_serial_build<3><<<(n + 255) / 256, 256, 0, s>>>(g, a, G, n);
        k_serial_sphere<3><<<1, 32, 0, s>>>(g, a, G, p, l, mask);
    }
    return cudaGetLastError();
}

}  // namespace hmc
