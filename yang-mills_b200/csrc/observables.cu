// observables.cu -- SU(3) gauge observables on device lattices (compiled
// with -fmad=false): lattice-averaged rectangular Wilson loops, Polyakov
// loops, and the scalar (A1++) glueball operator basis per time slice.
//
// Every per-site quantity is the reference's closed-path holonomy: segments
// multiplied left to right in traversal order starting from the identity,
// forward steps U_mu(x), backward steps U_mu(x-mu)^dag
// (reference/rust/src/path_holonomy.rs:132-181), normalised trace
// (1/3) Tr with the trace scaled by fl(1/3) as wilson_loop does.  Lattice
// sums use fixed-order tree reductions (deterministic; within 1e-12 relative
// of the reference's sequential sums).  The reference checks unitarity after
// every product; here the operands' residuals are gated once per measurement
// (ym_su3_max_residuals), since a product of links within the 5e-12 gate is
// itself within it.
#include <cuda_runtime.h>

#include "ym_internal.hpp"

namespace ym {

namespace {

constexpr int T = kSiteThreads;
constexpr int kMaxRT = 4;                  // R, T <= 4 (loops up to 4x4)

__device__ __forceinline__ m3 link_at_nb(const double2 *links, const ChainInfo &c, const Nb &n,
                                         int mu) {
    return load_su3(links, c, storage_index(c, n.lex, n.par), mu);
}

// A walker: current site (coordinates, lex, parity) and the holonomy so far.
struct Walker {
    int32_t x[4];
    int64_t lex;
    int par;
};

__device__ __forceinline__ void walk_forward(const double2 *links, const ChainInfo &c, Walker &w,
                                             int mu, m3 &h, bool &first) {
    const m3 u = load_su3(links, c, storage_index(c, w.lex, w.par), mu);
    h = first ? u : mul(h, u);
    first = false;
    const Nb n = step(c, w.x, w.lex, w.par, mu, +1);
    w.x[mu] = w.x[mu] == c.n[mu] - 1 ? 0 : w.x[mu] + 1;
    w.lex = n.lex;
    w.par = n.par;
}

__device__ __forceinline__ void walk_backward(const double2 *links, const ChainInfo &c, Walker &w,
                                              int mu, m3 &h, bool &first) {
    const Nb n = step(c, w.x, w.lex, w.par, mu, -1);
    w.x[mu] = w.x[mu] == 0 ? c.n[mu] - 1 : w.x[mu] - 1;
    w.lex = n.lex;
    w.par = n.par;
    const m3 u = load_su3(links, c, storage_index(c, w.lex, w.par), mu);
    h = first ? adj(u) : mul_adj(h, u);
    first = false;
}

// Re (1/3) Tr of a holonomy: Mat3::trace then Complex64::scale(1.0/3.0).
__device__ __forceinline__ double retrace_third(const m3 &h) {
    return ((h.e[0][0].re + h.e[1][1].re) + h.e[2][2].re) * (1.0 / 3.0);
}

// Closed rectangle: R forward mu, T forward nu, R backward mu, T backward nu
// (rectangular_path path_holonomy.rs:219-260) from site (x, lex, par).
__device__ __forceinline__ double rectangle(const double2 *links, const ChainInfo &c,
                                            const Walker &start, int mu, int nu, int r, int t) {
    Walker w = start;
    m3 h;
    bool first = true;
    for (int i = 0; i < r; ++i) walk_forward(links, c, w, mu, h, first);
    for (int i = 0; i < t; ++i) walk_forward(links, c, w, nu, h, first);
    for (int i = 0; i < r; ++i) walk_backward(links, c, w, mu, h, first);
    for (int i = 0; i < t; ++i) walk_backward(links, c, w, nu, h, first);
    return retrace_third(h);
}

__device__ __forceinline__ Walker walker_of(const Coord &x) {
    Walker w;
#pragma unroll
    for (int d = 0; d < 4; ++d) w.x[d] = x.x[d];
    w.lex = x.lex;
    w.par = x.par;
    return w;
}

// Block sum of 16 values per thread into out[16] (thread 0 writes).
__device__ __forceinline__ void block_sum16(double v[16], double *out) {
    __shared__ double red[16][T / 32];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        double a = v[k];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) a += __shfl_down_sync(0xffffffffu, a, off);
        if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = a;
    }
    __syncthreads();
    if (threadIdx.x < 16) {
        double a = red[threadIdx.x][0];
        for (int w = 1; w < T / 32; ++w) a += red[threadIdx.x][w];
        out[threadIdx.x] = a;
    }
}

// Wilson loops: grid (site tiles, 6 planes).  Each thread: one site, one
// plane (mu < nu), R along mu, T along nu, every (R, T) <= (rmax, tmax).
// partial[(tile * 6 + plane) * 16 + (R-1)*4 + (T-1)] = tile sum.
__global__ void __launch_bounds__(T)
k_wilson_loops(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
               const double2 *__restrict__ links, int rmax, int tmax, double *__restrict__ partial) {
    const int plane = blockIdx.y;
    const int mu = plane < 3 ? 0 : (plane < 5 ? 1 : 2);
    const int nu = plane < 3 ? plane + 1 : (plane < 5 ? plane - 1 : 3);
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t s = tile.start + threadIdx.x;
    double v[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = 0.0;
    if (s < c.volume) {
        const Walker w0 = walker_of(decode_storage(c, s));
        for (int r = 1; r <= rmax; ++r)
            for (int t = 1; t <= tmax; ++t) {
                const double val = rectangle(links, c, w0, mu, nu, r, t);
#pragma unroll
                for (int k = 0; k < 16; ++k)
                    if (k == (r - 1) * 4 + (t - 1)) v[k] = val;
            }
    }
    block_sum16(v, partial + ((int64_t)blockIdx.x * 6 + plane) * 16);
}

// Per chain: fixed-order sums over the chain's tiles -> mean over sites.
__global__ void k_wilson_reduce(const double *__restrict__ partial, const int32_t *__restrict__ first,
                                const ChainInfo *__restrict__ chains, double *__restrict__ out) {
    const int chain = blockIdx.x;
    const int k = threadIdx.x;          // plane*16 + rt, 96 threads
    if (k >= 96) return;
    double a = 0.0;
    for (int i = first[chain]; i < first[chain + 1]; ++i) a = (i == first[chain]) ? partial[(int64_t)i * 96 + k] : a + partial[(int64_t)i * 96 + k];
    out[(int64_t)chain * 96 + k] = a / (double)chains[chain].volume;
}

// Polyakov loop along `dir` from every site with x_dir = 0: ordered product
// of the n_dir links (polyakov_holonomy su3_lattice.rs:185-212), (1/3) Tr.
// partial[tile*2 + {0,1}] = tile sums of re, im.
__global__ void __launch_bounds__(T)
k_polyakov(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
           const double2 *__restrict__ links, int dir, double *__restrict__ partial) {
    __shared__ double red[2][T / 32];
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t s = tile.start + threadIdx.x;
    double re = 0.0, im = 0.0;
    if (s < c.volume) {
        const Coord x = decode_storage(c, s);
        if (x.x[dir] == 0) {
            Walker w = walker_of(x);
            m3 h;
            bool first = true;
            for (int k = 0; k < c.n[dir]; ++k) walk_forward(links, c, w, dir, h, first);
            re = ((h.e[0][0].re + h.e[1][1].re) + h.e[2][2].re) * (1.0 / 3.0);
            im = ((h.e[0][0].im + h.e[1][1].im) + h.e[2][2].im) * (1.0 / 3.0);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        re += __shfl_down_sync(0xffffffffu, re, off);
        im += __shfl_down_sync(0xffffffffu, im, off);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = re;
        red[1][threadIdx.x >> 5] = im;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double a = red[threadIdx.x][0];
        for (int w = 1; w < T / 32; ++w) a += red[threadIdx.x][w];
        partial[(int64_t)blockIdx.x * 2 + threadIdx.x] = a;
    }
}

__global__ void k_polyakov_reduce(const double *__restrict__ partial, const int32_t *__restrict__ first,
                                  const ChainInfo *__restrict__ chains, int dir, double *__restrict__ out) {
    const int chain = blockIdx.x;
    const int k = threadIdx.x;
    if (k >= 2) return;
    double a = 0.0;
    for (int i = first[chain]; i < first[chain + 1]; ++i) a = (i == first[chain]) ? partial[(int64_t)i * 2 + k] : a + partial[(int64_t)i * 2 + k];
    const double starts = (double)(chains[chain].volume / chains[chain].n[dir]);
    out[(int64_t)chain * 2 + k] = a / starts;
}

// Scalar operator basis, per site with x3 = t: sum of Re W over the three
// 1x1 spatial orientations (0,1),(0,2),(1,2) and the six 2x1 orientations
// (0,1),(0,2),(1,0),(1,2),(2,0),(2,1) (glueball_operators.rs:24-26).
__global__ void __launch_bounds__(T)
k_operator_sites(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                 const double2 *__restrict__ links, double2 *__restrict__ site_vals) {
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t s = tile.start + threadIdx.x;
    if (s >= c.volume) return;
    const Walker w0 = walker_of(decode_storage(c, s));
    const int po[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    const int ro[6][2] = {{0, 1}, {0, 2}, {1, 0}, {1, 2}, {2, 0}, {2, 1}};
    double p = 0.0, r = 0.0;
    for (int o = 0; o < 3; ++o) {
        const double v = rectangle(links, c, w0, po[o][0], po[o][1], 1, 1);
        p = o == 0 ? v : p + v;
    }
    for (int o = 0; o < 6; ++o) {
        const double v = rectangle(links, c, w0, ro[o][0], ro[o][1], 2, 1);
        r = o == 0 ? v : r + v;
    }
    // indexed by the chain's storage slot
    site_vals[c.offset / 36 + s] = make_double2(p, r);
}

// One block per (chain, time slice): fixed-order sum over the slice's
// spatial sites, mean = sum / count (count = 3 V_s and 6 V_s).
__global__ void k_operator_reduce(const ChainInfo *__restrict__ chains, const int32_t *__restrict__ slice_chain,
                                  const int32_t *__restrict__ slice_t, const double2 *__restrict__ site_vals,
                                  double *__restrict__ out_plaq, double *__restrict__ out_rect) {
    __shared__ double red[2][8];
    const int slice = blockIdx.x;
    const ChainInfo c = chains[slice_chain[slice]];
    const int t = slice_t[slice];
    const int64_t vs = (int64_t)c.n[0] * c.n[1] * c.n[2];
    double p = 0.0, r = 0.0;
    bool first = true;
    for (int64_t i = threadIdx.x; i < vs; i += blockDim.x) {
        const int64_t lex = i * c.n[3] + t;
        int32_t x[4];
        int64_t q = i;
        x[2] = (int32_t)(q % c.n[2]); q /= c.n[2];
        x[1] = (int32_t)(q % c.n[1]);
        x[0] = (int32_t)(q / c.n[1]);
        x[3] = t;
        const int par = (x[0] + x[1] + x[2] + x[3]) & 1;
        const double2 v = site_vals[c.offset / 36 + storage_index(c, lex, par)];
        p = first ? v.x : p + v.x;
        r = first ? v.y : r + v.y;
        first = false;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        p += __shfl_down_sync(0xffffffffu, p, off);
        r += __shfl_down_sync(0xffffffffu, r, off);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = p;
        red[1][threadIdx.x >> 5] = r;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = red[0][0], b = red[1][0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            a += red[0][w];
            b += red[1][w];
        }
        out_plaq[slice] = a / (double)(3 * vs);
        out_rect[slice] = b / (double)(6 * vs);
    }
}

}  // namespace

cudaError_t launch_wilson_loops(ym_ensemble *e, int rmax, int tmax, double *d_partial, double *d_out) {
    const dim3 g((unsigned)e->n_site_tiles, 6);
    k_wilson_loops<<<g, T, 0, e->stream>>>(e->d_chains, e->d_site_tiles, e->d_links, rmax, tmax, d_partial);
    k_wilson_reduce<<<(unsigned)e->n_chains, 96, 0, e->stream>>>(d_partial, e->d_site_tile_first,
                                                                e->d_chains, d_out);
    return cudaGetLastError();
}

cudaError_t launch_polyakov(ym_ensemble *e, int dir, double *d_partial, double *d_out) {
    k_polyakov<<<(unsigned)e->n_site_tiles, T, 0, e->stream>>>(e->d_chains, e->d_site_tiles, e->d_links,
                                                              dir, d_partial);
    k_polyakov_reduce<<<(unsigned)e->n_chains, 32, 0, e->stream>>>(d_partial, e->d_site_tile_first,
                                                                  e->d_chains, dir, d_out);
    return cudaGetLastError();
}

cudaError_t launch_operator_basis(ym_ensemble *e, double2 *d_site_vals, const int32_t *d_slice_chain,
                                  const int32_t *d_slice_t, int64_t n_slices, double *d_plaq,
                                  double *d_rect) {
    k_operator_sites<<<(unsigned)e->n_site_tiles, T, 0, e->stream>>>(e->d_chains, e->d_site_tiles,
                                                                    e->d_links, d_site_vals);
    k_operator_reduce<<<(unsigned)n_slices, 256, 0, e->stream>>>(e->d_chains, d_slice_chain, d_slice_t,
                                                                d_site_vals, d_plaq, d_rect);
    return cudaGetLastError();
}

}  // namespace ym
