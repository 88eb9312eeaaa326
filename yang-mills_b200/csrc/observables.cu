// observables.cu -- SU(3) gauge observables on device lattices (compiled
// with -fmad=false): lattice-averaged rectangular Wilson loops, Polyakov
// loops, and the scalar (A1++) glueball operator basis per time slice.
//
// Every per-site quantity is the reference's closed-path holonomy
// (reference/rust/src/path_holonomy.rs:132-181) with its normalised trace
// (1/3) Tr, the trace scaled by fl(1/3) as wilson_loop does.  A rectangle's
// holonomy P C^dag D^dag is evaluated as Re Tr(P Q^dag) of its two halves
// (P: the mu then nu edges, Q = D C: the nu then mu edges), each multiplied
// left to right in traversal order with fma() chains, and a Polyakov line as
// its ordered product; results differ from the reference's single
// left-to-right chain only by rounding.  Lattice sums use fixed-order tree
// reductions (deterministic; within 1e-12 relative of the reference's
// sequential sums).  The reference checks unitarity after
// every product; here the operands' residuals are gated once per measurement
// (ym_su3_max_residuals), since a product of links within the 5e-12 gate is
// itself within it.
#include <cuda_runtime.h>

#include "su3_sites.cuh"
#include "ym_internal.hpp"

namespace ym {

namespace {

constexpr int T = kSiteThreads;
constexpr int kMaxRT = 4;                  // R, T <= 4 (loops up to 4x4)

// A walker: current site (coordinates, lex, parity).
struct Walker {
    int32_t x[4];
    int64_t lex;
    int par;
};

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

// Wilson loops: grid (site tiles, 6 planes).  Each thread: one site x, one
// plane (mu < nu), R along mu, T along nu, every (R, T) <= (rmax, tmax).
// The rectangle's holonomy (R forward mu, T forward nu, R back, T back) is
// P C^dag D^dag = P Q^dag with its two halves
//   P_{R,T} = U_mu(x)..U_mu(x+(R-1)mu) U_nu(x+R mu)..U_nu(x+R mu+(T-1)nu)
//   Q_{R,T} = U_nu(x)..U_nu(x+(T-1)nu) U_mu(x+T nu)..U_mu(x+T nu+(R-1)mu)
// each multiplied left to right in traversal order (fma chains); P grows in T from the
// mu-line A_R, Q grows in R (Q_{0,T} = the nu-line D_T), so all sixteen loops
// take 38 products instead of 160.  The four Q_{R-1,T} wait in shared memory
// between R steps, and the sixteen loop values are written straight to the
// thread's shared-memory column (fewer registers than an indexed array).  Re (1/3) Tr(P Q^dag) differs from the single-chain
// product only by rounding (<= 1e-12 relative on lattice means).
// partial[(tile * 6 + plane) * 16 + (R-1)*4 + (T-1)] = tile sum.
constexpr size_t kWilsonSmem = (size_t)kMaxRT * 9 * T * sizeof(double2);

__device__ __forceinline__ void step_walker(const ChainInfo &c, Walker &w, int mu) {
    const Nb n = step(c, w.x, w.lex, w.par, mu, +1);
    w.x[mu] = w.x[mu] == c.n[mu] - 1 ? 0 : w.x[mu] + 1;
    w.lex = n.lex;
    w.par = n.par;
}

__device__ __forceinline__ m3 link_of(const double2 *links, const ChainInfo &c, const Walker &w, int mu) {
    return load_su3(links, c, storage_index(c, w.lex, w.par), mu);
}

__device__ __forceinline__ void q_put(double2 *qs, int t, const m3 &q) {
#pragma unroll
    for (int e = 0; e < 9; ++e)
        qs[((size_t)t * 9 + e) * T + threadIdx.x] = make_double2(q.e[e / 3][e % 3].re, q.e[e / 3][e % 3].im);
}

__device__ __forceinline__ m3 q_get(const double2 *qs, int t) {
    m3 q;
#pragma unroll
    for (int e = 0; e < 9; ++e) {
        const double2 v = qs[((size_t)t * 9 + e) * T + threadIdx.x];
        q.e[e / 3][e % 3] = cmake(v.x, v.y);
    }
    return q;
}

template <int MU, int NU>
__device__ __forceinline__ void wilson_site(const double2 *links, const ChainInfo &c, const Walker &w0,
                                            int rmax, int tmax, double2 *qs, double (*vs)[T]) {
    {   // D_T, stored as Q_{0,T}
        Walker w = w0;
        m3 d;
#pragma unroll 1
        for (int t = 0; t < tmax; ++t) {
            {
                const m3 u = link_of(links, c, w, NU);
                d = t == 0 ? u : mul_fma(d, u);
                q_put(qs, t, d);
                step_walker(c, w, NU);
            }
        }
    }
    Walker wa = w0;   // x + (R-1) mu
    m3 a;
#pragma unroll 1
    for (int r = 0; r < rmax; ++r) {
        {
            const m3 ua = link_of(links, c, wa, MU);
            a = r == 0 ? ua : mul_fma(a, ua);
            Walker wq = wa;          // x + (R-1) mu, walked along nu with T
            step_walker(c, wa, MU);  // x + R mu
            Walker wp = wa;
            m3 p = a;
#pragma unroll 1
            for (int t = 0; t < tmax; ++t) {
                {
                    p = mul_fma(p, link_of(links, c, wp, NU));
                    step_walker(c, wp, NU);
                    step_walker(c, wq, NU);
                    const m3 q = mul_fma(q_get(qs, t), link_of(links, c, wq, MU));
                    q_put(qs, t, q);
                    vs[r * kMaxRT + t][threadIdx.x] = retrace_mul_adj(p, q) * (1.0 / 3.0);
                }
            }
        }
    }
}

__global__ void __launch_bounds__(T)
k_wilson_loops(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
               const double2 *__restrict__ links, int rmax, int tmax, double *__restrict__ partial) {
    extern __shared__ __align__(16) double2 qs[];
    __shared__ double vs[16][T];
    const int plane = blockIdx.y;
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t s = tile.start + threadIdx.x;
#pragma unroll
    for (int k = 0; k < 16; ++k) vs[k][threadIdx.x] = 0.0;
    if (s < c.volume) {
        const Walker w0 = walker_of(decode_storage(c, s));
        switch (plane) {
            case 0: wilson_site<0, 1>(links, c, w0, rmax, tmax, qs, vs); break;
            case 1: wilson_site<0, 2>(links, c, w0, rmax, tmax, qs, vs); break;
            case 2: wilson_site<0, 3>(links, c, w0, rmax, tmax, qs, vs); break;
            case 3: wilson_site<1, 2>(links, c, w0, rmax, tmax, qs, vs); break;
            case 4: wilson_site<1, 3>(links, c, w0, rmax, tmax, qs, vs); break;
            default: wilson_site<2, 3>(links, c, w0, rmax, tmax, qs, vs); break;
        }
    }
    double v[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = vs[k][threadIdx.x];
    block_sum16(v, partial + ((int64_t)blockIdx.x * 6 + plane) * 16);
}

// One block per (chain, value k): the chain's tile partials
// partial[tile * width + k], summed in a fixed order (thread i takes tiles
// i, i + blockDim, ... in turn, then block_reduce's tree), divided by the
// chain's count: its volume (loops) or its number of lines along `dir`
// (Polyakov, dir >= 0).  Deterministic, and parallel over the thousands of
// tiles of a large lattice.
__global__ void k_tile_mean(const double *__restrict__ partial, const int32_t *__restrict__ first,
                            const ChainInfo *__restrict__ chains, int width, int dir,
                            double *__restrict__ out) {
    const int chain = blockIdx.x, k = blockIdx.y;
    const int b = first[chain], e = first[chain + 1];
    double v = 0.0;
    for (int i = b + threadIdx.x; i < e; i += blockDim.x) {
        const double p = partial[(int64_t)i * width + k];
        v = (i == b + (int)threadIdx.x) ? p : v + p;
    }
    v = block_reduce<false>(v);
    if (threadIdx.x == 0) {
        const ChainInfo &c = chains[chain];
        const double count = dir < 0 ? (double)c.volume : (double)(c.volume / c.n[dir]);
        out[(int64_t)chain * width + k] = v / count;
    }
}

// Polyakov loop along `dir` from every site with x_dir = 0: ordered product
// of the n_dir links (polyakov_holonomy su3_lattice.rs:185-212), (1/3) Tr.
// One thread per line: line l of a chain is the l-th site with x_dir = 0 in
// lexicographic order of the other three coordinates, taken by the chain's
// first site tiles (thread = tile.start + threadIdx.x); the walk never wraps,
// so its k-th site is lex + k * stride with the parity flipped k times.  The
// links are loaded four ahead of the fma-chain products.
// partial[tile*2 + {0,1}] = tile sums of re, im (zero for tiles past the lines).
template <int DIR>
__device__ __forceinline__ cplx polyakov_line(const double2 *links, const ChainInfo &c, int64_t line) {
    int32_t x[4];
    int64_t q = line;
#pragma unroll
    for (int d = 3; d >= 0; --d) {
        if (d == DIR) {
            x[d] = 0;
        } else {
            x[d] = (int32_t)(q % c.n[d]);
            q /= c.n[d];
        }
    }
    const int64_t lex0 = ((int64_t)(x[0] * c.n[1] + x[1]) * c.n[2] + x[2]) * c.n[3] + x[3];
    const int par0 = (x[0] + x[1] + x[2] + x[3]) & 1;
    const int64_t stride = stride_of(c, DIR);
    const int n = c.n[DIR];
    m3 h;
#pragma unroll 1
    for (int k0 = 0; k0 < n; k0 += 4) {
        m3 u[4];
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (k0 + j < n) u[j] = load_su3(links, c, storage_index(c, lex0 + (k0 + j) * stride, par0 ^ ((k0 + j) & 1)), DIR);
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (k0 + j < n) h = (k0 + j == 0) ? u[j] : mul_fma(h, u[j]);
    }
    return cmake(((h.e[0][0].re + h.e[1][1].re) + h.e[2][2].re) * (1.0 / 3.0),
                 ((h.e[0][0].im + h.e[1][1].im) + h.e[2][2].im) * (1.0 / 3.0));
}

__global__ void __launch_bounds__(T)
k_polyakov(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
           const double2 *__restrict__ links, int dir, double *__restrict__ partial) {
    __shared__ double red[2][T / 32];
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t line = tile.start + threadIdx.x;
    double re = 0.0, im = 0.0;
    if (line < c.volume / c.n[dir]) {
        cplx v;
        switch (dir) {
            case 0: v = polyakov_line<0>(links, c, line); break;
            case 1: v = polyakov_line<1>(links, c, line); break;
            case 2: v = polyakov_line<2>(links, c, line); break;
            default: v = polyakov_line<3>(links, c, line); break;
        }
        re = v.re;
        im = v.im;
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

// The 1x1 loop of spatial plane (A, B) and the 2x1 loops (A, B) and (B, A)
// of one site, each as Re (1/3) Tr(P Q^dag) of the two halves of its closed
// path in traversal order (fma chains): for an R x 1 rectangle (R along M,
// one step along N) P = U_M(x)..U_M(x+(R-1)M) U_N(x+R M) and
// Q = U_N(x) U_M(x+N)..U_M(x+N+(R-1)M), 2R products instead of the single
// chain's 2R + 1.  The halves of the 1x1 loop are the corners
// K_AB = U_A(x) U_B(x+A) and K_BA, and they are the first products of the
// 2x1 loops' Q halves (Q of (A, B) is K_BA U_A(x+B+A), Q of (B, A) is
// K_AB U_B(x+A+B)), so the three loops take 8 products instead of 10 with
// every product the same.
template <int A, int B>
__device__ __forceinline__ void plane_loops(const double2 *links, const ChainInfo &c, const Walker &w0,
                                            double &plaq, double &rect_ab, double &rect_ba) {
    Walker wa = w0, wb = w0;
    step_walker(c, wa, A);
    step_walker(c, wb, B);
    Walker wab = wa;
    step_walker(c, wab, B);
    const m3 kab = mul_fma(link_of(links, c, w0, A), link_of(links, c, wa, B));
    const m3 kba = mul_fma(link_of(links, c, w0, B), link_of(links, c, wb, A));
    plaq = retrace_mul_adj(kab, kba) * (1.0 / 3.0);
    {
        const m3 qq = mul_fma(kba, link_of(links, c, wab, A));
        Walker w = wa;
        step_walker(c, w, A);
        const m3 pp = mul_fma(mul_fma(link_of(links, c, w0, A), link_of(links, c, wa, A)), link_of(links, c, w, B));
        rect_ab = retrace_mul_adj(pp, qq) * (1.0 / 3.0);
    }
    {
        const m3 qq = mul_fma(kab, link_of(links, c, wab, B));
        Walker w = wb;
        step_walker(c, w, B);
        const m3 pp = mul_fma(mul_fma(link_of(links, c, w0, B), link_of(links, c, wb, B)), link_of(links, c, w, A));
        rect_ba = retrace_mul_adj(pp, qq) * (1.0 / 3.0);
    }
}

// Scalar operator basis, per site with x3 = t: sum of Re W over the three
// 1x1 spatial orientations (0,1),(0,2),(1,2) and the six 2x1 orientations
// (0,1),(0,2),(1,0),(1,2),(2,0),(2,1) (glueball_operators.rs:24-26), summed
// in that order.
// (250 registers, two blocks per SM: 0.52 ms at 32^4; capped at three
// blocks, 168 registers with spills, 0.66 ms)
__global__ void __launch_bounds__(T)
k_operator_sites(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                 const double2 *__restrict__ links, double2 *__restrict__ site_vals) {
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t s = tile.start + threadIdx.x;
    if (s >= c.volume) return;
    const Walker w0 = walker_of(decode_storage(c, s));
    double p01, p02, p12, r01, r10, r02, r20, r12, r21;
    plane_loops<0, 1>(links, c, w0, p01, r01, r10);
    plane_loops<0, 2>(links, c, w0, p02, r02, r20);
    plane_loops<1, 2>(links, c, w0, p12, r12, r21);
    const double p = (p01 + p02) + p12;
    const double r = ((((r01 + r02) + r10) + r12) + r20) + r21;
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
    static thread_local int configured_device = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (configured_device != dev) {
        const cudaError_t err = cudaFuncSetAttribute(k_wilson_loops, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     (int)kWilsonSmem);
        if (err != cudaSuccess) return err;
        configured_device = dev;
    }
    const dim3 g((unsigned)e->n_site_tiles, 6);
    k_wilson_loops<<<g, T, kWilsonSmem, e->stream>>>(e->d_chains, e->d_site_tiles, e->d_links, rmax, tmax,
                                                      d_partial);
    k_tile_mean<<<dim3((unsigned)e->n_chains, 96), 256, 0, e->stream>>>(d_partial, e->d_site_tile_first,
                                                                       e->d_chains, 96, -1, d_out);
    return cudaGetLastError();
}

cudaError_t launch_tile_mean(ym_ensemble *e, const double *d_partial, int width, int dir, double *d_out) {
    k_tile_mean<<<dim3((unsigned)e->n_chains, (unsigned)width), 256, 0, e->stream>>>(
        d_partial, e->d_site_tile_first, e->d_chains, width, dir, d_out);
    return cudaGetLastError();
}

cudaError_t launch_polyakov(ym_ensemble *e, int dir, double *d_partial, double *d_out) {
    k_polyakov<<<(unsigned)e->n_site_tiles, T, 0, e->stream>>>(e->d_chains, e->d_site_tiles, e->d_links,
                                                              dir, d_partial);
    k_tile_mean<<<dim3((unsigned)e->n_chains, 2), 256, 0, e->stream>>>(d_partial, e->d_site_tile_first,
                                                                      e->d_chains, 2, dir, d_out);
    return cudaGetLastError();
}

cudaError_t launch_operator_basis(ym_ensemble *e, double2 *d_site_vals, const int32_t *d_slice_chain,
                                  const int32_t *d_slice_t, int64_t n_slices, double *d_plaq,
                                  double *d_rect, const double2 *links) {
    k_operator_sites<<<(unsigned)e->n_site_tiles, T, 0, e->stream>>>(e->d_chains, e->d_site_tiles,
                                                                    links ? links : e->d_links, d_site_vals);
    k_operator_reduce<<<(unsigned)n_slices, 256, 0, e->stream>>>(e->d_chains, d_slice_chain, d_slice_t,
                                                                d_site_vals, d_plaq, d_rect);
    return cudaGetLastError();
}

}  // namespace ym
