// su3_f64.cu -- SU(3) measurement, replay and layout kernels of the FP64
// path (compiled with -fmad=false; the sweep itself is su3_metropolis.cu).
//
//   k_su3_plaquette       per-tile plaquette sums  (su3_ensemble.rs:228-259)
//   k_chain_reduce        fixed-order per-chain reductions of tile partials
//   k_su3_residuals       unitarity / determinant residuals (su3_lattice.rs:285-297)
//   k_su3_reference_*     the reference's lexicographic single-stream sweep and
//                         sequential plaquette, one thread per chain
//   k_su3_hot_start       Haar-random links
//   k_su3_{identity,from_aos,to_aos}  layout conversion, reference <-> SoA
#include <cuda_runtime.h>

#include "su3_exp.cuh"
#include "su3_haar.cuh"
#include "su3_sites.cuh"
#include "ym_internal.hpp"

namespace ym {

// ------------------------------------------------------------ reductions

// ---- the plaquette with its neighbour links staged ------------------------
// site_plaquette_sum<false> with each plane's two neighbour links,
// U_nu(x+mu) and U_mu(x+nu), copied global -> shared by cp.async one plane
// ahead, in a ring of two sets, so their latency overlaps the previous
// plane's products; the site's own links keep their cached loads (each is
// read by three planes).  The values and their order are
// site_plaquette_sum's, so the sum is bit for bit the same.  72 KB of
// staging per 128-thread block keeps three blocks per SM: 0.301 ms per
// 32^4 call against 0.324 ms unstaged (two blocks per SM, leaving more L1
// for the own links, 0.366 ms).
constexpr size_t kPlaqStageBytes = (size_t)4 * 9 * kSiteThreads * sizeof(double2);

using PlaqBuf = double2 (*)[kSiteThreads];

template <int MU, int NU>
__device__ __forceinline__ void plaq_stage(PlaqBuf b, PlaqBuf cb, const double2 *links, const ChainInfo &c,
                                           const Coord &x) {
    const Nb pm = step(c, x.x, x.lex, x.par, MU, +1);
    const Nb pn = step(c, x.x, x.lex, x.par, NU, +1);
    const double2 *pb = links + c.offset + (int64_t)(NU * 9) * c.volume + storage_index(c, pm.lex, pm.par);
    const double2 *pc = links + c.offset + (int64_t)(MU * 9) * c.volume + storage_index(c, pn.lex, pn.par);
#pragma unroll
    for (int e = 0; e < 9; ++e) {
        cp_async16(&b[e][threadIdx.x], pb + (int64_t)e * c.volume);
        cp_async16(&cb[e][threadIdx.x], pc + (int64_t)e * c.volume);
    }
    cp_async_commit();
}

__device__ __forceinline__ m3 plaq_staged(const PlaqBuf b) {
    m3 o;
#pragma unroll
    for (int e = 0; e < 9; ++e) {
        const double2 v = b[e][threadIdx.x];
        o.e[e / 3][e % 3] = cmake(v.x, v.y);
    }
    return o;
}

// Plane (MU, NU) from one set, then (HAS_NEXT) plane (NMU, NNU) staged into
// the same set.
template <int MU, int NU, bool HAS_NEXT, int NMU, int NNU>
__device__ __forceinline__ double plaq_plane(PlaqBuf b, PlaqBuf cb, const double2 *links, const ChainInfo &c,
                                             const Coord &x, int64_t s) {
    if (HAS_NEXT) cp_async_wait_one(); else cp_async_wait_all();
    m3 p = mul_fma(load_su3(links, c, s, MU), plaq_staged(b));
    p = mul_adj_fma(p, plaq_staged(cb));
    if (HAS_NEXT) plaq_stage<NMU, NNU>(b, cb, links, c, x);
    return retrace_mul_adj(p, load_su3(links, c, s, NU)) / 3.0;
}

__device__ __forceinline__ double site_plaquette_sum_staged(const double2 *links, const ChainInfo &c, int64_t s,
                                                            double2 *stage) {
    const PlaqBuf b0 = reinterpret_cast<PlaqBuf>(stage);
    const PlaqBuf c0 = reinterpret_cast<PlaqBuf>(stage + 9 * kSiteThreads);
    const PlaqBuf b1 = reinterpret_cast<PlaqBuf>(stage + 18 * kSiteThreads);
    const PlaqBuf c1 = reinterpret_cast<PlaqBuf>(stage + 27 * kSiteThreads);
    const Coord x = decode_storage(c, s);
    plaq_stage<0, 1>(b0, c0, links, c, x);
    plaq_stage<0, 2>(b1, c1, links, c, x);
    double v = plaq_plane<0, 1, true, 0, 3>(b0, c0, links, c, x, s);
    v = v + plaq_plane<0, 2, true, 1, 2>(b1, c1, links, c, x, s);
    v = v + plaq_plane<0, 3, true, 1, 3>(b0, c0, links, c, x, s);
    v = v + plaq_plane<1, 2, true, 2, 3>(b1, c1, links, c, x, s);
    v = v + plaq_plane<1, 3, false, 0, 0>(b0, c0, links, c, x, s);
    v = v + plaq_plane<2, 3, false, 0, 0>(b1, c1, links, c, x, s);
    return v;
}

// One 1024-thread block per chain: the plaquette shares the last three
// sub-sweeps of a sweep wrote for the chain's CTAs (planes (0,1); (0,2),
// (1,2); (0,3), (1,3), (2,3)), summed CTA by CTA in a fixed order, then the
// average plaquette sum / (6 V).
__global__ void k_chain_reduce_sweep(const double *__restrict__ tr_partial, int64_t ctas,
                                     const int32_t *__restrict__ cta_range, const ChainInfo *__restrict__ chains,
                                     double *__restrict__ out) {
    const int chain = blockIdx.x;
    const int b = cta_range[2 * chain], e = cta_range[2 * chain + 1];
    double v = 0.0;
    for (int i = b + threadIdx.x; i < e; i += blockDim.x) {
        const double p = (tr_partial[i] + tr_partial[ctas + i]) + tr_partial[2 * ctas + i];
        v = (i == b + (int)threadIdx.x) ? p : v + p;
    }
    v = block_reduce<false>(v);
    if (threadIdx.x == 0) out[chain] = v / (6.0 * (double)chains[chain].volume);
}

// Sum of the six plaquette values (1/3) Re Tr P of each site, site order
// (mu, nu) = (0,1),(0,2),(0,3),(1,2),(1,3),(2,3), per tile; tiles visited in
// serpentine order.
__global__ void __launch_bounds__(kSiteThreads)
k_su3_plaquette(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                const double2 *__restrict__ links, double *__restrict__ partial) {
    const int64_t tix = serpentine_tile(blockIdx.x, gridDim.x);
    const Tile tile = tiles[tix];
    const ChainInfo c = chains[tile.chain];
    const int64_t s = tile.start + threadIdx.x;
    extern __shared__ __align__(16) double2 plaq_stage_mem[];
    double v = 0.0;
    if (s < c.volume) v = site_plaquette_sum_staged(links, c, s, plaq_stage_mem);
    v = block_reduce<false>(v);
    if (threadIdx.x == 0) partial[tix] = v;
}

// One block per chain: fixed-order reduction of the chain's tile partials.
// mode 0: out = sum / scale;  mode 1: out = max.
__global__ void k_chain_reduce(const double *__restrict__ partial, const int32_t *__restrict__ first,
                               const ChainInfo *__restrict__ chains, double *__restrict__ out,
                               int mode, double per_site) {
    const int chain = blockIdx.x;
    const int b = first[chain], e = first[chain + 1];
    double v = 0.0;
    for (int i = b + threadIdx.x; i < e; i += blockDim.x) {
        const double p = partial[i];
        v = (i == b + (int)threadIdx.x) ? p : (mode ? fmax(v, p) : v + p);
    }
    v = mode ? block_reduce<true>(v) : block_reduce<false>(v);
    if (threadIdx.x == 0)
        out[chain] = mode ? v : v / (per_site * (double)chains[chain].volume);
}

__device__ __forceinline__ double cabs_(cplx z) { return hypot(z.re, z.im); }

// Mat3::determinant (su3.rs:175-189).
__device__ __forceinline__ cplx det3(const m3 &m) {
    const cplx t1 = cmul(m.e[0][0], csub(cmul(m.e[1][1], m.e[2][2]), cmul(m.e[1][2], m.e[2][1])));
    const cplx t2 = cmul(m.e[0][1], csub(cmul(m.e[1][0], m.e[2][2]), cmul(m.e[1][2], m.e[2][0])));
    const cplx t3 = cmul(m.e[0][2], csub(cmul(m.e[1][0], m.e[2][1]), cmul(m.e[1][1], m.e[2][0])));
    return cadd(csub(t1, t2), t3);
}

__device__ __forceinline__ double max_abs_minus_identity(const m3 &m) {
    double r = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            r = fmax(r, cabs_(csub(m.e[i][j], cmake(i == j ? 1.0 : 0.0, 0.0))));
    return r;
}

// Per tile: max unitarity residual into partial, max determinant residual
// into partial2 (Mat3::unitarity_residual / determinant_residual).
__global__ void __launch_bounds__(kSiteThreads)
k_su3_residuals(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                const double2 *__restrict__ links, double *__restrict__ partial,
                double *__restrict__ partial2) {
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t s = tile.start + threadIdx.x;
    double ru = 0.0, rd = 0.0;
    if (s < c.volume) {
#pragma unroll 1
        for (int mu = 0; mu < 4; ++mu) {
            const m3 u = load_su3(links, c, s, mu);
            const double left = max_abs_minus_identity(adj_mul(u, u));
            const double right = max_abs_minus_identity(mul_adj(u, u));
            ru = fmax(ru, fmax(left, right));
            const double dd = cabs_(csub(det3(u), cmake(1.0, 0.0)));
            const double dg = cabs_(csub(det3(adj(u)), cmake(1.0, 0.0)));
            rd = fmax(rd, fmax(dd, dg));
        }
    }
    ru = block_reduce<true>(ru);
    __syncthreads();
    rd = block_reduce<true>(rd);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = ru;
        partial2[blockIdx.x] = rd;
    }
}

// ------------------------------------------------------------ reference order

__device__ __forceinline__ int64_t lex_of(const ChainInfo &c, const int *x) {
    return ((int64_t)(x[0] * c.n[1] + x[1]) * c.n[2] + x[2]) * c.n[3] + x[3];
}

__device__ __forceinline__ m3 link_at(const double2 *links, const ChainInfo &c, const int *x, int mu) {
    const int64_t lex = lex_of(c, x);
    const int par = (x[0] + x[1] + x[2] + x[3]) & 1;
    return load_su3_rw(links, c, storage_index(c, lex, par), mu);
}

// local_link_action_with_value (su3_ensemble.rs:261-307) without the checks.
__device__ double reference_local_action(const double2 *links, const ChainInfo &c, const int *x,
                                         int mu, const m3 &val) {
    double sum = 0.0;
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == mu) continue;
        int xm[4] = {x[0], x[1], x[2], x[3]}, xn[4] = {x[0], x[1], x[2], x[3]};
        xm[mu] = (x[mu] + 1) % c.n[mu];
        xn[nu] = (x[nu] + 1) % c.n[nu];
        m3 f = mul(val, link_at(links, c, xm, nu));
        f = mul_adj(f, link_at(links, c, xn, mu));
        const double tf = retrace_mul_adj(f, link_at(links, c, x, nu));
        int bx[4] = {x[0], x[1], x[2], x[3]};
        bx[nu] = x[nu] == 0 ? c.n[nu] - 1 : x[nu] - 1;
        int bxm[4] = {bx[0], bx[1], bx[2], bx[3]};
        bxm[mu] = (bx[mu] + 1) % c.n[mu];
        m3 b = mul(link_at(links, c, bx, mu), link_at(links, c, bxm, nu));
        b = mul_adj(b, val);
        const double tb = retrace_mul_adj(b, link_at(links, c, bx, nu));
        sum += 1.0 - tf / 3.0;
        sum += 1.0 - tb / 3.0;
    }
    return c.beta * sum;
}

__global__ void k_su3_reference_sweeps(const ChainInfo *__restrict__ chains, int n_chains,
                                       double2 *links, double angle, uint64_t *rng, int64_t n_sweeps,
                                       unsigned long long *prop, unsigned long long *acc) {
    const int chain = blockIdx.x * blockDim.x + threadIdx.x;
    if (chain >= n_chains) return;
    const ChainInfo c = chains[chain];
    uint64_t state = rng[chain];
    unsigned long long np = 0, na = 0;
    for (int64_t sw = 0; sw < n_sweeps; ++sw) {
        int x[4];
        for (x[0] = 0; x[0] < c.n[0]; ++x[0])
            for (x[1] = 0; x[1] < c.n[1]; ++x[1])
                for (x[2] = 0; x[2] < c.n[2]; ++x[2])
                    for (x[3] = 0; x[3] < c.n[3]; ++x[3])
                        for (int mu = 0; mu < 4; ++mu)
                            for (int g = 0; g < 8; ++g) {
                                state += kGolden;
                                const double theta = grid_angle(mix64(state), angle);
                                const m3 rot = generator_rotation_dense(g, theta);
                                const m3 old = link_at(links, c, x, mu);
                                const m3 cand = mul(rot, old);
                                const double d = reference_local_action(links, c, x, mu, cand) -
                                                 reference_local_action(links, c, x, mu, old);
                                const double a = exp(-fmax(d, 0.0));
                                state += kGolden;
                                const double u = unit_from(mix64(state));
                                np++;
                                if (u < a) {
                                    const int64_t lex = lex_of(c, x);
                                    store_su3(links, c, storage_index(c, lex, (x[0] + x[1] + x[2] + x[3]) & 1),
                                              mu, cand);
                                    na++;
                                }
                            }
    }
    rng[chain] = state;
    prop[chain] = np;
    acc[chain] = na;
}

// average_plaquette in the reference's sequential order (su3_ensemble.rs:228-259).
__global__ void k_su3_reference_plaquette(const ChainInfo *__restrict__ chains, int n_chains,
                                          const double2 *links, double *out) {
    const int chain = blockIdx.x * blockDim.x + threadIdx.x;
    if (chain >= n_chains) return;
    const ChainInfo c = chains[chain];
    double sum = 0.0;
    int64_t count = 0;
    int x[4];
    for (x[0] = 0; x[0] < c.n[0]; ++x[0])
        for (x[1] = 0; x[1] < c.n[1]; ++x[1])
            for (x[2] = 0; x[2] < c.n[2]; ++x[2])
                for (x[3] = 0; x[3] < c.n[3]; ++x[3])
                    for (int mu = 0; mu < 4; ++mu)
                        for (int nu = mu + 1; nu < 4; ++nu) {
                            int xm[4] = {x[0], x[1], x[2], x[3]}, xn[4] = {x[0], x[1], x[2], x[3]};
                            xm[mu] = (x[mu] + 1) % c.n[mu];
                            xn[nu] = (x[nu] + 1) % c.n[nu];
                            m3 p = mul(link_at(links, c, x, mu), link_at(links, c, xm, nu));
                            p = mul_adj(p, link_at(links, c, xn, mu));
                            sum += retrace_mul_adj(p, link_at(links, c, x, nu)) / 3.0;
                            count++;
                        }
    out[chain] = sum / (double)count;
}

// ------------------------------------------------------------ hot start


__global__ void __launch_bounds__(kSiteThreads)
k_su3_hot_start(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                double2 *__restrict__ links) {
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t s = tile.start + threadIdx.x;
    if (s >= c.volume) return;
    const Coord x = decode_storage(c, s);
    const uint64_t base = splitmix_at(c.seed ^ kHotStartDomain, 0);
#pragma unroll 1
    for (int mu = 0; mu < 4; ++mu)
        store_su3(links, c, s, mu, haar_su3(splitmix_at(base, (uint64_t)(4 * x.lex + mu))));
}

cudaError_t launch_su3_hot_start(ym_ensemble *e) {
    k_su3_hot_start<<<(unsigned)e->n_site_tiles, kSiteThreads, 0, e->stream>>>(
        e->d_chains, e->d_site_tiles, e->d_links);
    return cudaGetLastError();
}

// ------------------------------------------------------------ layout

// Every chain at once: blockIdx.y picks the chain, the blocks along x
// stride over its 36 V entries.
__global__ void k_su3_identity(const ChainInfo *__restrict__ chains, double2 *links) {
    const ChainInfo c = chains[blockIdx.y];
    const int64_t n = 36 * c.volume;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int entry = (int)((i / c.volume) % 9);
        links[c.offset + i] = make_double2((entry == 0 || entry == 4 || entry == 8) ? 1.0 : 0.0, 0.0);
    }
}

// staging holds the reference AoS image: link = lex*4+mu, 18 doubles.
__global__ void k_su3_from_aos(const ChainInfo *__restrict__ chains, int chain, double2 *links,
                               const double2 *__restrict__ staging) {
    const ChainInfo c = chains[chain];
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < c.volume;
         s += (int64_t)gridDim.x * blockDim.x) {
        const Coord x = decode_storage(c, s);
        for (int mu = 0; mu < 4; ++mu) {
            const double2 *src = staging + (x.lex * 4 + mu) * 9;
            double2 *dst = links + c.offset + (int64_t)(mu * 9) * c.volume + s;
            for (int e = 0; e < 9; ++e) dst[(int64_t)e * c.volume] = src[e];
        }
    }
}

__global__ void k_su3_to_aos(const ChainInfo *__restrict__ chains, int chain,
                             const double2 *__restrict__ links, double2 *staging) {
    const ChainInfo c = chains[chain];
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < c.volume;
         s += (int64_t)gridDim.x * blockDim.x) {
        const Coord x = decode_storage(c, s);
        for (int mu = 0; mu < 4; ++mu) {
            double2 *dst = staging + (x.lex * 4 + mu) * 9;
            const double2 *src = links + c.offset + (int64_t)(mu * 9) * c.volume + s;
            for (int e = 0; e < 9; ++e) dst[e] = src[(int64_t)e * c.volume];
        }
    }
}

// ------------------------------------------------------------ launchers

static int grid_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b > 148 * 16) b = 148 * 16;
    return (int)(b < 1 ? 1 : b);
}

cudaError_t launch_su3_identity(ym_ensemble *e) {
    int64_t vmax = 0;
    for (const ChainInfo &c : e->chains) vmax = c.volume > vmax ? c.volume : vmax;
    // one launch per 65,535 chains (the grid's y limit)
    for (int64_t first = 0; first < e->n_chains; first += 65535) {
        const int64_t count = e->n_chains - first < 65535 ? e->n_chains - first : 65535;
        const int64_t bx = (grid_for(36 * vmax, 256) + count - 1) / count;   // about grid_for's total
        k_su3_identity<<<dim3((unsigned)(bx < 1 ? 1 : bx), (unsigned)count), 256, 0, e->stream>>>(
            e->d_chains + first, e->d_links);
    }
    return cudaGetLastError();
}

cudaError_t launch_su3_from_aos(ym_ensemble *e, int64_t chain) {
    k_su3_from_aos<<<grid_for(e->chains[chain].volume, 128), 128, 0, e->stream>>>(
        e->d_chains, (int)chain, e->d_links, reinterpret_cast<const double2 *>(e->d_staging));
    return cudaGetLastError();
}

cudaError_t launch_su3_to_aos(ym_ensemble *e, int64_t chain) {
    k_su3_to_aos<<<grid_for(e->chains[chain].volume, 128), 128, 0, e->stream>>>(
        e->d_chains, (int)chain, e->d_links, reinterpret_cast<double2 *>(e->d_staging));
    return cudaGetLastError();
}

// Appends the per-chain results to row *counter of a device series and
// advances the counter (one block; replayable inside a graph).
__global__ void k_store_series(const double *__restrict__ result, double *__restrict__ series,
                               uint64_t *__restrict__ counter, int n_chains) {
    const uint64_t row = *counter;
    for (int c = threadIdx.x; c < n_chains; c += blockDim.x) series[row * n_chains + c] = result[c];
    __syncthreads();
    if (threadIdx.x == 0) *counter = row + 1;
}

// dst[row * n + i] = src[i] for row = *counter; advance: *counter = row + 1
// (one block; replayable inside a graph).
__global__ void k_store_rows(const double *__restrict__ src, int64_t n, double *__restrict__ dst,
                             uint64_t *__restrict__ counter, int advance) {
    const uint64_t row = *counter;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) dst[row * n + i] = src[i];
    __syncthreads();
    if (advance && threadIdx.x == 0) *counter = row + 1;
}

cudaError_t launch_store_rows(cudaStream_t st, const double *src, int64_t n, double *dst,
                              uint64_t *counter, int advance) {
    k_store_rows<<<1, 256, 0, st>>>(src, n, dst, counter, advance);
    return cudaGetLastError();
}

cudaError_t launch_store_series(ym_ensemble *e, double *series, uint64_t *counter) {
    k_store_series<<<1, 256, 0, e->stream>>>(e->d_result, series, counter, (int)e->n_chains);
    return cudaGetLastError();
}

cudaError_t launch_chain_reduce(ym_ensemble *e, const double *partial, double *out, int mode,
                                double per_site) {
    k_chain_reduce<<<(unsigned)e->n_chains, 256, 0, e->stream>>>(
        partial, e->d_site_tile_first, e->d_chains, out, mode, per_site);
    return cudaGetLastError();
}

cudaError_t launch_su3_plaquette(ym_ensemble *e) {
    static thread_local int configured_device = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (configured_device != dev) {
        cudaError_t err = cudaFuncSetAttribute(k_su3_plaquette, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)kPlaqStageBytes);
        if (err != cudaSuccess) return err;
        configured_device = dev;
    }
    k_su3_plaquette<<<(unsigned)e->n_site_tiles, kSiteThreads, kPlaqStageBytes, e->stream>>>(
        e->d_chains, e->d_site_tiles, e->d_links, e->d_partial);
    k_chain_reduce<<<(unsigned)e->n_chains, 256, 0, e->stream>>>(
        e->d_partial, e->d_site_tile_first, e->d_chains, e->d_result, 0, 6.0);
    return cudaGetLastError();
}

cudaError_t launch_su3_plaquette_from_sweep(ym_ensemble *e, const double *tr_partial) {
    const SweepLayout &L = e->layouts[e->sweep_layout];
    if (!L.d_chain_ctas) return cudaErrorInvalidValue;
    k_chain_reduce_sweep<<<(unsigned)e->n_chains, 1024, 0, e->stream>>>(tr_partial, L.ctas, L.d_chain_ctas,
                                                                         e->d_chains, e->d_result);
    return cudaGetLastError();
}

cudaError_t launch_su3_residuals(ym_ensemble *e) {
    k_su3_residuals<<<(unsigned)e->n_site_tiles, kSiteThreads, 0, e->stream>>>(
        e->d_chains, e->d_site_tiles, e->d_links, e->d_partial, e->d_partial2);
    k_chain_reduce<<<(unsigned)e->n_chains, 256, 0, e->stream>>>(
        e->d_partial, e->d_site_tile_first, e->d_chains, e->d_result, 1, 1.0);
    k_chain_reduce<<<(unsigned)e->n_chains, 256, 0, e->stream>>>(
        e->d_partial2, e->d_site_tile_first, e->d_chains, e->d_result2, 1, 1.0);
    return cudaGetLastError();
}

cudaError_t launch_su3_reference_sweeps(ym_ensemble *e, double angle, int64_t n_sweeps) {
    const int threads = 32;
    const int blocks = (int)((e->n_chains + threads - 1) / threads);
    k_su3_reference_sweeps<<<blocks, threads, 0, e->stream>>>(
        e->d_chains, (int)e->n_chains, e->d_links, angle, e->d_rng, n_sweeps, e->d_ref_counts,
        e->d_ref_counts + e->n_chains);
    return cudaGetLastError();
}

cudaError_t launch_su3_reference_plaquette(ym_ensemble *e) {
    const int threads = 32;
    const int blocks = (int)((e->n_chains + threads - 1) / threads);
    k_su3_reference_plaquette<<<blocks, threads, 0, e->stream>>>(e->d_chains, (int)e->n_chains,
                                                                 e->d_links, e->d_result);
    return cudaGetLastError();
}

}  // namespace ym
