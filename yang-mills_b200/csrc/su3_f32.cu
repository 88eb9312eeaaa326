// su3_f32.cu -- SU(3) links in binary32 two-row ("12-real") storage.
//
// Storage: the first two rows of every link, 6 complex floats = 48 bytes;
// the third row is rebuilt on load as the conjugate cross product
// conj(row0 x row1), which is exact for a unitary matrix with det 1.  Plane
// (mu*6 + e) holds entry e (row-major over rows 0-1) of every site as a
// float2, so a warp reads 256 contiguous bytes per entry.
//
// Arithmetic of the sub-sweep (fast mode; fused multiply-adds allowed):
// the staple sum and the candidate rows are binary32; the action change
// dS = (beta/3)(ReTr(U A) - ReTr(U' A)) and the accept test
// u < exp(-max(dS, 0)) are evaluated in binary64 from the stored values.  The
// update rule, stream words and generator order are the FP64 path's.  The
// plaquette and every conversion to FP64 are binary64 products of the
// stored values; k_f32_reunitarize restores unitarity in binary64
// (Gram-Schmidt on rows 0-1) and rounds back once per sweep.
#include <cuda_runtime.h>

#include "su3_f32.cuh"
#include "su3_haar.cuh"
#include "ym_internal.hpp"

namespace ym {

namespace {

constexpr int T = kSweepThreads;
using namespace f32;

#ifndef YM_F32_MIN_BLOCKS
#define YM_F32_MIN_BLOCKS 4
#endif

template <int MU>
__global__ void __launch_bounds__(T, YM_F32_MIN_BLOCKS)
k_f32_metropolis(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                 float2 *__restrict__ links, int parity, double angle, int uniform,
                 const uint64_t *__restrict__ sweep_ptr, unsigned long long *__restrict__ accepts,
                 int reverse) {
    __shared__ __align__(16) float2 stage[18][T];   // 18 KB: three staged factors
    const StageF<T> bufs{stage, stage + 6, stage + 12};
    const Tile tile = tiles[reverse ? gridDim.x - 1 - blockIdx.x : blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t t = tile.start + threadIdx.x;
    const uint64_t sweep = *sweep_ptr;
    unsigned accepted = 0;
    if (t < c.half) {
        const int64_t s = (int64_t)parity * c.half + t;
        const Coord x = decode_storage(c, s);
        const m3f a = staple_f_staged<MU>(links, c, x, parity, bufs);
        m3f u = load_f(links, c, s, MU);
        const uint64_t key = link_key(c.seed, sweep, x.lex, MU);
        accepted = visit_f(u, a, c.beta / 3.0, angle, key, uniform);
        store_f(links, c, s, MU, u);
    }
    const unsigned warp_sum = __reduce_add_sync(0xffffffffu, accepted);
    if ((threadIdx.x & 31) == 0 && warp_sum)
        atomicAdd(accepts + tile.chain, (unsigned long long)warp_sum);
}

// Gram-Schmidt of rows 0-1 in binary64, rounded back once.
__global__ void __launch_bounds__(kSiteThreads)
k_f32_reunitarize(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                  float2 *__restrict__ links) {
    // serpentine tile order: starts where the sweep's last sub-sweep ended
    // and ends where the plaquette that follows starts (per-site work, so
    // the order changes nothing else)
    const Tile tile = tiles[serpentine_tile(blockIdx.x, gridDim.x)];
    const ChainInfo c = chains[tile.chain];
    const int64_t s = tile.start + threadIdx.x;
    if (s >= c.volume) return;
    for (int mu = 0; mu < 4; ++mu) {
        m3 u = load_as_f64(links, c, s, mu);
        double n0 = 0.0;
#pragma unroll
        for (int k = 0; k < 3; ++k) n0 += u.e[0][k].re * u.e[0][k].re + u.e[0][k].im * u.e[0][k].im;
        n0 = 1.0 / sqrt(n0);
#pragma unroll
        for (int k = 0; k < 3; ++k) u.e[0][k] = cmake(u.e[0][k].re * n0, u.e[0][k].im * n0);
        cplx dot = cmake(0.0, 0.0);
#pragma unroll
        for (int k = 0; k < 3; ++k) dot = cadd(dot, cmul(cconj(u.e[0][k]), u.e[1][k]));
        double n1 = 0.0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            u.e[1][k] = csub(u.e[1][k], cmul(dot, u.e[0][k]));
            n1 += u.e[1][k].re * u.e[1][k].re + u.e[1][k].im * u.e[1][k].im;
        }
        n1 = 1.0 / sqrt(n1);
#pragma unroll
        for (int k = 0; k < 3; ++k) u.e[1][k] = cmake(u.e[1][k].re * n1, u.e[1][k].im * n1);
        store_rows_from_f64(links, c, s, mu, u);
    }
}

// Plaquette of the stored links in binary64 (products and accumulation).
__global__ void __launch_bounds__(kSiteThreads)
k_f32_plaquette(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                const float2 *__restrict__ links, double *__restrict__ partial) {
    __shared__ double warp_vals[32];
    const int64_t tix = serpentine_tile(blockIdx.x, gridDim.x);   // tiles in serpentine order
    const Tile tile = tiles[tix];
    const ChainInfo c = chains[tile.chain];
    const int64_t s = tile.start + threadIdx.x;
    double v = 0.0;
    if (s < c.volume) {
        const Coord x = decode_storage(c, s);
        bool first = true;
#pragma unroll 1
        for (int mu = 0; mu < 3; ++mu) {
            const m3 umu = load_as_f64(links, c, s, mu);
            const Nb pm = step(c, x.x, x.lex, x.par, mu, +1);
#pragma unroll 1
            for (int nu = mu + 1; nu < 4; ++nu) {
                const Nb pn = step(c, x.x, x.lex, x.par, nu, +1);
                m3 p = mul(umu, load_as_f64(links, c, storage_index(c, pm.lex, pm.par), nu));
                p = mul_adj(p, load_as_f64(links, c, storage_index(c, pn.lex, pn.par), mu));
                const double val = retrace_mul_adj(p, load_as_f64(links, c, s, nu)) / 3.0;
                v = first ? val : v + val;
                first = false;
            }
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) warp_vals[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < (blockDim.x >> 5) ? warp_vals[threadIdx.x] : 0.0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (threadIdx.x == 0) partial[tix] = v;
    }
}

// Every chain at once: blockIdx.y picks the chain.
__global__ void k_f32_identity(const ChainInfo *__restrict__ chains, float2 *links) {
    const ChainInfo c = chains[blockIdx.y];
    const int64_t n = 24 * c.volume;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int e = (int)((i / c.volume) % 6);
        links[c.offset + i] = make_float2((e == 0 || e == 4) ? 1.f : 0.f, 0.f);
    }
}

__global__ void __launch_bounds__(kSiteThreads)
k_f32_hot_start(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                float2 *__restrict__ links) {
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t s = tile.start + threadIdx.x;
    if (s >= c.volume) return;
    const Coord x = decode_storage(c, s);
#pragma unroll 1
    for (int mu = 0; mu < 4; ++mu)
        store_rows_from_f64(links, c, s, mu, haar_su3(hot_start_key(c.seed, x.lex, mu)));
}

// Reference AoS (18 doubles per link) <-> two-row binary32.
__global__ void k_f32_from_aos(const ChainInfo *__restrict__ chains, int chain, float2 *links,
                               const double2 *__restrict__ staging) {
    const ChainInfo c = chains[chain];
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < c.volume;
         s += (int64_t)gridDim.x * blockDim.x) {
        const Coord x = decode_storage(c, s);
        for (int mu = 0; mu < 4; ++mu) {
            const double2 *src = staging + (x.lex * 4 + mu) * 9;
            float2 *dst = links + c.offset + (int64_t)(mu * 6) * c.volume + s;
            for (int e = 0; e < 6; ++e)
                dst[(int64_t)e * c.volume] = make_float2((float)src[e].x, (float)src[e].y);
        }
    }
}

__global__ void k_f32_to_aos(const ChainInfo *__restrict__ chains, int chain,
                             const float2 *__restrict__ links, double2 *staging) {
    const ChainInfo c = chains[chain];
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < c.volume;
         s += (int64_t)gridDim.x * blockDim.x) {
        const Coord x = decode_storage(c, s);
        for (int mu = 0; mu < 4; ++mu) {
            const m3 u = load_as_f64(links, c, s, mu);
            double2 *dst = staging + (x.lex * 4 + mu) * 9;
            for (int e = 0; e < 9; ++e) dst[e] = make_double2(u.e[e / 3][e % 3].re, u.e[e / 3][e % 3].im);
        }
    }
}

// One link of a two-row chain as binary64 (the third row rebuilt, as
// k_f32_to_aos writes it) / from binary64 (its first two rows rounded).
__global__ void k_f32_get_link(const ChainInfo *__restrict__ chains, int chain, const float2 *links,
                               int64_t s, int mu, double2 *out) {
    const ChainInfo c = chains[chain];
    const m3 u = load_as_f64(links, c, s, mu);
    for (int e = 0; e < 9; ++e) out[e] = make_double2(u.e[e / 3][e % 3].re, u.e[e / 3][e % 3].im);
}

__global__ void k_f32_set_link(const ChainInfo *__restrict__ chains, int chain, float2 *links,
                               int64_t s, int mu, const double2 *in) {
    const ChainInfo c = chains[chain];
    m3 u;
    for (int e = 0; e < 9; ++e) u.e[e / 3][e % 3] = cmake(in[e].x, in[e].y);
    store_rows_from_f64(links, c, s, mu, u);
}

// Two-row binary32 handle -> full binary64 handle of the same geometry.
__global__ void __launch_bounds__(kSiteThreads)
k_f32_to_f64(const ChainInfo *__restrict__ src_chains, const ChainInfo *__restrict__ dst_chains,
             const Tile *__restrict__ tiles, const float2 *__restrict__ src, double2 *__restrict__ dst) {
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = src_chains[tile.chain];
    const ChainInfo d = dst_chains[tile.chain];
    const int64_t s = tile.start + threadIdx.x;
    if (s >= c.volume) return;
    for (int mu = 0; mu < 4; ++mu) store_su3(dst, d, s, mu, load_as_f64(src, c, s, mu));
}

__global__ void __launch_bounds__(kSiteThreads)
k_f64_to_f32(const ChainInfo *__restrict__ src_chains, const ChainInfo *__restrict__ dst_chains,
             const Tile *__restrict__ tiles, const double2 *__restrict__ src, float2 *__restrict__ dst) {
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = src_chains[tile.chain];
    const ChainInfo d = dst_chains[tile.chain];
    const int64_t s = tile.start + threadIdx.x;
    if (s >= c.volume) return;
    for (int mu = 0; mu < 4; ++mu) store_rows_from_f64(dst, d, s, mu, load_su3(src, c, s, mu));
}

int grid_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b > 148 * 16) b = 148 * 16;
    return (int)(b < 1 ? 1 : b);
}

float2 *f32_links(ym_ensemble *e) { return reinterpret_cast<float2 *>(e->d_links); }

}  // namespace

cudaError_t launch_f32_metropolis(ym_ensemble *e, int parity, int mu, double angle, int uniform) {
    const dim3 g((unsigned)e->n_half_tiles), b(T);
    float2 *l = f32_links(e);
    // consecutive sub-sweeps in opposite tile orders (each starts on the
    // links the previous one left in L2; the order changes no bit)
    const int reverse = (parity * 4 + mu) & 1;
    switch (mu) {
    case 0: k_f32_metropolis<0><<<g, b, 0, e->stream>>>(e->d_chains, e->d_half_tiles, l, parity, angle, uniform, e->d_sweep, e->d_accepts, reverse); break;
    case 1: k_f32_metropolis<1><<<g, b, 0, e->stream>>>(e->d_chains, e->d_half_tiles, l, parity, angle, uniform, e->d_sweep, e->d_accepts, reverse); break;
    case 2: k_f32_metropolis<2><<<g, b, 0, e->stream>>>(e->d_chains, e->d_half_tiles, l, parity, angle, uniform, e->d_sweep, e->d_accepts, reverse); break;
    default: k_f32_metropolis<3><<<g, b, 0, e->stream>>>(e->d_chains, e->d_half_tiles, l, parity, angle, uniform, e->d_sweep, e->d_accepts, reverse); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_f32_reunitarize(ym_ensemble *e) {
    k_f32_reunitarize<<<(unsigned)e->n_site_tiles, kSiteThreads, 0, e->stream>>>(e->d_chains, e->d_site_tiles,
                                                                                 f32_links(e));
    return cudaGetLastError();
}

cudaError_t launch_f32_plaquette_partials(ym_ensemble *e) {
    k_f32_plaquette<<<(unsigned)e->n_site_tiles, kSiteThreads, 0, e->stream>>>(e->d_chains, e->d_site_tiles,
                                                                               f32_links(e), e->d_partial);
    return cudaGetLastError();
}

cudaError_t launch_f32_identity(ym_ensemble *e) {
    int64_t vmax = 0;
    for (const ChainInfo &c : e->chains) vmax = c.volume > vmax ? c.volume : vmax;
    for (int64_t first = 0; first < e->n_chains; first += 65535) {   // the grid's y limit
        const int64_t count = e->n_chains - first < 65535 ? e->n_chains - first : 65535;
        const int64_t bx = (grid_for(24 * vmax, 256) + count - 1) / count;
        k_f32_identity<<<dim3((unsigned)(bx < 1 ? 1 : bx), (unsigned)count), 256, 0, e->stream>>>(
            e->d_chains + first, f32_links(e));
    }
    return cudaGetLastError();
}

cudaError_t launch_f32_hot_start(ym_ensemble *e) {
    k_f32_hot_start<<<(unsigned)e->n_site_tiles, kSiteThreads, 0, e->stream>>>(e->d_chains, e->d_site_tiles,
                                                                               f32_links(e));
    return cudaGetLastError();
}

cudaError_t launch_f32_from_aos(ym_ensemble *e, int64_t chain) {
    k_f32_from_aos<<<grid_for(e->chains[chain].volume, 128), 128, 0, e->stream>>>(
        e->d_chains, (int)chain, f32_links(e), reinterpret_cast<const double2 *>(e->d_staging));
    return cudaGetLastError();
}

cudaError_t launch_f32_to_aos(ym_ensemble *e, int64_t chain) {
    k_f32_to_aos<<<grid_for(e->chains[chain].volume, 128), 128, 0, e->stream>>>(
        e->d_chains, (int)chain, f32_links(e), reinterpret_cast<double2 *>(e->d_staging));
    return cudaGetLastError();
}

cudaError_t launch_f32_get_link(ym_ensemble *e, int64_t chain, int64_t s, int mu, double2 *out) {
    k_f32_get_link<<<1, 1, 0, e->stream>>>(e->d_chains, (int)chain, f32_links(e), s, mu, out);
    return cudaGetLastError();
}

cudaError_t launch_f32_set_link(ym_ensemble *e, int64_t chain, int64_t s, int mu, const double2 *in) {
    k_f32_set_link<<<1, 1, 0, e->stream>>>(e->d_chains, (int)chain, f32_links(e), s, mu, in);
    return cudaGetLastError();
}

cudaError_t launch_convert(ym_ensemble *src, ym_ensemble *dst) {
    if (src->precision == YM_PREC_F32_TWO_ROW && dst->precision == YM_PREC_F64) {
        k_f32_to_f64<<<(unsigned)dst->n_site_tiles, kSiteThreads, 0, dst->stream>>>(
            src->d_chains, dst->d_chains, dst->d_site_tiles, f32_links(src), dst->d_links);
    } else if (src->precision == YM_PREC_F64 && dst->precision == YM_PREC_F32_TWO_ROW) {
        k_f64_to_f32<<<(unsigned)dst->n_site_tiles, kSiteThreads, 0, dst->stream>>>(
            src->d_chains, dst->d_chains, dst->d_site_tiles, src->d_links, f32_links(dst));
    } else {
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace ym
