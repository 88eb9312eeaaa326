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

#include "su3_haar.cuh"
#include "ym_internal.hpp"

namespace ym {

namespace {

constexpr int T = kSweepThreads;

struct cf {
    float re, im;
};

__device__ __forceinline__ cf cfm(float r, float i) { return cf{r, i}; }
__device__ __forceinline__ cf cfadd(cf a, cf b) { return cf{a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cf cfsub(cf a, cf b) { return cf{a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ cf cfmul(cf a, cf b) {
    return cf{fmaf(a.re, b.re, -a.im * b.im), fmaf(a.re, b.im, a.im * b.re)};
}
__device__ __forceinline__ cf cfconj(cf a) { return cf{a.re, -a.im}; }
// acc += a * b
__device__ __forceinline__ void cffma(cf &acc, cf a, cf b) {
    acc.re = fmaf(a.re, b.re, acc.re);
    acc.re = fmaf(-a.im, b.im, acc.re);
    acc.im = fmaf(a.re, b.im, acc.im);
    acc.im = fmaf(a.im, b.re, acc.im);
}

struct m3f {
    cf e[3][3];
};

__device__ __forceinline__ void third_row(m3f &u) {
    u.e[2][0] = cfconj(cfsub(cfmul(u.e[0][1], u.e[1][2]), cfmul(u.e[0][2], u.e[1][1])));
    u.e[2][1] = cfconj(cfsub(cfmul(u.e[0][2], u.e[1][0]), cfmul(u.e[0][0], u.e[1][2])));
    u.e[2][2] = cfconj(cfsub(cfmul(u.e[0][0], u.e[1][1]), cfmul(u.e[0][1], u.e[1][0])));
}

__device__ __forceinline__ m3f load_f(const float2 *__restrict__ links, const ChainInfo &c, int64_t s,
                                      int mu) {
    const float2 *p = links + c.offset + (int64_t)(mu * 6) * c.volume + s;
    m3f u;
#pragma unroll
    for (int e = 0; e < 6; ++e) {
        const float2 v = __ldg(p + (int64_t)e * c.volume);
        u.e[e / 3][e % 3] = cfm(v.x, v.y);
    }
    third_row(u);
    return u;
}

__device__ __forceinline__ void store_f(float2 *links, const ChainInfo &c, int64_t s, int mu,
                                        const m3f &u) {
    float2 *p = links + c.offset + (int64_t)(mu * 6) * c.volume + s;
#pragma unroll
    for (int e = 0; e < 6; ++e) p[(int64_t)e * c.volume] = make_float2(u.e[e / 3][e % 3].re, u.e[e / 3][e % 3].im);
}

// Two stored rows -> a binary64 matrix with the third row rebuilt in binary64.
__device__ __forceinline__ m3 load_as_f64(const float2 *__restrict__ links, const ChainInfo &c,
                                          int64_t s, int mu) {
    const float2 *p = links + c.offset + (int64_t)(mu * 6) * c.volume + s;
    m3 u;
#pragma unroll
    for (int e = 0; e < 6; ++e) {
        const float2 v = __ldg(p + (int64_t)e * c.volume);
        u.e[e / 3][e % 3] = cmake((double)v.x, (double)v.y);
    }
    u.e[2][0] = cconj(csub(cmul(u.e[0][1], u.e[1][2]), cmul(u.e[0][2], u.e[1][1])));
    u.e[2][1] = cconj(csub(cmul(u.e[0][2], u.e[1][0]), cmul(u.e[0][0], u.e[1][2])));
    u.e[2][2] = cconj(csub(cmul(u.e[0][0], u.e[1][1]), cmul(u.e[0][1], u.e[1][0])));
    return u;
}

__device__ __forceinline__ void store_rows_from_f64(float2 *links, const ChainInfo &c, int64_t s,
                                                    int mu, const m3 &u) {
    float2 *p = links + c.offset + (int64_t)(mu * 6) * c.volume + s;
#pragma unroll
    for (int e = 0; e < 6; ++e)
        p[(int64_t)e * c.volume] = make_float2((float)u.e[e / 3][e % 3].re, (float)u.e[e / 3][e % 3].im);
}

__device__ __forceinline__ m3f lkf(const float2 *links, const ChainInfo &c, const Nb &n, int mu) {
    return load_f(links, c, storage_index(c, n.lex, n.par), mu);
}

// Staple sum in binary32: same terms and order as the FP64 path.
template <int MU>
__device__ __forceinline__ m3f staple_f(const float2 *__restrict__ links, const ChainInfo &c,
                                        const Coord &x, int par) {
    m3f a;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) a.e[i][j] = cfm(0.f, 0.f);
    const Nb self{x.lex, par};
    const Nb pm = step(c, x.x, x.lex, par, MU, +1);
#pragma unroll
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == MU) continue;
        const Nb pn = step(c, x.x, x.lex, par, nu, +1);
        const Nb mn = step(c, x.x, x.lex, par, nu, -1);
        const Nb mnpm = step(c, x.x, mn.lex, mn.par, MU, +1);
        {
            const m3f l2 = lkf(links, c, pn, MU);
            const m3f l1 = lkf(links, c, pm, nu);
            m3f p;
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    cf v = cfm(0.f, 0.f);
#pragma unroll
                    for (int j = 0; j < 3; ++j) cffma(v, l1.e[r][j], cfconj(l2.e[k][j]));
                    p.e[r][k] = v;
                }
            const m3f l3 = lkf(links, c, self, nu);
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int col = 0; col < 3; ++col)
#pragma unroll
                    for (int k = 0; k < 3; ++k) cffma(a.e[r][col], p.e[r][k], cfconj(l3.e[col][k]));
        }
        {
            const m3f l2 = lkf(links, c, mn, MU);
            const m3f l1 = lkf(links, c, mnpm, nu);
            m3f p;
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    cf v = cfm(0.f, 0.f);
#pragma unroll
                    for (int j = 0; j < 3; ++j) cffma(v, cfconj(l1.e[j][r]), cfconj(l2.e[k][j]));
                    p.e[r][k] = v;
                }
            const m3f l3 = lkf(links, c, mn, nu);
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int col = 0; col < 3; ++col)
#pragma unroll
                    for (int k = 0; k < 3; ++k) cffma(a.e[r][col], p.e[r][k], l3.e[k][col]);
        }
    }
    return a;
}

// Row i of Re Tr(X A) in binary64 from binary32 operands.
__device__ __forceinline__ double retr_row64(const cf *xrow, const m3f &a, int i) {
    double acc = (double)xrow[0].re * (double)a.e[0][i].re;
    acc = fma(-(double)xrow[0].im, (double)a.e[0][i].im, acc);
    acc = fma((double)xrow[1].re, (double)a.e[1][i].re, acc);
    acc = fma(-(double)xrow[1].im, (double)a.e[1][i].im, acc);
    acc = fma((double)xrow[2].re, (double)a.e[2][i].re, acc);
    acc = fma(-(double)xrow[2].im, (double)a.e[2][i].im, acc);
    return acc;
}

__device__ __forceinline__ bool accept64(double old_tr, double new_tr, double beta3, double unif) {
    const double m = fmax(beta3 * (old_tr - new_tr), 0.0);
    return (m == 0.0) ? true : (unif < exp(-m));
}

template <int I0, int I1>
__device__ __forceinline__ void hit_block_f(m3f &u, const m3f &a, double rr[3], double &old_tr,
                                            int kind, float c, float s, double beta3, double unif,
                                            unsigned &accepted) {
    cf n0[3], n1[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float x0 = u.e[I0][k].re, y0 = u.e[I0][k].im;
        const float x1 = u.e[I1][k].re, y1 = u.e[I1][k].im;
        if (kind == 0) {
            n0[k] = cfm(fmaf(c, x0, -s * y1), fmaf(c, y0, s * x1));
            n1[k] = cfm(fmaf(c, x1, -s * y0), fmaf(s, x0, c * y1));
        } else if (kind == 1) {
            n0[k] = cfm(fmaf(c, x0, s * x1), fmaf(c, y0, s * y1));
            n1[k] = cfm(fmaf(c, x1, -s * x0), fmaf(c, y1, -s * y0));
        } else {
            n0[k] = cfm(fmaf(c, x0, -s * y0), fmaf(c, y0, s * x0));
            n1[k] = cfm(fmaf(c, x1, s * y1), fmaf(c, y1, -s * x1));
        }
    }
    double q[3] = {rr[0], rr[1], rr[2]};
    q[I0] = retr_row64(n0, a, I0);
    q[I1] = retr_row64(n1, a, I1);
    const double new_tr = (q[0] + q[1]) + q[2];
    if (accept64(old_tr, new_tr, beta3, unif)) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            u.e[I0][k] = n0[k];
            u.e[I1][k] = n1[k];
        }
        rr[I0] = q[I0];
        rr[I1] = q[I1];
        old_tr = new_tr;
        accepted++;
    }
}

__device__ __forceinline__ void hit_diag_f(m3f &u, const m3f &a, double rr[3], double &old_tr,
                                           cf e1, cf e2, double beta3, double unif,
                                           unsigned &accepted) {
    cf n[3][3];
    double q[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const cf e = i < 2 ? e1 : e2;
#pragma unroll
        for (int k = 0; k < 3; ++k) n[i][k] = cfmul(e, u.e[i][k]);
        q[i] = retr_row64(n[i], a, i);
    }
    const double new_tr = (q[0] + q[1]) + q[2];
    if (accept64(old_tr, new_tr, beta3, unif)) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
#pragma unroll
            for (int k = 0; k < 3; ++k) u.e[i][k] = n[i][k];
            rr[i] = q[i];
        }
        old_tr = new_tr;
        accepted++;
    }
}

// exp(i theta T^a) in closed form: c = cos(theta/2), s = sin(theta/2) for
// the SU(2) subgroups; diag(e^{i theta/(2 sqrt3)} x2, e^{-i theta/sqrt3}).
__device__ __forceinline__ unsigned visit_f(m3f &u, const m3f &a, double beta3, double angle,
                                            uint64_t key, int uniform) {
    double rr[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) rr[i] = retr_row64(u.e[i], a, i);
    double old_tr = (rr[0] + rr[1]) + rr[2];
    unsigned accepted = 0;
#pragma unroll 1
    for (int h = 0; h < 8; ++h) {
        const uint64_t w_angle = splitmix_at(key, (uint64_t)(2 * h));
        const uint64_t w_acc = splitmix_at(key, (uint64_t)(2 * h + 1));
        const int g = uniform ? (int)((w_angle >> 52) & 7) : h;
        const float theta = (float)grid_angle(w_angle, angle);
        const double unif = unit_from(w_acc);
        if (g == 7) {
            float s1, c1, s2, c2;
            sincosf(theta * 0.28867513459481287f, &s1, &c1);
            sincosf(theta * -0.57735026918962573f, &s2, &c2);
            hit_diag_f(u, a, rr, old_tr, cfm(c1, s1), cfm(c2, s2), beta3, unif, accepted);
        } else {
            float s, c;
            sincosf(0.5f * theta, &s, &c);
            const int kind = (g == 2) ? 2 : ((g == 1 || g == 4 || g == 6) ? 1 : 0);
            if (g <= 2)
                hit_block_f<0, 1>(u, a, rr, old_tr, kind, c, s, beta3, unif, accepted);
            else if (g <= 4)
                hit_block_f<0, 2>(u, a, rr, old_tr, kind, c, s, beta3, unif, accepted);
            else
                hit_block_f<1, 2>(u, a, rr, old_tr, kind, c, s, beta3, unif, accepted);
        }
    }
    return accepted;
}

template <int MU>
__global__ void __launch_bounds__(T)
k_f32_metropolis(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                 float2 *__restrict__ links, int parity, double angle, int uniform,
                 const uint64_t *__restrict__ sweep_ptr, unsigned long long *__restrict__ accepts) {
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t t = tile.start + threadIdx.x;
    unsigned accepted = 0;
    if (t < c.half) {
        const int64_t s = (int64_t)parity * c.half + t;
        const Coord x = decode_storage(c, s);
        const m3f a = staple_f<MU>(links, c, x, parity);
        m3f u = load_f(links, c, s, MU);
        const uint64_t key = link_key(c.seed, *sweep_ptr, x.lex, MU);
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
    const Tile tile = tiles[blockIdx.x];
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
    const Tile tile = tiles[blockIdx.x];
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
        if (threadIdx.x == 0) partial[blockIdx.x] = v;
    }
}

__global__ void k_f32_identity(float2 *links, int64_t offset, int64_t volume) {
    const int64_t n = 24 * volume;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int e = (int)((i / volume) % 6);
        links[offset + i] = make_float2((e == 0 || e == 4) ? 1.f : 0.f, 0.f);
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
    switch (mu) {
    case 0: k_f32_metropolis<0><<<g, b, 0, e->stream>>>(e->d_chains, e->d_half_tiles, l, parity, angle, uniform, e->d_sweep, e->d_accepts); break;
    case 1: k_f32_metropolis<1><<<g, b, 0, e->stream>>>(e->d_chains, e->d_half_tiles, l, parity, angle, uniform, e->d_sweep, e->d_accepts); break;
    case 2: k_f32_metropolis<2><<<g, b, 0, e->stream>>>(e->d_chains, e->d_half_tiles, l, parity, angle, uniform, e->d_sweep, e->d_accepts); break;
    default: k_f32_metropolis<3><<<g, b, 0, e->stream>>>(e->d_chains, e->d_half_tiles, l, parity, angle, uniform, e->d_sweep, e->d_accepts); break;
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
    for (int64_t ch = 0; ch < e->n_chains; ++ch) {
        const ChainInfo &c = e->chains[ch];
        k_f32_identity<<<grid_for(24 * c.volume, 256), 256, 0, e->stream>>>(f32_links(e), c.offset, c.volume);
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
