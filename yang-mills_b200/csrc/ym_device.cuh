// ym_device.cuh -- device-side building blocks of the engine: complex and
// 3x3 link algebra in the reference's operation order, counter-based
// SplitMix64 streams, and the ensemble's storage geometry.
//
// Arithmetic contract: translation units that include this header for the
// bit-reproducible FP64 path are compiled with -fmad=false, so every a*b+c
// below is two rounded operations exactly as in the reference crate
// (reference/rust/src/su3.rs:27-230) and the CPU oracle.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ym {

// ---------------------------------------------------------------- complex

struct cplx {
    double re, im;
};

__device__ __forceinline__ cplx cmake(double r, double i) { return cplx{r, i}; }
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return cplx{a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cplx csub(cplx a, cplx b) { return cplx{a.re - b.re, a.im - b.im}; }
// Complex64::mul (su3.rs:57-62): (a.re*b.re - a.im*b.im, a.re*b.im + a.im*b.re)
__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
    return cplx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ cplx cconj(cplx a) { return cplx{a.re, -a.im}; }

// A 3x3 complex matrix held in registers, row-major.
struct m3 {
    cplx e[3][3];
};

// Mat3::mul (su3.rs:147-159): each entry accumulated over k = 0,1,2.  The
// reference starts from an exact zero; adding +0 to the first product only
// changes the sign of an exactly-zero entry, never a value.
__device__ __forceinline__ m3 mul(const m3 &a, const m3 &b) {
    m3 o;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            cplx v = cmul(a.e[r][0], b.e[0][c]);
            v = cadd(v, cmul(a.e[r][1], b.e[1][c]));
            v = cadd(v, cmul(a.e[r][2], b.e[2][c]));
            o.e[r][c] = v;
        }
    return o;
}

// a * b^dagger with the dagger materialised as conjugated entries first,
// exactly as Mat3::dagger followed by Mat3::mul.
__device__ __forceinline__ m3 mul_adj(const m3 &a, const m3 &b) {
    m3 o;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            cplx v = cmul(a.e[r][0], cconj(b.e[c][0]));
            v = cadd(v, cmul(a.e[r][1], cconj(b.e[c][1])));
            v = cadd(v, cmul(a.e[r][2], cconj(b.e[c][2])));
            o.e[r][c] = v;
        }
    return o;
}

// a^dagger * b
__device__ __forceinline__ m3 adj_mul(const m3 &a, const m3 &b) {
    m3 o;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            cplx v = cmul(cconj(a.e[0][r]), b.e[0][c]);
            v = cadd(v, cmul(cconj(a.e[1][r]), b.e[1][c]));
            v = cadd(v, cmul(cconj(a.e[2][r]), b.e[2][c]));
            o.e[r][c] = v;
        }
    return o;
}

// a^dagger * b^dagger
__device__ __forceinline__ m3 adj_mul_adj(const m3 &a, const m3 &b) {
    m3 o;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            cplx v = cmul(cconj(a.e[0][r]), cconj(b.e[c][0]));
            v = cadd(v, cmul(cconj(a.e[1][r]), cconj(b.e[c][1])));
            v = cadd(v, cmul(cconj(a.e[2][r]), cconj(b.e[c][2])));
            o.e[r][c] = v;
        }
    return o;
}

__device__ __forceinline__ m3 adj(const m3 &a) {
    m3 o;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) o.e[r][c] = cconj(a.e[c][r]);
    return o;
}

__device__ __forceinline__ void add_into(m3 &acc, const m3 &b) {
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) acc.e[r][c] = cadd(acc.e[r][c], b.e[r][c]);
}

__device__ __forceinline__ m3 identity3() {
    m3 o;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) o.e[r][c] = cmake(r == c ? 1.0 : 0.0, 0.0);
    return o;
}

// Re Tr(P * B^dagger) computed from the diagonal of the product only:
// Mat3::trace (su3.rs:171-173) sums the diagonal as (d0 + d1) + d2.
__device__ __forceinline__ double retrace_mul_adj(const m3 &p, const m3 &b) {
    double d[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        cplx v = cmul(p.e[r][0], cconj(b.e[r][0]));
        v = cadd(v, cmul(p.e[r][1], cconj(b.e[r][1])));
        v = cadd(v, cmul(p.e[r][2], cconj(b.e[r][2])));
        d[r] = v.re;
    }
    return (d[0] + d[1]) + d[2];
}

// Row contribution to Re Tr(X A): (t_i0 + t_i1) + t_i2,
// t_ik = X_ik.re*A_ki.re - X_ik.im*A_ki.im.
__device__ __forceinline__ double retr_row(const cplx *xrow, const m3 &a, int i) {
    double t0 = xrow[0].re * a.e[0][i].re - xrow[0].im * a.e[0][i].im;
    double t1 = xrow[1].re * a.e[1][i].re - xrow[1].im * a.e[1][i].im;
    double t2 = xrow[2].re * a.e[2][i].re - xrow[2].im * a.e[2][i].im;
    return (t0 + t1) + t2;
}

// ---------------------------------------------------------------- fused forms
//
// The staple sum and the trace contraction are the engine's own formulation
// (the reference multiplies out whole plaquettes instead), so they are free
// to use fused multiply-adds.  Each is a fixed chain of correctly rounded
// fma() calls, which the CPU oracle repeats with C99 fma() bit for bit.

// acc += a * b, as: re = fma(a.re,b.re,re); re = fma(-a.im,b.im,re);
//                   im = fma(a.re,b.im,im); im = fma(a.im,b.re,im).
__device__ __forceinline__ void cfma(cplx &acc, cplx a, cplx b) {
    acc.re = fma(a.re, b.re, acc.re);
    acc.re = fma(-a.im, b.im, acc.re);
    acc.im = fma(a.re, b.im, acc.im);
    acc.im = fma(a.im, b.re, acc.im);
}

// a * b and a * b^dagger with every entry one fixed chain of cfma() over
// k = 0, 1, 2 from zero: about half the FP64 instructions of mul / mul_adj,
// for measurements held to 1e-12 relative rather than bitwise.
__device__ __forceinline__ m3 mul_fma(const m3 &a, const m3 &b) {
    m3 o;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            cplx v = cmake(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < 3; ++k) cfma(v, a.e[r][k], b.e[k][c]);
            o.e[r][c] = v;
        }
    return o;
}

__device__ __forceinline__ m3 mul_adj_fma(const m3 &a, const m3 &b) {
    m3 o;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            cplx v = cmake(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < 3; ++k) cfma(v, a.e[r][k], cconj(b.e[c][k]));
            o.e[r][c] = v;
        }
    return o;
}

// Row i of Re Tr(X A): x0.re*A0i.re, then fma(-x0.im, A0i.im), fma(x1.re,
// A1i.re), fma(-x1.im, A1i.im), fma(x2.re, A2i.re), fma(-x2.im, A2i.im).
__device__ __forceinline__ double retr_row_fma(const cplx *xrow, const cplx *acol) {
    double acc = xrow[0].re * acol[0].re;
    acc = fma(-xrow[0].im, acol[0].im, acc);
    acc = fma(xrow[1].re, acol[1].re, acc);
    acc = fma(-xrow[1].im, acol[1].im, acc);
    acc = fma(xrow[2].re, acol[2].re, acc);
    acc = fma(-xrow[2].im, acol[2].im, acc);
    return acc;
}

// ---------------------------------------------------------------- RNG

constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ULL;

// SplitMix64 finaliser (su2_ensemble.rs:46-50).
__device__ __forceinline__ uint64_t mix64(uint64_t v) {
    v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ULL;
    v = (v ^ (v >> 27)) * 0x94D049BB133111EBULL;
    return v ^ (v >> 31);
}
// Output n (0-based) of SplitMix64::new(seed): O(1) at any position.
__device__ __forceinline__ uint64_t splitmix_at(uint64_t seed, uint64_t n) {
    return mix64(seed + (n + 1) * kGolden);
}
// unit_f64 (su2_ensemble.rs:40-43): high 53 bits times 2^-53.
__device__ __forceinline__ double unit_from(uint64_t w) {
    return (double)(w >> 11) * (1.0 / 9007199254740992.0);
}
// Stream key of one link visit.
__device__ __forceinline__ uint64_t link_key(uint64_t chain_seed, uint64_t sweep, int64_t lex,
                                             int mu) {
    return splitmix_at(splitmix_at(chain_seed, sweep), (uint64_t)(4 * lex + mu));
}
// proposal_angle_from_u64 (su3_ensemble.rs:199-213) for a validated angle.
__device__ __forceinline__ double grid_angle(uint64_t raw, double angle) {
    uint64_t m = raw & ((1ULL << 52) - 1);
    double magnitude = angle * (double)(2 * m + 1) * (1.0 / 9007199254740992.0);
    double sign = (raw >> 63) == 0 ? -1.0 : 1.0;
    return sign * magnitude;
}

// ------------------------------------------------- asynchronous staging
// Global -> shared copies (cp.async) that land while the thread computes,
// without holding registers for the data: 16 bytes through L2 only, 8 bytes
// through L1 (the 8-byte form has no L2-only variant).  Groups are
// committed per batch and waited for oldest first.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Tile visited by block b of n in serpentine order: the first half of the
// tiles in order, the second half from the last tile down.  A site-tile
// kernel launched right after a sweep whose last sub-sweep ended at the
// lattice's start begins there (the links it touched last sit in L2), and
// ends there again for the next sweep's first sub-sweep: with checkerboard
// storage the first half of a chain's site tiles are its even sites, the
// second half its odd ones, both in lexicographic order.  Results keyed by
// tile are unchanged by the order.
__device__ __forceinline__ int64_t serpentine_tile(int64_t b, int64_t n) {
    const int64_t h = n / 2;
    return b < h ? b : n - 1 - (b - h);
}

// ---------------------------------------------------------------- geometry

// One chain of an ensemble.  Sites are stored in checkerboard order when the
// last extent is even (storage = parity*Vh + lex/2), lexicographically
// otherwise.  Links are structure-of-arrays: plane (mu, entry) holds one
// complex (double2) per site; SU(3) has 9 entries per link, SU(2) stores its
// quaternion as 2 complex entries.
struct ChainInfo {
    int32_t n[4];
    int32_t eo;          // checkerboard storage order
    int32_t pad;
    int64_t volume;      // sites
    int64_t half;        // volume / 2 (eo) or volume
    int64_t offset;      // first double2 of this chain's block
    double beta;
    uint64_t seed;
};

struct Tile {
    int32_t chain;
    int32_t pad;
    int64_t start;       // first work item of the tile within its chain
};

__device__ __forceinline__ int64_t storage_index(const ChainInfo &c, int64_t lex, int par) {
    return c.eo ? (int64_t)par * c.half + (lex >> 1) : lex;
}

struct Coord {
    int32_t x[4];
    int64_t lex;
    int par;
};

// Decode the site that storage slot `s` (0 <= s < volume) holds.
__device__ __forceinline__ Coord decode_storage(const ChainInfo &c, int64_t s) {
    Coord k;
    int64_t lex;
    if (c.eo) {
        int par = s >= c.half ? 1 : 0;
        int64_t t = s - (int64_t)par * c.half;
        int64_t two_t = 2 * t;
        int x3b;
        if (c.volume <= 0x7fffffff) {
            // 32-bit divisions (a few instructions each instead of a 64-bit
            // division routine) whenever every site index fits.
            const uint32_t tt = (uint32_t)two_t, n3 = (uint32_t)c.n[3];
            const uint32_t n2 = (uint32_t)c.n[2], n1 = (uint32_t)c.n[1];
            const uint32_t r1 = tt / n3, r2 = r1 / n2, r3 = r2 / n1;
            x3b = (int)(tt - r1 * n3);
            k.x[2] = (int)(r1 - r2 * n2);
            k.x[1] = (int)(r2 - r3 * n1);
            k.x[0] = (int)r3;
        } else {
            int64_t row = two_t / c.n[3];
            x3b = (int)(two_t - row * c.n[3]);
            k.x[2] = (int)(row % c.n[2]);
            int64_t r2 = row / c.n[2];
            k.x[1] = (int)(r2 % c.n[1]);
            k.x[0] = (int)(r2 / c.n[1]);
        }
        int b = (par + k.x[0] + k.x[1] + k.x[2]) & 1;
        k.x[3] = x3b + b;
        lex = two_t + b;
        k.par = par;
    } else {
        lex = s;
        k.x[3] = (int)(s % c.n[3]);
        int64_t r = s / c.n[3];
        k.x[2] = (int)(r % c.n[2]);
        r /= c.n[2];
        k.x[1] = (int)(r % c.n[1]);
        k.x[0] = (int)(r / c.n[1]);
        k.par = (k.x[0] + k.x[1] + k.x[2] + k.x[3]) & 1;
    }
    k.lex = lex;
    return k;
}

__device__ __forceinline__ int64_t stride_of(const ChainInfo &c, int d) {
    int64_t s = 1;
    for (int i = 3; i > d; --i) s *= c.n[i];
    return s;
}

// Lexicographic index of x shifted by +1 (dir>0) or -1 along d.
__device__ __forceinline__ int64_t shift_lex(const ChainInfo &c, const int32_t *x, int64_t lex,
                                             int d, int dir) {
    int64_t st = stride_of(c, d);
    if (dir > 0) return x[d] == c.n[d] - 1 ? lex - (int64_t)(c.n[d] - 1) * st : lex + st;
    return x[d] == 0 ? lex + (int64_t)(c.n[d] - 1) * st : lex - st;
}

// A neighbouring site: lexicographic index and parity.  A unit step flips the
// parity, except a periodic wrap across an odd extent (a shift of n-1).
struct Nb {
    int64_t lex;
    int par;
};

__device__ __forceinline__ Nb step(const ChainInfo &c, const int32_t *x, int64_t lex, int par,
                                   int d, int dir) {
    const bool wrap = dir > 0 ? (x[d] == c.n[d] - 1) : (x[d] == 0);
    const int flip = (wrap && (c.n[d] & 1)) ? 0 : 1;
    return Nb{shift_lex(c, x, lex, d, dir), par ^ flip};
}

__device__ __forceinline__ int32_t coord_of(const int32_t *x, int d) {
    return d == 0 ? x[0] : (d == 1 ? x[1] : (d == 2 ? x[2] : x[3]));
}

// step() for a direction chosen per thread at run time: the coordinate and
// stride are picked with selects, so no array is indexed dynamically (a
// dynamically indexed coordinate array would live in local memory).
__device__ __forceinline__ Nb step_any(const ChainInfo &c, const int32_t *x, int64_t lex, int par,
                                       int d, int dir) {
    const int32_t xd = coord_of(x, d), nd = coord_of(c.n, d);
    const int64_t st = d == 3 ? 1 : (d == 2 ? (int64_t)c.n[3]
                                            : (d == 1 ? (int64_t)c.n[2] * c.n[3]
                                                      : (int64_t)c.n[1] * c.n[2] * c.n[3]));
    const bool wrap = dir > 0 ? (xd == nd - 1) : (xd == 0);
    const int64_t nl = dir > 0 ? (wrap ? lex - (int64_t)(nd - 1) * st : lex + st)
                               : (wrap ? lex + (int64_t)(nd - 1) * st : lex - st);
    const int flip = (wrap && (nd & 1)) ? 0 : 1;
    return Nb{nl, par ^ flip};
}

// SU(3) FP64 link access: plane (mu*9 + entry) of a chain's block.
__device__ __forceinline__ m3 load_su3(const double2 *__restrict__ links, const ChainInfo &c,
                                       int64_t s, int mu) {
    const double2 *p = links + c.offset + (int64_t)(mu * 9) * c.volume + s;
    m3 o;
#pragma unroll
    for (int e = 0; e < 9; ++e) {
        double2 v = __ldg(p + (int64_t)e * c.volume);
        o.e[e / 3][e % 3] = cmake(v.x, v.y);
    }
    return o;
}

__device__ __forceinline__ m3 load_su3_rw(const double2 *links, const ChainInfo &c, int64_t s,
                                          int mu) {
    const double2 *p = links + c.offset + (int64_t)(mu * 9) * c.volume + s;
    m3 o;
#pragma unroll
    for (int e = 0; e < 9; ++e) {
        double2 v = p[(int64_t)e * c.volume];
        o.e[e / 3][e % 3] = cmake(v.x, v.y);
    }
    return o;
}

__device__ __forceinline__ void store_su3(double2 *links, const ChainInfo &c, int64_t s, int mu,
                                          const m3 &u) {
    double2 *p = links + c.offset + (int64_t)(mu * 9) * c.volume + s;
#pragma unroll
    for (int e = 0; e < 9; ++e) p[(int64_t)e * c.volume] = make_double2(u.e[e / 3][e % 3].re, u.e[e / 3][e % 3].im);
}

}  // namespace ym
