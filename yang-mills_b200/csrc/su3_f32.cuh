// su3_f32.cuh -- device helpers of the two-row binary32 SU(3) storage,
// shared by the plain (su3_f32.cu) and learned (learned.cu) sub-sweeps.
//
// Storage: the first two rows of every link, 6 complex floats = 48 bytes;
// the third row is rebuilt on load as conj(row0 x row1).  Plane (mu*6 + e)
// holds entry e (row-major over rows 0-1) of every site as a float2.
#pragma once

#include <cuda_runtime.h>

#include "ym_internal.hpp"

namespace ym {
namespace f32 {

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

// staple_f with every factor staged global -> shared by cp.async ahead of
// its use: the first two factors of a term one term ahead, the third when
// its own term starts, so each product starts on data that has landed and
// loads in flight hold no registers.  Same terms, order and arithmetic as
// staple_f, so the same bits.  Each thread owns column threadIdx.x of three
// [6][TT] float2 buffers (two stored rows per link).
template <int TT>
struct StageF {
    float2 (*l1)[TT];
    float2 (*l2)[TT];
    float2 (*l3)[TT];
};

template <int TT>
__device__ __forceinline__ void stage_f(float2 (*buf)[TT], const float2 *links, const ChainInfo &c,
                                        int64_t s, int mu) {
    const float2 *p = links + c.offset + (int64_t)(mu * 6) * c.volume + s;
#pragma unroll
    for (int e = 0; e < 6; ++e) cp_async8(&buf[e][threadIdx.x], p + (int64_t)e * c.volume);
}

template <int TT>
__device__ __forceinline__ m3f staged_f(const float2 (*buf)[TT]) {
    m3f u;
#pragma unroll
    for (int e = 0; e < 6; ++e) {
        const float2 v = buf[e][threadIdx.x];
        u.e[e / 3][e % 3] = cfm(v.x, v.y);
    }
    third_row(u);
    return u;
}

// Storage indices of a term's three factors.
struct TermF {
    int64_t s1, s2, s3;
};

template <int MU, int NU, bool BWD>
__device__ __forceinline__ TermF term_f(const ChainInfo &c, const Coord &x, int par, const Nb &pm) {
    if (!BWD) {
        const Nb pn = step(c, x.x, x.lex, par, NU, +1);
        return TermF{storage_index(c, pm.lex, pm.par), storage_index(c, pn.lex, pn.par),
                     storage_index(c, x.lex, par)};
    }
    const Nb mn = step(c, x.x, x.lex, par, NU, -1);
    const Nb mnpm = step(c, x.x, mn.lex, mn.par, MU, +1);
    const int64_t smn = storage_index(c, mn.lex, mn.par);
    return TermF{storage_index(c, mnpm.lex, mnpm.par), smn, smn};
}

// Term (NU, BWD) on sites `cur`; stages the next term's first two factors
// (sites `nxt`, directions NNU / MU) when HAS_NEXT.
template <int MU, int NU, bool BWD, bool HAS_NEXT, int NNU, int TT>
__device__ __forceinline__ void staged_term_f(const float2 *links, const ChainInfo &c, const TermF &cur,
                                              const TermF &nxt, const StageF<TT> &b, m3f &a) {
    stage_f(b.l3, links, c, cur.s3, NU);
    cp_async_commit();
    cp_async_wait_one();   // this term's first two factors have landed
    m3f p;
    {
        const m3f l1 = staged_f(b.l1), l2 = staged_f(b.l2);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                cf v = cfm(0.f, 0.f);
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    if (!BWD) cffma(v, l1.e[r][j], cfconj(l2.e[k][j]));
                    else cffma(v, cfconj(l1.e[j][r]), cfconj(l2.e[k][j]));
                }
                p.e[r][k] = v;
            }
    }
    if (HAS_NEXT) {
        stage_f(b.l1, links, c, nxt.s1, NNU);
        stage_f(b.l2, links, c, nxt.s2, MU);
        cp_async_commit();
        cp_async_wait_one();   // the third factor (older group) has landed
    } else {
        cp_async_wait_all();
    }
    const m3f l3 = staged_f(b.l3);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int col = 0; col < 3; ++col)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (!BWD) cffma(a.e[r][col], p.e[r][k], cfconj(l3.e[col][k]));
                else cffma(a.e[r][col], p.e[r][k], l3.e[k][col]);
            }
}

template <int MU, int I>
struct NuF {   // the I-th direction other than MU
    static constexpr int v = I < MU ? I : I + 1;
};

template <int MU, int TT>
__device__ __forceinline__ m3f staple_f_staged(const float2 *links, const ChainInfo &c, const Coord &x,
                                               int par, const StageF<TT> &b) {
    constexpr int N0 = NuF<MU, 0>::v, N1 = NuF<MU, 1>::v, N2 = NuF<MU, 2>::v;
    m3f a;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) a.e[i][j] = cfm(0.f, 0.f);
    const Nb pm = step(c, x.x, x.lex, par, MU, +1);
    const TermF t0 = term_f<MU, N0, false>(c, x, par, pm);
    const TermF t1 = term_f<MU, N0, true>(c, x, par, pm);
    stage_f(b.l1, links, c, t0.s1, N0);
    stage_f(b.l2, links, c, t0.s2, MU);
    cp_async_commit();
    staged_term_f<MU, N0, false, true, N0>(links, c, t0, t1, b, a);
    const TermF t2 = term_f<MU, N1, false>(c, x, par, pm);
    staged_term_f<MU, N0, true, true, N1>(links, c, t1, t2, b, a);
    const TermF t3 = term_f<MU, N1, true>(c, x, par, pm);
    staged_term_f<MU, N1, false, true, N1>(links, c, t2, t3, b, a);
    const TermF t4 = term_f<MU, N2, false>(c, x, par, pm);
    staged_term_f<MU, N1, true, true, N2>(links, c, t3, t4, b, a);
    const TermF t5 = term_f<MU, N2, true>(c, x, par, pm);
    staged_term_f<MU, N2, false, true, N2>(links, c, t4, t5, b, a);
    staged_term_f<MU, N2, true, false, N2>(links, c, t5, t5, b, a);
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

// Re of a row of X times a column of A, in binary64 (the retr_row64 chain
// with the column passed by value, for rows chosen at run time).
__device__ __forceinline__ double retr_col64(const cf *x, cf c0, cf c1, cf c2) {
    double acc = (double)x[0].re * (double)c0.re;
    acc = fma(-(double)x[0].im, (double)c0.im, acc);
    acc = fma((double)x[1].re, (double)c1.re, acc);
    acc = fma(-(double)x[1].im, (double)c1.im, acc);
    acc = fma((double)x[2].re, (double)c2.re, acc);
    acc = fma(-(double)x[2].im, (double)c2.im, acc);
    return acc;
}

__device__ __forceinline__ cf csel(bool p, cf a, cf b) { return cf{p ? a.re : b.re, p ? a.im : b.im}; }

// cos h and sin h by Horner's rule in y = h^2 (Taylor coefficients through
// h^14 / h^15: for |h| <= 1.45, the largest argument the lifted half width
// 2.5 gives, the next term is below 2e-9), binary32 fused multiply-adds.
__device__ __forceinline__ void cos_sin_f(float h, float &c, float &s) {
    const float y = h * h;
    c = fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(-1.f / 87178291200.f, y, 1.f / 479001600.f), y, -1.f / 3628800.f), y,
                                 1.f / 40320.f), y, -1.f / 720.f), y, 1.f / 24.f), y, -0.5f), y, 1.f);
    s = h * fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(fmaf(-1.f / 1307674368000.f, y, 1.f / 6227020800.f), y,
                                          -1.f / 39916800.f), y, 1.f / 362880.f), y, -1.f / 5040.f), y,
                           1.f / 120.f), y, -1.f / 6.f), y, 1.f);
}

// One hit of a generator chosen per thread, without divergent control
// flow.  exp(i theta T^g) acts on rows (i, j) as the 2x2 matrix
// [[r00, r01], [r10, r11]] and multiplies the remaining row k by ek:
//   sigma_1 type (g = 0, 3, 5): [[c, i s], [i s, c]]
//   sigma_2 type (g = 1, 4, 6): [[c, s], [-s, c]]
//   sigma_3      (g = 2):       diag(c + i s, c - i s)
//   lambda_8     (g = 7):       rows 0, 1 times e^{i phi}, row 2 times e^{-2 i phi}
// with c = cos(theta/2), s = sin(theta/2), phi = theta/(2 sqrt 3).  Rows are
// picked with selects, so threads with different generators stay converged.
__device__ __forceinline__ void hit_any_f(m3f &u, const m3f &a, double rr[3], double &old_tr, int g,
                                          float theta, double beta3, double unif,
                                          unsigned &accepted) {
    const bool diag = g == 7;
    float s1, c1;
    cos_sin_f(diag ? theta * 0.28867513459481287f : 0.5f * theta, c1, s1);
    // e^{-2 i phi} of lambda_8 from the same pair by the double-angle
    // identities (one cos/sin pair per hit instead of two)
    const float c2 = fmaf(c1, c1, -s1 * s1), s2 = -2.f * s1 * c1;
    const int kind = diag ? 3 : ((g == 2) ? 2 : ((g == 1 || g == 4 || g == 6) ? 1 : 0));
    const cf zero = cfm(0.f, 0.f);
    const cf r00 = (kind == 0 || kind == 1) ? cfm(c1, 0.f) : cfm(c1, s1);
    const cf r11 = (kind == 0 || kind == 1) ? cfm(c1, 0.f) : cfm(c1, kind == 2 ? -s1 : s1);
    const cf r01 = kind == 0 ? cfm(0.f, s1) : (kind == 1 ? cfm(s1, 0.f) : zero);
    const cf r10 = kind == 0 ? cfm(0.f, s1) : (kind == 1 ? cfm(-s1, 0.f) : zero);
    const cf ek = diag ? cfm(c2, s2) : cfm(1.f, 0.f);
    const int i = (g <= 4 || diag) ? 0 : 1;
    const int j = (g <= 2 || diag) ? 1 : 2;
    const int k = 3 - i - j;
    cf ri[3], rj[3], rk[3], ni[3], nj[3], nk[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        ri[c] = csel(i == 0, u.e[0][c], u.e[1][c]);
        rj[c] = csel(j == 1, u.e[1][c], u.e[2][c]);
        rk[c] = csel(k == 2, u.e[2][c], csel(k == 1, u.e[1][c], u.e[0][c]));
        ni[c] = cfadd(cfmul(r00, ri[c]), cfmul(r01, rj[c]));
        nj[c] = cfadd(cfmul(r10, ri[c]), cfmul(r11, rj[c]));
        nk[c] = cfmul(ek, rk[c]);
    }
    cf ci[3], cj[3], ck[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        ci[r] = csel(i == 0, a.e[r][0], a.e[r][1]);
        cj[r] = csel(j == 1, a.e[r][1], a.e[r][2]);
        ck[r] = csel(k == 2, a.e[r][2], csel(k == 1, a.e[r][1], a.e[r][0]));
    }
    const double qi = retr_col64(ni, ci[0], ci[1], ci[2]);
    const double qj = retr_col64(nj, cj[0], cj[1], cj[2]);
    const double qk = retr_col64(nk, ck[0], ck[1], ck[2]);
    const double q0 = i == 0 ? qi : qk;
    const double q1 = i == 1 ? qi : (j == 1 ? qj : qk);
    const double q2 = j == 2 ? qj : qk;
    const double new_tr = (q0 + q1) + q2;
    const bool acc = accept64(old_tr, new_tr, beta3, unif);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const cf n0 = csel(i == 0, ni[c], nk[c]);
        const cf n1 = csel(i == 1, ni[c], csel(j == 1, nj[c], nk[c]));
        const cf n2 = csel(j == 2, nj[c], nk[c]);
        u.e[0][c] = csel(acc, n0, u.e[0][c]);
        u.e[1][c] = csel(acc, n1, u.e[1][c]);
        u.e[2][c] = csel(acc, n2, u.e[2][c]);
    }
    rr[0] = acc ? q0 : rr[0];
    rr[1] = acc ? q1 : rr[1];
    rr[2] = acc ? q2 : rr[2];
    old_tr = acc ? new_tr : old_tr;
    accepted += acc ? 1u : 0u;
}

// The reference's eight ordered hits, unrolled: every hit's generator is a
// compile-time constant (no branches), and the link-independent work of
// later hits (stream words, angle, rotation entries) is free to overlap the
// current hit's dependent chain.
__device__ __forceinline__ unsigned visit_ordered_f(m3f &u, const m3f &a, double beta3, double angle,
                                                    uint64_t key) {
    double rr[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) rr[i] = retr_row64(u.e[i], a, i);
    double old_tr = (rr[0] + rr[1]) + rr[2];
    unsigned accepted = 0;
#pragma unroll
    for (int h = 0; h < 8; ++h) {
        const uint64_t w_angle = splitmix_at(key, (uint64_t)(2 * h));
        const uint64_t w_acc = splitmix_at(key, (uint64_t)(2 * h + 1));
        const float theta = (float)grid_angle(w_angle, angle);
        const double unif = unit_from(w_acc);
        if (h == 7) {
            float s1, c1, s2, c2;
            cos_sin_f(theta * 0.28867513459481287f, c1, s1);
            cos_sin_f(theta * -0.57735026918962573f, c2, s2);
            hit_diag_f(u, a, rr, old_tr, cfm(c1, s1), cfm(c2, s2), beta3, unif, accepted);
        } else {
            float s, c;
            cos_sin_f(0.5f * theta, c, s);
            const int kind = (h == 2) ? 2 : ((h == 1 || h == 4 || h == 6) ? 1 : 0);
            if (h <= 2)
                hit_block_f<0, 1>(u, a, rr, old_tr, kind, c, s, beta3, unif, accepted);
            else if (h <= 4)
                hit_block_f<0, 2>(u, a, rr, old_tr, kind, c, s, beta3, unif, accepted);
            else
                hit_block_f<1, 2>(u, a, rr, old_tr, kind, c, s, beta3, unif, accepted);
        }
    }
    return accepted;
}

// exp(i theta T^a) in closed form: c = cos(theta/2), s = sin(theta/2) for
// the SU(2) subgroups; diag(e^{i theta/(2 sqrt3)} x2, e^{-i theta/sqrt3}).
// Ordered generators take the specialised per-generator code (every thread
// of a warp runs the same generator); uniformly drawn generators take the
// converged hit_any_f.
__device__ __forceinline__ unsigned visit_f(m3f &u, const m3f &a, double beta3, double angle,
                                            uint64_t key, int uniform) {
    if (!uniform) return visit_ordered_f(u, a, beta3, angle, key);
    double rr[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) rr[i] = retr_row64(u.e[i], a, i);
    double old_tr = (rr[0] + rr[1]) + rr[2];
    unsigned accepted = 0;
#pragma unroll 1
    for (int h = 0; h < 8; ++h) {
        const uint64_t w_angle = splitmix_at(key, (uint64_t)(2 * h));
        const uint64_t w_acc = splitmix_at(key, (uint64_t)(2 * h + 1));
        hit_any_f(u, a, rr, old_tr, (int)((w_angle >> 52) & 7),
                  (float)grid_angle(w_angle, angle), beta3, unit_from(w_acc), accepted);
    }
    return accepted;
}

// Sixteen gauge-invariant features of the staple sum (the definition in
// include/ym_learned.h), in binary32.
__device__ __forceinline__ void staple_features(const m3f &a, float beta, float f[16]) {
    cf h[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) h[r][c] = cfm(a.e[r][c].re * (1.f / 6.f), a.e[r][c].im * (1.f / 6.f));
    cf b[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            cf v = cfm(0.f, 0.f);
#pragma unroll
            for (int k = 0; k < 3; ++k) cffma(v, h[r][k], cfconj(h[c][k]));
            b[r][c] = v;
        }
    float t1 = (b[0][0].re + b[1][1].re + b[2][2].re) * (1.f / 3.f);
    float t2 = 0.f;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) t2 = fmaf(b[r][c].re, b[r][c].re, fmaf(b[r][c].im, b[r][c].im, t2));
    t2 *= (1.f / 3.f);
    // ReTr(B B B) = sum_{r,c} Re((B B)[r][c] B[c][r])
    float t3 = 0.f;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            cf bb = cfm(0.f, 0.f);
#pragma unroll
            for (int k = 0; k < 3; ++k) cffma(bb, b[r][k], b[k][c]);
            t3 = fmaf(bb.re, b[c][r].re, fmaf(-bb.im, b[c][r].im, t3));
        }
    t3 *= (1.f / 3.f);
    const cf d = cfadd(cfadd(cfmul(h[0][0], cfsub(cfmul(h[1][1], h[2][2]), cfmul(h[1][2], h[2][1]))),
                             cfmul(h[0][1], cfsub(cfmul(h[1][2], h[2][0]), cfmul(h[1][0], h[2][2])))),
                       cfmul(h[0][2], cfsub(cfmul(h[1][0], h[2][1]), cfmul(h[1][1], h[2][0]))));
    const float d2 = fmaf(d.re, d.re, d.im * d.im);
    const float st1 = sqrtf(fmaxf(t1, 0.f));
    const float k = beta * st1, b6 = beta * (1.f / 6.f), spread = t2 - t1 * t1;
    f[0] = t1;
    f[1] = t2;
    f[2] = t3;
    f[3] = st1;
    f[4] = d.re;
    f[5] = d.im;
    f[6] = d2;
    f[7] = spread;
    f[8] = b6;
    f[9] = k * (1.f / 6.f);
    f[10] = (k * (1.f / 6.f)) * (k * (1.f / 6.f));
    f[11] = 1.f / (1.f + k);
    f[12] = b6 * d.re;
    f[13] = b6 * t2;
    f[14] = b6 * d2;
    f[15] = b6 * spread;
}

// One learned visit: eight hits, generator drawn from the cumulative
// probabilities cum[0..6] with the 11 bits 52..62 of the angle word, angle
// on the paired grid of half width `scale`.
__device__ __forceinline__ unsigned visit_learned_f(m3f &u, const m3f &a, double beta3,
                                                    const float cum[7], float scale, uint64_t key) {
    double rr[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) rr[i] = retr_row64(u.e[i], a, i);
    double old_tr = (rr[0] + rr[1]) + rr[2];
    unsigned accepted = 0;
#pragma unroll 1
    for (int h = 0; h < 8; ++h) {
        const uint64_t w_angle = splitmix_at(key, (uint64_t)(2 * h));
        const uint64_t w_acc = splitmix_at(key, (uint64_t)(2 * h + 1));
        const float ug = ((float)((w_angle >> 52) & 0x7FF) + 0.5f) * (1.f / 2048.f);
        int g = 0;
#pragma unroll
        for (int q = 0; q < 7; ++q) g += (ug >= cum[q]) ? 1 : 0;
        hit_any_f(u, a, rr, old_tr, g, (float)grid_angle(w_angle, (double)scale), beta3,
                  unit_from(w_acc), accepted);
    }
    return accepted;
}

}  // namespace f32
}  // namespace ym
