// su3_tiled.cuh -- the tiled SU(3) FP64 Metropolis sub-sweep, the engine's
// hot kernels.
//
// One launch updates every link U_mu(x) with x of one checkerboard parity,
// in every chain of the ensemble: staple sum -> eight Metropolis hits ->
// store.  The per-link update rule is the reference's metropolis_sweep
// (reference/rust/src/su3_ensemble.rs:342-391): proposal R = exp(i theta T^a)
// on the paired angle grid, candidate R*U, accept iff u < exp(-max(dS, 0)),
// two stream words per hit.  Links of one parity and direction do not touch
// each other's staples, so all of them update concurrently.
//
// Two translation units compile these kernels:
//   * su3_metropolis.cu (-fmad=false): the reference's bits.  The candidate
//     R*U is the reference's (dense-order products, no fused multiply-add);
//     the staple sum A and the contraction Re Tr(X A) are the engine's own
//     formulation of the action change, dS = (beta/3)(ReTr(U A) - ReTr(U'A)),
//     written as fixed chains of fma() that the CPU oracle repeats bit for
//     bit;
//   * su3_metropolis_fast.cu (YM_TILED_FAST, fused multiply-adds): the same
//     algorithm in binary64 with every product free to round once, and the
//     rotation entries from cos_sin_horner instead of the reference's Taylor
//     recurrence (ym_ensemble_set_fast_sweeps).
//
// Layout: every factor of the six staple terms is copied global -> shared by
// cp.async ahead of its use.  Ordered hits (k_su3_metropolis_ring) keep the
// staple accumulator in registers and stage two terms ahead, two 128-thread
// blocks per SM; drawn generators (k_su3_metropolis) keep it in shared
// memory (nine double2 per thread, conflict-free column layout) and stage
// one term ahead, three blocks per SM.
#pragma once
#include <cuda_runtime.h>

#include "su3_exp.cuh"
#include "su3_sites.cuh"
#include "ym_internal.hpp"

#ifndef YM_METRO_MIN_BLOCKS
// Resident 128-thread blocks per SM the register budget of k_su3_metropolis
// targets: the staging buffers (54 KB dynamic + the 18 KB accumulator per
// block) fit three blocks per SM, and at three blocks 168 registers per
// thread leave no spills.
#define YM_METRO_MIN_BLOCKS 3
#endif

// The two compilations live in different namespaces, so that their kernels
// are told apart by name (profilers show ym::tiled_exact::... and
// ym::tiled_fast::...).
#ifdef YM_TILED_FAST
#define YM_TILED_NS tiled_fast
#else
#define YM_TILED_NS tiled_exact
#endif

namespace ym {
namespace YM_TILED_NS {
namespace {

constexpr int T = kSweepThreads;

__device__ __forceinline__ cplx sa_get(const double2 (*sa)[T], int e) {
    const double2 v = sa[e][threadIdx.x];
    return cmake(v.x, v.y);
}
__device__ __forceinline__ void sa_put(double2 (*sa)[T], int e, cplx v) {
    sa[e][threadIdx.x] = make_double2(v.re, v.im);
}

// Column i of A: A[0][i], A[1][i], A[2][i].
__device__ __forceinline__ void sa_col(const double2 (*sa)[T], int i, cplx col[3]) {
#pragma unroll
    for (int k = 0; k < 3; ++k) col[k] = sa_get(sa, 3 * k + i);
}

// Link (s, mu) into this thread's column of the staging buffer.
__device__ __forceinline__ void stage_link(double2 (*buf)[T], const double2 *links, const ChainInfo &c,
                                           int64_t s, int mu) {
    const double2 *p = links + c.offset + (int64_t)(mu * 9) * c.volume + s;
#pragma unroll
    for (int e = 0; e < 9; ++e) cp_async16(&buf[e][threadIdx.x], p + (int64_t)e * c.volume);
    cp_async_commit();
}

__device__ __forceinline__ m3 staged_link(const double2 (*buf)[T]) {
    m3 o;
#pragma unroll
    for (int e = 0; e < 9; ++e) {
        const double2 v = buf[e][threadIdx.x];
        o.e[e / 3][e % 3] = cmake(v.x, v.y);
    }
    return o;
}

// Staple sum A for link (x, MU): for each NU != MU in ascending order, the
// forward term U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag, then the backward term
// U_nu(x-nu+mu)^dag U_mu(x-nu)^dag U_nu(x-nu); P = the first two factors (fma
// chains from zero), then A += P * third factor.  Every factor is staged by
// cp.async: the first two one term ahead, the third at the start of its own
// term, so each product starts on data that has already landed.
struct TermSites {
    int64_t s1, s2, s3;   // storage indices of the three factors
};

template <int MU, int NU, bool BWD>
__device__ __forceinline__ TermSites term_sites(const ChainInfo &c, const Coord &x, int par,
                                                const Nb &pm) {
    if (!BWD) {
        const Nb pn = step(c, x.x, x.lex, par, NU, +1);
        return TermSites{storage_index(c, pm.lex, pm.par), storage_index(c, pn.lex, pn.par),
                         storage_index(c, x.lex, par)};
    }
    const Nb mn = step(c, x.x, x.lex, par, NU, -1);
    const Nb mnpm = step(c, x.x, mn.lex, mn.par, MU, +1);
    const int64_t smn = storage_index(c, mn.lex, mn.par);
    return TermSites{storage_index(c, mnpm.lex, mnpm.par), smn, smn};
}

struct StageBufs {
    double2 (*l1)[T];
    double2 (*l2)[T];
    double2 (*l3)[T];
};

__device__ __forceinline__ void stage_pair(const StageBufs &b, const double2 *links, const ChainInfo &c,
                                           const TermSites &t, int d1, int d2) {
    const double2 *p1 = links + c.offset + (int64_t)(d1 * 9) * c.volume + t.s1;
    const double2 *p2 = links + c.offset + (int64_t)(d2 * 9) * c.volume + t.s2;
#pragma unroll
    for (int e = 0; e < 9; ++e) {
        cp_async16(&b.l1[e][threadIdx.x], p1 + (int64_t)e * c.volume);
        cp_async16(&b.l2[e][threadIdx.x], p2 + (int64_t)e * c.volume);
    }
    cp_async_commit();
}

// Term (NU, BWD) with its sites `cur`; stages the next term's first two
// factors (sites `nxt`, directions NNU / MU) when HAS_NEXT, else the updated
// link U_MU at storage index nxt.s1 into the first buffer, so it lands
// during the last product.
template <int MU, int NU, bool BWD, bool HAS_NEXT, int NNU>
__device__ __forceinline__ void staged_term(const double2 *links, const ChainInfo &c, const TermSites &cur,
                                            const TermSites &nxt, const StageBufs &b, double2 (*sa)[T]) {
    stage_link(b.l3, links, c, cur.s3, NU);
    cp_async_wait_one();   // this term's first two factors have landed
    m3 p;
    {
        const m3 l1 = staged_link(b.l1), l2 = staged_link(b.l2);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                cplx v = cmake(0.0, 0.0);
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    if (!BWD) cfma(v, l1.e[r][j], cconj(l2.e[k][j]));
                    else cfma(v, cconj(l1.e[j][r]), cconj(l2.e[k][j]));
                }
                p.e[r][k] = v;
            }
    }
    if (HAS_NEXT) {
        stage_pair(b, links, c, nxt, NNU, MU);
        cp_async_wait_one();   // the third factor (older group) has landed
    } else {
        stage_link(b.l1, links, c, nxt.s1, MU);   // the updated link itself (sites `nxt`)
        cp_async_wait_one();
    }
    const m3 l3 = staged_link(b.l3);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int col = 0; col < 3; ++col) {
            cplx a = sa_get(sa, 3 * r + col);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (!BWD) cfma(a, p.e[r][k], cconj(l3.e[col][k]));
                else cfma(a, p.e[r][k], l3.e[k][col]);
            }
            sa_put(sa, 3 * r + col, a);
        }
}

template <int MU, int I>
struct Nu {   // the I-th direction other than MU
    static constexpr int v = I < MU ? I : I + 1;
};

template <int MU>
__device__ __forceinline__ void staple_pipelined(const double2 *links, const ChainInfo &c, const Coord &x,
                                                 int par, const Nb &pm, double2 (*sa)[T], const StageBufs &b,
                                                 int64_t s_self) {
    constexpr int N0 = Nu<MU, 0>::v, N1 = Nu<MU, 1>::v, N2 = Nu<MU, 2>::v;
    const TermSites t0 = term_sites<MU, N0, false>(c, x, par, pm);
    const TermSites t1 = term_sites<MU, N0, true>(c, x, par, pm);
    stage_pair(b, links, c, t0, N0, MU);
    staged_term<MU, N0, false, true, N0>(links, c, t0, t1, b, sa);
    const TermSites t2 = term_sites<MU, N1, false>(c, x, par, pm);
    staged_term<MU, N0, true, true, N1>(links, c, t1, t2, b, sa);
    const TermSites t3 = term_sites<MU, N1, true>(c, x, par, pm);
    staged_term<MU, N1, false, true, N1>(links, c, t2, t3, b, sa);
    const TermSites t4 = term_sites<MU, N2, false>(c, x, par, pm);
    staged_term<MU, N1, true, true, N2>(links, c, t3, t4, b, sa);
    const TermSites t5 = term_sites<MU, N2, true>(c, x, par, pm);
    staged_term<MU, N2, false, true, N2>(links, c, t4, t5, b, sa);
    staged_term<MU, N2, true, false, N2>(links, c, t5, TermSites{s_self, 0, 0}, b, sa);
}

// Metropolis decision shared by the block and diagonal hits.
__device__ __forceinline__ bool accept_step(double old_tr, double new_tr, double beta3,
                                            double unif) {
    const double ds = beta3 * (old_tr - new_tr);
    const double m = fmax(ds, 0.0);          // (-delta.max(0.0)).exp() su3_ensemble.rs:368
    return (m == 0.0) ? true : (unif < exp(-m));
}

// Hit with a block rotation on rows (I0, I1): [[c, i s],[i s, c]] (kind 0),
// [[c, s],[-s, c]] (kind 1) or diag(c + i s, c - i s) (kind 2).  Candidate
// rows are Mat3::mul's values (no fused multiply-add).
template <int I0, int I1>
__device__ __forceinline__ void hit_block(m3 &u, const double2 (*sa)[T], double rr[3], double &old_tr,
                                          int kind, double c, double s, double beta3, double unif,
                                          unsigned &accepted) {
    cplx n0[3], n1[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double x0 = u.e[I0][k].re, y0 = u.e[I0][k].im;
        const double x1 = u.e[I1][k].re, y1 = u.e[I1][k].im;
        if (kind == 0) {
            n0[k] = cmake(c * x0 - s * y1, c * y0 + s * x1);
            n1[k] = cmake(c * x1 - s * y0, s * x0 + c * y1);
        } else if (kind == 1) {
            n0[k] = cmake(c * x0 + s * x1, c * y0 + s * y1);
            n1[k] = cmake(c * x1 - s * x0, c * y1 - s * y0);
        } else {
            n0[k] = cmake(c * x0 - s * y0, c * y0 + s * x0);
            n1[k] = cmake(c * x1 + s * y1, c * y1 - s * x1);
        }
    }
    cplx col0[3], col1[3];
    sa_col(sa, I0, col0);
    sa_col(sa, I1, col1);
    double q[3] = {rr[0], rr[1], rr[2]};
    q[I0] = retr_row_fma(n0, col0);
    q[I1] = retr_row_fma(n1, col1);
    const double new_tr = (q[0] + q[1]) + q[2];
    if (accept_step(old_tr, new_tr, beta3, unif)) {
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

__device__ __forceinline__ void hit_diag(m3 &u, const double2 (*sa)[T], double rr[3], double &old_tr,
                                         cplx e1, cplx e2, double beta3, double unif,
                                         unsigned &accepted) {
    cplx n[3][3];
    double q[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const cplx e = i < 2 ? e1 : e2;
#pragma unroll
        for (int k = 0; k < 3; ++k) n[i][k] = cmul(e, u.e[i][k]);
        cplx col[3];
        sa_col(sa, i, col);
        q[i] = retr_row_fma(n[i], col);
    }
    const double new_tr = (q[0] + q[1]) + q[2];
    if (accept_step(old_tr, new_tr, beta3, unif)) {
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

// hit_block for a generator drawn per link (g < 7): rows i0, i1 picked by
// selects and A's columns read from shared memory, so threads of a warp
// with different SU(2)-subgroup generators stay converged.  Each kind of
// hit_block writes its candidate entries as c*x + s*a with a one of the
// other entries or its negation (c*x - s*y == c*x + s*(-y) exactly), so the
// single formula gives hit_block's bits.
__device__ __forceinline__ void hit_block_drawn(m3 &u, const double2 (*sa)[T], double rr[3],
                                                double &old_tr, int g, double c, double s,
                                                double beta3, double unif, unsigned &accepted) {
    const int kind = (g == 2) ? 2 : ((g == 1 || g == 4 || g == 6) ? 1 : 0);
    const int i0 = g <= 4 ? 0 : 1, i1 = g <= 2 ? 1 : 2;
    cplx n0[3], n1[3], col0[3], col1[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const cplx r0 = i0 == 0 ? u.e[0][k] : u.e[1][k];
        const cplx r1 = i1 == 1 ? u.e[1][k] : u.e[2][k];
        const double x0 = r0.re, y0 = r0.im, x1 = r1.re, y1 = r1.im;
        const double a0 = kind == 0 ? -y1 : (kind == 1 ? x1 : -y0);
        const double b0 = kind == 0 ? x1 : (kind == 1 ? y1 : x0);
        const double a1 = kind == 0 ? -y0 : (kind == 1 ? -x0 : y1);
        const double b1 = kind == 0 ? x0 : (kind == 1 ? -y0 : -x1);
        n0[k] = cmake(c * x0 + s * a0, c * y0 + s * b0);
        n1[k] = cmake(c * x1 + s * a1, c * y1 + s * b1);
    }
    sa_col(sa, i0, col0);
    sa_col(sa, i1, col1);
    const double q0n = retr_row_fma(n0, col0), q1n = retr_row_fma(n1, col1);
    const double q0 = i0 == 0 ? q0n : rr[0];
    const double q1 = i0 == 1 ? q0n : (i1 == 1 ? q1n : rr[1]);
    const double q2 = i1 == 2 ? q1n : rr[2];
    const double new_tr = (q0 + q1) + q2;
    if (accept_step(old_tr, new_tr, beta3, unif)) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (i0 == 0) u.e[0][k] = n0[k];
            u.e[1][k] = i0 == 1 ? n0[k] : (i1 == 1 ? n1[k] : u.e[1][k]);
            if (i1 == 2) u.e[2][k] = n1[k];
        }
        rr[0] = q0;
        rr[1] = q1;
        rr[2] = q2;
        old_tr = new_tr;
        accepted++;
    }
}

// Fast form only (YM_TILED_FAST): cos h and sin h as polynomials in
// y = h^2 by Horner's rule with fused multiply-adds, the Taylor coefficients
// 1/k! truncated where the next term is below 1e-19 for the half widths
// served: through h^14 / h^15 for K <= 13 (|h| <= 0.173), through h^18 /
// h^19 above (|h| <= 0.578).
template <int K>
__device__ __forceinline__ void cos_sin_horner(double h, double &c, double &s) {
    constexpr int NT = K <= 13 ? 7 : 9;
    constexpr double kc[10] = {1.0, -1.0 / 2, 1.0 / 24, -1.0 / 720, 1.0 / 40320, -1.0 / 3628800,
                               1.0 / 479001600, -1.0 / 87178291200.0, 1.0 / 20922789888000.0,
                               -1.0 / 6402373705728000.0};
    constexpr double ks[10] = {1.0, -1.0 / 6, 1.0 / 120, -1.0 / 5040, 1.0 / 362880, -1.0 / 39916800,
                               1.0 / 6227020800.0, -1.0 / 1307674368000.0, 1.0 / 355687428096000.0,
                               -1.0 / 121645100408832000.0};
    const double y = h * h;
    double pc = kc[NT], ps = ks[NT];
#pragma unroll
    for (int k = NT - 1; k >= 0; --k) {
        pc = fma(pc, y, kc[k]);
        ps = fma(ps, y, ks[k]);
    }
    c = pc;
    s = h * ps;
}

// Eight hits on u: generator h (ordered) or bits 52..54 of the hit's angle
// word (uniform).  Words 2h and 2h+1 of the link's stream.
__device__ __forceinline__ unsigned visit(m3 &u, const double2 (*sa)[T], double beta3,
                                          double angle, uint64_t key, int uniform) {
    double rr[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        cplx col[3];
        sa_col(sa, i, col);
        rr[i] = retr_row_fma(u.e[i], col);
    }
    double old_tr = (rr[0] + rr[1]) + rr[2];
    unsigned accepted = 0;
#pragma unroll 1
    for (int h = 0; h < 8; ++h) {
        const uint64_t w_angle = splitmix_at(key, (uint64_t)(2 * h));
        const uint64_t w_acc = splitmix_at(key, (uint64_t)(2 * h + 1));
        const int g = uniform ? (int)((w_angle >> 52) & 7) : h;
        const double theta = grid_angle(w_angle, angle);
        const double unif = unit_from(w_acc);
        if (g == 7) {
            cplx e1, e2;
#ifdef YM_TILED_FAST
            double c1, s1, c2, s2;
            cos_sin_horner<16>((0.5 * kInvSqrt3) * theta, c1, s1);
            cos_sin_horner<16>((-kInvSqrt3) * theta, c2, s2);
            e1 = cmake(c1, s1);
            e2 = cmake(c2, s2);
#else
            lambda8_rotation(theta, e1, e2);
#endif
            hit_diag(u, sa, rr, old_tr, e1, e2, beta3, unif, accepted);
        } else {
            double c, s;
#ifdef YM_TILED_FAST
            cos_sin_horner<16>(0.5 * theta, c, s);
#else
            taylor_chain(0.5 * theta, c, s);   // |0.5 theta| < 0.5: no squaring
#endif
            if (uniform) {
                hit_block_drawn(u, sa, rr, old_tr, g, c, s, beta3, unif, accepted);
                continue;
            }
            const int kind = (g == 2) ? 2 : ((g == 1 || g == 4 || g == 6) ? 1 : 0);
            if (g <= 2)
                hit_block<0, 1>(u, sa, rr, old_tr, kind, c, s, beta3, unif, accepted);
            else if (g <= 4)
                hit_block<0, 2>(u, sa, rr, old_tr, kind, c, s, beta3, unif, accepted);
            else
                hit_block<1, 2>(u, sa, rr, old_tr, kind, c, s, beta3, unif, accepted);
        }
    }
    return accepted;
}

// ---- the reference's ordered hits, software-pipelined ---------------------
// A hit has a link-independent half (its two stream words, the angle, the
// rotation entries from the Taylor chain, the uniform) and a link-dependent
// half (candidate rows, Re Tr against the staple, the decision).  visit()
// runs them back to back, and the Taylor chain's early exits split the code
// into many small blocks; here every hit's link-independent half is computed
// while the previous hit's link-dependent half runs, both branch-free in one
// straight-line block, so each link carries two independent dependency
// chains instead of one.  The values are visit()'s, bit for bit:
//   * taylor_fixed<K> evaluates K terms of taylor_chain's recurrence and adds
//     term k only while no earlier term was at or below the 1e-18 cutoff.
//     K is taken from the proposal half width a so that every admissible
//     angle stops within K terms: |t_k| <= |h|^k / k! with |h| <= a/2 for
//     generators 1..7 and |h| <= 0.5774 a (at most 0.5 after lambda8's
//     halving) for generator 8.  Terms the reference still adds past K
//     must be too small to move their sum (below half an ulp of it): for
//     a <= 0.3, K = 11 (t_12 <= 0.1732^12/12! = 1.5e-18 against sums near
//     0.985, t_13 / s <= 0.1732^12/13! = 1.2e-19); for a <= 1, K = 14
//     (t_15 / s <= 0.5^14/15! = 4.7e-17 < 2^-54, t_16 <= 7.3e-19), so the
//     sums are the reference's bit for bit (checked on the CPU against
//     the loop run to the cutoff over millions of grid angles).
//   * the decision is accept_step's u < exp(-max(dS, 0)) (for m = 0,
//     exp(-0) = 1 > u, as its explicit branch gives); the accepted rows are
//     selected, not branched to.
template <int K>
__device__ __forceinline__ void taylor_fixed(double h, double &c, double &s) {
    double t = 1.0;
    c = 1.0;
    s = 0.0;
    bool done = false;
#pragma unroll
    for (int k = 1; k <= K; ++k) {
        t = (t * h) * c_inv[k];
        if ((k & 3) == 1) { const double v = s + t; s = done ? s : v; }
        else if ((k & 3) == 2) { const double v = c - t; c = done ? c : v; }
        else if ((k & 3) == 3) { const double v = s - t; s = done ? s : v; }
        else { const double v = c + t; c = done ? c : v; }
        done = done || fabs(t) <= kTermCutoff;
    }
}

// lambda8_rotation with taylor_chain2's lockstep chains (stopping on the
// larger term) evaluated for K terms; |theta| <= 1 needs at most one halving.
template <int K>
__device__ __forceinline__ void lambda8_fixed(double theta, cplx &e1, cplx &e2) {
    const double d1 = (0.5 * kInvSqrt3) * theta;
    const double d2 = (-kInvSqrt3) * theta;
    const bool sq = fmax(fabs(d1), fabs(d2)) > 0.5;
    const double sc = sq ? 0.5 : 1.0;
    const double h1 = d1 * sc, h2 = d2 * sc;
    double t1 = 1.0, t2 = 1.0, c1 = 1.0, s1 = 0.0, c2 = 1.0, s2 = 0.0;
    bool done = false;
#pragma unroll
    for (int k = 1; k <= K; ++k) {
        t1 = (t1 * h1) * c_inv[k];
        t2 = (t2 * h2) * c_inv[k];
        if ((k & 3) == 1) { const double a = s1 + t1, b = s2 + t2; s1 = done ? s1 : a; s2 = done ? s2 : b; }
        else if ((k & 3) == 2) { const double a = c1 - t1, b = c2 - t2; c1 = done ? c1 : a; c2 = done ? c2 : b; }
        else if ((k & 3) == 3) { const double a = s1 - t1, b = s2 - t2; s1 = done ? s1 : a; s2 = done ? s2 : b; }
        else { const double a = c1 + t1, b = c2 + t2; c1 = done ? c1 : a; c2 = done ? c2 : b; }
        done = done || fmax(fabs(t1), fabs(t2)) <= kTermCutoff;
    }
    e1 = cmake(c1, s1);
    e2 = cmake(c2, s2);
    const cplx q1 = cmul(e1, e1), q2 = cmul(e2, e2);
    e1 = sq ? q1 : e1;
    e2 = sq ? q2 : e2;
}

// Rotation entries of a hit: the reference's bits (taylor_fixed,
// lambda8_fixed), or in the fast form cos_sin_horner for both generators'
// phases (lambda8's two directly, without halving and squaring).
template <int K>
__device__ __forceinline__ void block_rotation(double h, double &c, double &s) {
#ifdef YM_TILED_FAST
    cos_sin_horner<K>(h, c, s);
#else
    taylor_fixed<K>(h, c, s);
#endif
}

template <int K>
__device__ __forceinline__ void diag_rotation(double theta, cplx &e1, cplx &e2) {
#ifdef YM_TILED_FAST
    double c1, s1, c2, s2;
    cos_sin_horner<K>((0.5 * kInvSqrt3) * theta, c1, s1);
    cos_sin_horner<K>((-kInvSqrt3) * theta, c2, s2);
    e1 = cmake(c1, s1);
    e2 = cmake(c2, s2);
#else
    lambda8_fixed<K>(theta, e1, e2);
#endif
}

struct BlockPre {
    double c, s, unif;
};
struct DiagPre {
    cplx e1, e2;
    double unif;
};

template <int K>
__device__ __forceinline__ BlockPre pre_block(uint64_t key, int h, double angle) {
    BlockPre p;
    block_rotation<K>(0.5 * grid_angle(splitmix_at(key, (uint64_t)(2 * h)), angle), p.c, p.s);
    p.unif = unit_from(splitmix_at(key, (uint64_t)(2 * h + 1)));
    return p;
}

template <int K>
__device__ __forceinline__ DiagPre pre_diag(uint64_t key, int h, double angle) {
    DiagPre p;
    diag_rotation<K>(grid_angle(splitmix_at(key, (uint64_t)(2 * h)), angle), p.e1, p.e2);
    p.unif = unit_from(splitmix_at(key, (uint64_t)(2 * h + 1)));
    return p;
}

// hit_block for a compile-time generator, decision by selects.
template <int I0, int I1, int KIND>
__device__ __forceinline__ void hit_block_sel(m3 &u, const double2 (*sa)[T], double rr[3], double &old_tr,
                                              const BlockPre &p, double beta3, unsigned &accepted) {
    const double c = p.c, s = p.s;
    cplx n0[3], n1[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double x0 = u.e[I0][k].re, y0 = u.e[I0][k].im;
        const double x1 = u.e[I1][k].re, y1 = u.e[I1][k].im;
        if (KIND == 0) {
            n0[k] = cmake(c * x0 - s * y1, c * y0 + s * x1);
            n1[k] = cmake(c * x1 - s * y0, s * x0 + c * y1);
        } else if (KIND == 1) {
            n0[k] = cmake(c * x0 + s * x1, c * y0 + s * y1);
            n1[k] = cmake(c * x1 - s * x0, c * y1 - s * y0);
        } else {
            n0[k] = cmake(c * x0 - s * y0, c * y0 + s * x0);
            n1[k] = cmake(c * x1 + s * y1, c * y1 - s * x1);
        }
    }
    cplx col0[3], col1[3];
    sa_col(sa, I0, col0);
    sa_col(sa, I1, col1);
    double q[3] = {rr[0], rr[1], rr[2]};
    q[I0] = retr_row_fma(n0, col0);
    q[I1] = retr_row_fma(n1, col1);
    const double new_tr = (q[0] + q[1]) + q[2];
    const double m = fmax(beta3 * (old_tr - new_tr), 0.0);
    const bool acc = p.unif < exp(-m);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        u.e[I0][k] = acc ? n0[k] : u.e[I0][k];
        u.e[I1][k] = acc ? n1[k] : u.e[I1][k];
    }
    rr[I0] = acc ? q[I0] : rr[I0];
    rr[I1] = acc ? q[I1] : rr[I1];
    old_tr = acc ? new_tr : old_tr;
    accepted += acc ? 1u : 0u;
}

__device__ __forceinline__ void hit_diag_sel(m3 &u, const double2 (*sa)[T], double rr[3], double &old_tr,
                                             const DiagPre &p, double beta3, unsigned &accepted) {
    cplx n[3][3];
    double q[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const cplx e = i < 2 ? p.e1 : p.e2;
#pragma unroll
        for (int k = 0; k < 3; ++k) n[i][k] = cmul(e, u.e[i][k]);
        cplx col[3];
        sa_col(sa, i, col);
        q[i] = retr_row_fma(n[i], col);
    }
    const double new_tr = (q[0] + q[1]) + q[2];
    const double m = fmax(beta3 * (old_tr - new_tr), 0.0);
    const bool acc = p.unif < exp(-m);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int k = 0; k < 3; ++k) u.e[i][k] = acc ? n[i][k] : u.e[i][k];
        rr[i] = acc ? q[i] : rr[i];
    }
    old_tr = acc ? new_tr : old_tr;
    accepted += acc ? 1u : 0u;
}

// The eight ordered hits (generators 1..8, su3_ensemble.rs:361): hit h+1's
// link-independent half is written next to hit h.
// tr receives Re Tr(U' A) of the final link, the sum of its six plaquettes.
template <int K>
__device__ __forceinline__ unsigned visit_ordered(m3 &u, const double2 (*sa)[T], double beta3,
                                                  double angle, uint64_t key, double &tr) {
    double rr[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        cplx col[3];
        sa_col(sa, i, col);
        rr[i] = retr_row_fma(u.e[i], col);
    }
    double old_tr = (rr[0] + rr[1]) + rr[2];
    unsigned accepted = 0;
    const BlockPre p0 = pre_block<K>(key, 0, angle);
    const BlockPre p1 = pre_block<K>(key, 1, angle);
    hit_block_sel<0, 1, 0>(u, sa, rr, old_tr, p0, beta3, accepted);
    const BlockPre p2 = pre_block<K>(key, 2, angle);
    hit_block_sel<0, 1, 1>(u, sa, rr, old_tr, p1, beta3, accepted);
    const BlockPre p3 = pre_block<K>(key, 3, angle);
    hit_block_sel<0, 1, 2>(u, sa, rr, old_tr, p2, beta3, accepted);
    const BlockPre p4 = pre_block<K>(key, 4, angle);
    hit_block_sel<0, 2, 0>(u, sa, rr, old_tr, p3, beta3, accepted);
    const BlockPre p5 = pre_block<K>(key, 5, angle);
    hit_block_sel<0, 2, 1>(u, sa, rr, old_tr, p4, beta3, accepted);
    const BlockPre p6 = pre_block<K>(key, 6, angle);
    hit_block_sel<1, 2, 0>(u, sa, rr, old_tr, p5, beta3, accepted);
    const DiagPre p7 = pre_diag<K>(key, 7, angle);
    hit_block_sel<1, 2, 1>(u, sa, rr, old_tr, p6, beta3, accepted);
    hit_diag_sel(u, sa, rr, old_tr, p7, beta3, accepted);
    tr = old_tr;
    return accepted;
}

// Drawn generators (visit()): three CTAs per SM, the accumulator in shared
// memory, one staple term staged ahead.
template <int MU>
__global__ void __launch_bounds__(T, YM_METRO_MIN_BLOCKS)
k_su3_metropolis(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                 double2 *__restrict__ links, int parity, double angle, int uniform,
                 const uint64_t *__restrict__ sweep_ptr, unsigned long long *__restrict__ accepts,
                 int log2_item, int reverse) {
    __shared__ double2 sa[9][T];
    extern __shared__ __align__(16) double2 stage_mem[];
    const StageBufs bufs{reinterpret_cast<double2 (*)[T]>(stage_mem),
                         reinterpret_cast<double2 (*)[T]>(stage_mem + 9 * T),
                         reinterpret_cast<double2 (*)[T]>(stage_mem + 18 * T)};
    // The CTA takes T >> log2_item work items of 2^log2_item sites each
    // (possibly of different chains); padding items have chain < 0.
    const int64_t cta = reverse ? (int64_t)gridDim.x - 1 - blockIdx.x : (int64_t)blockIdx.x;
    const Tile tile = tiles[cta * (T >> log2_item) + (threadIdx.x >> log2_item)];
    const bool live = tile.chain >= 0;
    const ChainInfo c = chains[live ? tile.chain : 0];
    const int64_t t = tile.start + (threadIdx.x & ((1u << log2_item) - 1u));
    const uint64_t sweep = *sweep_ptr;
    unsigned accepted = 0;
    if (live && t < c.half) {
        const int64_t s = (int64_t)parity * c.half + t;
        const Coord x = decode_storage(c, s);
#pragma unroll
        for (int e = 0; e < 9; ++e) sa[e][threadIdx.x] = make_double2(0.0, 0.0);
        const Nb pm = step(c, x.x, x.lex, parity, MU, +1);
        staple_pipelined<MU>(links, c, x, parity, pm, sa, bufs, s);
        cp_async_wait_all();
        m3 u = staged_link(bufs.l1);
        const uint64_t key = link_key(c.seed, sweep, x.lex, MU);
        accepted = visit(u, sa, c.beta / 3.0, angle, key, uniform);
        store_su3(links, c, s, MU, u);
    }
    const unsigned warp_sum = __reduce_add_sync(0xffffffffu, accepted);
    if ((threadIdx.x & 31) == 0 && warp_sum)
        atomicAdd(accepts + tile.chain, (unsigned long long)warp_sum);
}

// ---- ordered hits: two staple terms in flight, two CTAs per SM -----------
// The ordered-hit sub-sweep keeps the staple accumulator in registers and a
// ring of two three-factor staging sets, so term k+2's factors are loading
// while term k multiplies (one term ahead in k_su3_metropolis).  Two
// 128-thread CTAs per SM fit (registers and 108 KB of staging each); after
// the staple the accumulator is written once to the second set's memory for
// the hits.  The products and their order are staple_pipelined's, so A has
// the same bits.  On a 32^4 lattice this is 1.4 % faster than the
// three-CTA form with the ordered visit, and 20 % slower with the drawn
// generators' visit, whose loop-carried hits need the third CTA's warps.
struct TermSet {
    double2 (*f[3])[T];
};

template <int MU, int NU>
__device__ __forceinline__ void stage_term3(const TermSet &b, const double2 *links, const ChainInfo &c,
                                            const TermSites &t) {
    const double2 *p1 = links + c.offset + (int64_t)(NU * 9) * c.volume + t.s1;
    const double2 *p2 = links + c.offset + (int64_t)(MU * 9) * c.volume + t.s2;
    const double2 *p3 = links + c.offset + (int64_t)(NU * 9) * c.volume + t.s3;
#pragma unroll
    for (int e = 0; e < 9; ++e) {
        cp_async16(&b.f[0][e][threadIdx.x], p1 + (int64_t)e * c.volume);
        cp_async16(&b.f[1][e][threadIdx.x], p2 + (int64_t)e * c.volume);
        cp_async16(&b.f[2][e][threadIdx.x], p3 + (int64_t)e * c.volume);
    }
    cp_async_commit();
}

template <bool BWD>
__device__ __forceinline__ void term_accumulate(const TermSet &b, m3 &a) {
    m3 p;
    {
        const m3 l1 = staged_link(b.f[0]), l2 = staged_link(b.f[1]);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                cplx v = cmake(0.0, 0.0);
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    if (!BWD) cfma(v, l1.e[r][j], cconj(l2.e[k][j]));
                    else cfma(v, cconj(l1.e[j][r]), cconj(l2.e[k][j]));
                }
                p.e[r][k] = v;
            }
    }
    const m3 l3 = staged_link(b.f[2]);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int col = 0; col < 3; ++col)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (!BWD) cfma(a.e[r][col], p.e[r][k], cconj(l3.e[col][k]));
                else cfma(a.e[r][col], p.e[r][k], l3.e[k][col]);
            }
}

// SAVE = 2 or 4: a_part receives the accumulator after the first SAVE terms
// (the terms of the first one or two directions other than MU).
template <int MU, int SAVE = 0>
__device__ __forceinline__ m3 staple_ring(const double2 *links, const ChainInfo &c, const Coord &x, int par,
                                          const Nb &pm, const TermSet &s0, const TermSet &s1, int64_t s_self,
                                          m3 *a_part = nullptr) {
    constexpr int N0 = Nu<MU, 0>::v, N1 = Nu<MU, 1>::v, N2 = Nu<MU, 2>::v;
    stage_term3<MU, N0>(s0, links, c, term_sites<MU, N0, false>(c, x, par, pm));
    stage_term3<MU, N0>(s1, links, c, term_sites<MU, N0, true>(c, x, par, pm));
    m3 a;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) a.e[r][k] = cmake(0.0, 0.0);
    cp_async_wait_one();
    term_accumulate<false>(s0, a);
    stage_term3<MU, N1>(s0, links, c, term_sites<MU, N1, false>(c, x, par, pm));
    cp_async_wait_one();
    term_accumulate<true>(s1, a);
    if (SAVE == 2) *a_part = a;
    stage_term3<MU, N1>(s1, links, c, term_sites<MU, N1, true>(c, x, par, pm));
    cp_async_wait_one();
    term_accumulate<false>(s0, a);
    stage_term3<MU, N2>(s0, links, c, term_sites<MU, N2, false>(c, x, par, pm));
    cp_async_wait_one();
    term_accumulate<true>(s1, a);
    if (SAVE == 4) *a_part = a;
    stage_term3<MU, N2>(s1, links, c, term_sites<MU, N2, true>(c, x, par, pm));
    cp_async_wait_one();
    term_accumulate<false>(s0, a);
    stage_link(s0.f[0], links, c, s_self, MU);   // the updated link itself
    cp_async_wait_one();
    term_accumulate<true>(s1, a);
    return a;
}

constexpr int kRingBuffers = 6;   // two sets of three factors

// MEASURE (parity 1, MU = 1, 2 or 3: the last three sub-sweeps of a sweep,
// one chain per CTA): each CTA also writes tr_partial[cta], the sum over its
// links of (1/3) Re Tr(U' A_p) with A_p the staple terms of the directions
// nu < MU (MU = 1: nu = 0; MU = 2: nu = 0, 1; MU = 3: all of A).  Once this
// sub-sweep has run, every link of those terms is final (directions below
// MU are done, direction MU's even links were done in parity 0, its odd
// links here), and each plaquette of plane (nu, MU) holds exactly one
// odd-site MU-link, so the three launches' sums are the plaquettes of
// planes (0,1); (0,2), (1,2); (0,3), (1,3), (2,3): all six planes.
template <int MU, int K, bool MEASURE = false>
__global__ void __launch_bounds__(T, 2)
k_su3_metropolis_ring(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                      double2 *__restrict__ links, int parity, double angle,
                      const uint64_t *__restrict__ sweep_ptr, unsigned long long *__restrict__ accepts,
                      int log2_item, int reverse, double *__restrict__ tr_partial = nullptr) {
    extern __shared__ __align__(16) double2 ring_mem[];
    auto buf = [&](int i) { return reinterpret_cast<double2 (*)[T]>(ring_mem + (size_t)i * 9 * T); };
    const TermSet s0{{buf(0), buf(1), buf(2)}}, s1{{buf(3), buf(4), buf(5)}};
    const int64_t cta = reverse ? (int64_t)gridDim.x - 1 - blockIdx.x : (int64_t)blockIdx.x;
    const Tile tile = tiles[cta * (T >> log2_item) + (threadIdx.x >> log2_item)];
    const bool live = tile.chain >= 0;
    const ChainInfo c = chains[live ? tile.chain : 0];
    const int64_t t = tile.start + (threadIdx.x & ((1u << log2_item) - 1u));
    const uint64_t sweep = *sweep_ptr;
    unsigned accepted = 0;
    double tr = 0.0;
    if (live && t < c.half) {
        const int64_t s = (int64_t)parity * c.half + t;
        const Coord x = decode_storage(c, s);
        const Nb pm = step(c, x.x, x.lex, parity, MU, +1);
        constexpr int kSave = (MEASURE && MU == 1) ? 2 : ((MEASURE && MU == 2) ? 4 : 0);
        m3 a_part;
        const m3 a = staple_ring<MU, kSave>(links, c, x, parity, pm, s0, s1, s, &a_part);
        cp_async_wait_all();
        m3 u = staged_link(s0.f[0]);
        // the accumulator, for the hits, in the second set's (now free) memory
        double2 (*sa)[T] = s1.f[0];
#pragma unroll
        for (int e = 0; e < 9; ++e) sa[e][threadIdx.x] = make_double2(a.e[e / 3][e % 3].re, a.e[e / 3][e % 3].im);
        const uint64_t key = link_key(c.seed, sweep, x.lex, MU);
        accepted = visit_ordered<K>(u, sa, c.beta / 3.0, angle, key, tr);
        store_su3(links, c, s, MU, u);
        if (kSave) {   // Re Tr(U' A_p)
            double q = 0.0;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const cplx col[3] = {a_part.e[0][i], a_part.e[1][i], a_part.e[2][i]};
                q = q + retr_row_fma(u.e[i], col);
            }
            tr = q;
        }
    }
    const unsigned warp_sum = __reduce_add_sync(0xffffffffu, accepted);
    if ((threadIdx.x & 31) == 0 && warp_sum)
        atomicAdd(accepts + tile.chain, (unsigned long long)warp_sum);
    if (MEASURE) {
        double v = (live && t < c.half) ? tr / 3.0 : 0.0;
        v = block_reduce<false>(v);
        if (threadIdx.x == 0) tr_partial[cta] = v;
    }
}


constexpr size_t kStageBytes = 27 * T * sizeof(double2);   // three staged factors per thread

constexpr size_t kRingBytes = (size_t)kRingBuffers * 9 * T * sizeof(double2);

// Both launchers take the handle's sweep layout: work items of 2^log2
// sites, chain order or by descending chain volume (all layouts give the
// same bits).
template <int K>
void metro_launch_ordered(ym_ensemble *e, int parity, int mu, double angle, int reverse) {
    const SweepLayout &L = e->layouts[e->sweep_layout];
    const dim3 grid((unsigned)L.ctas), block(T);
    const Tile *items = L.d_items;
    switch (mu) {
    case 0: k_su3_metropolis_ring<0, K><<<grid, block, kRingBytes, e->stream>>>(e->d_chains, items, e->d_links, parity, angle, e->d_sweep, e->d_accepts, L.log2_item, reverse); break;
    case 1: k_su3_metropolis_ring<1, K><<<grid, block, kRingBytes, e->stream>>>(e->d_chains, items, e->d_links, parity, angle, e->d_sweep, e->d_accepts, L.log2_item, reverse); break;
    case 2: k_su3_metropolis_ring<2, K><<<grid, block, kRingBytes, e->stream>>>(e->d_chains, items, e->d_links, parity, angle, e->d_sweep, e->d_accepts, L.log2_item, reverse); break;
    default: k_su3_metropolis_ring<3, K><<<grid, block, kRingBytes, e->stream>>>(e->d_chains, items, e->d_links, parity, angle, e->d_sweep, e->d_accepts, L.log2_item, reverse); break;
    }
}

void metro_launch_drawn(ym_ensemble *e, int parity, int mu, double angle, int reverse) {
    const SweepLayout &L = e->layouts[e->sweep_layout];
    const dim3 grid((unsigned)L.ctas), block(T);
    const Tile *items = L.d_items;
    switch (mu) {
    case 0: k_su3_metropolis<0><<<grid, block, kStageBytes, e->stream>>>(e->d_chains, items, e->d_links, parity, angle, 1, e->d_sweep, e->d_accepts, L.log2_item, reverse); break;
    case 1: k_su3_metropolis<1><<<grid, block, kStageBytes, e->stream>>>(e->d_chains, items, e->d_links, parity, angle, 1, e->d_sweep, e->d_accepts, L.log2_item, reverse); break;
    case 2: k_su3_metropolis<2><<<grid, block, kStageBytes, e->stream>>>(e->d_chains, items, e->d_links, parity, angle, 1, e->d_sweep, e->d_accepts, L.log2_item, reverse); break;
    default: k_su3_metropolis<3><<<grid, block, kStageBytes, e->stream>>>(e->d_chains, items, e->d_links, parity, angle, 1, e->d_sweep, e->d_accepts, L.log2_item, reverse); break;
    }
}

// The last sub-sweep of a sweep (parity 1, direction 3, ordered hits) with
// its plaquette share (MEASURE): the handle's layout must put one chain in
// each CTA (128-site items).
template <int K>
void metro_launch_measure(ym_ensemble *e, int mu, double angle, double *tr_partial) {
    const SweepLayout &L = e->layouts[e->sweep_layout];
    const dim3 g((unsigned)L.ctas), b(T);
    const int rev = (1 * 4 + mu) & 1;   // the tile order tiled_launch gives (parity 1, mu)
    if (mu == 1)
        k_su3_metropolis_ring<1, K, true><<<g, b, kRingBytes, e->stream>>>(e->d_chains, L.d_items, e->d_links, 1, angle, e->d_sweep, e->d_accepts, L.log2_item, rev, tr_partial);
    else if (mu == 2)
        k_su3_metropolis_ring<2, K, true><<<g, b, kRingBytes, e->stream>>>(e->d_chains, L.d_items, e->d_links, 1, angle, e->d_sweep, e->d_accepts, L.log2_item, rev, tr_partial);
    else
        k_su3_metropolis_ring<3, K, true><<<g, b, kRingBytes, e->stream>>>(e->d_chains, L.d_items, e->d_links, 1, angle, e->d_sweep, e->d_accepts, L.log2_item, rev, tr_partial);
}

cudaError_t set_smem(const void *f, size_t bytes) {
    cudaError_t err = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (err == cudaSuccess)
        err = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    return err;
}

// Shared-memory limits of the sub-sweep kernels, set once per device.
cudaError_t configure_kernels() {
    static thread_local int configured_device = -1;
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (configured_device != dev) {
        const void *drawn[4] = {(const void *)k_su3_metropolis<0>, (const void *)k_su3_metropolis<1>,
                                (const void *)k_su3_metropolis<2>, (const void *)k_su3_metropolis<3>};
        const void *ordered[14] = {(const void *)k_su3_metropolis_ring<0, 11>, (const void *)k_su3_metropolis_ring<1, 11>,
                                   (const void *)k_su3_metropolis_ring<2, 11>, (const void *)k_su3_metropolis_ring<3, 11>,
                                   (const void *)k_su3_metropolis_ring<0, 14>, (const void *)k_su3_metropolis_ring<1, 14>,
                                   (const void *)k_su3_metropolis_ring<2, 14>, (const void *)k_su3_metropolis_ring<3, 14>,
                                   (const void *)k_su3_metropolis_ring<1, 11, true>,
                                   (const void *)k_su3_metropolis_ring<2, 11, true>,
                                   (const void *)k_su3_metropolis_ring<3, 11, true>,
                                   (const void *)k_su3_metropolis_ring<1, 14, true>,
                                   (const void *)k_su3_metropolis_ring<2, 14, true>,
                                   (const void *)k_su3_metropolis_ring<3, 14, true>};
        for (const void *f : drawn)
            if ((err = set_smem(f, kStageBytes)) != cudaSuccess) return err;
        for (const void *f : ordered)
            if ((err = set_smem(f, kRingBytes)) != cudaSuccess) return err;
        configured_device = dev;
    }
    return cudaSuccess;
}

// One sub-sweep of the handle: ordered hits on the ring kernel with the
// term count the half width allows (angles are validated to lie in
// [1e-8, 1] for binary64 handles), drawn generators on the three-CTA kernel.
cudaError_t tiled_launch(ym_ensemble *e, int parity, int mu, double angle, int uniform) {
    if (cudaError_t err = configure_kernels()) return err;
    // Consecutive sub-sweeps walk the lattice in opposite directions (odd
    // ones from the last CTA down), so each starts on the links the previous
    // one touched last and finds its first waves' staple links in L2.  The
    // links of one sub-sweep are independent, so the order changes no bit.
    const int reverse = (parity * 4 + mu) & 1;
    if (uniform) metro_launch_drawn(e, parity, mu, angle, reverse);
    else if (angle <= 0.3) metro_launch_ordered<11>(e, parity, mu, angle, reverse);
    else metro_launch_ordered<14>(e, parity, mu, angle, reverse);
    return cudaGetLastError();
}

// tiled_launch(e, 1, mu, angle, ordered hits), mu = 1, 2 or 3, that also
// writes each CTA's plaquette share of the planes (nu, mu), nu < mu, to
// tr_partial[cta] (the handle's layout must hold one chain per CTA).
cudaError_t tiled_launch_measure(ym_ensemble *e, int mu, double angle, double *tr_partial) {
    if (cudaError_t err = configure_kernels()) return err;
    if (angle <= 0.3) metro_launch_measure<11>(e, mu, angle, tr_partial);
    else metro_launch_measure<14>(e, mu, angle, tr_partial);
    return cudaGetLastError();
}

}  // namespace
}  // namespace YM_TILED_NS
}  // namespace ym
