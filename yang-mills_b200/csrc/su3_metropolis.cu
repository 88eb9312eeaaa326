// su3_metropolis.cu -- the SU(3) Metropolis sub-sweep, the engine's hot
// kernel (compiled with -fmad=false).
//
// One launch updates every link U_mu(x) with x of one checkerboard parity,
// in every chain of the ensemble: staple sum -> eight Metropolis hits ->
// store.  The per-link update rule is the reference's metropolis_sweep
// (reference/rust/src/su3_ensemble.rs:342-391): proposal R = exp(i theta T^a)
// on the paired angle grid, candidate R*U, accept iff u < exp(-max(dS, 0)),
// two stream words per hit.  Links of one parity and direction do not touch
// each other's staples, so all of them update concurrently.
//
// Arithmetic:
//   * the candidate R*U is the reference's (dense-order products, no fused
//     multiply-add), bitwise;
//   * the staple sum A and the contraction Re Tr(X A) are the engine's own
//     formulation of the action change, dS = (beta/3)(ReTr(U A) - ReTr(U'A)),
//     written as fixed chains of fma() that the CPU oracle repeats bit for
//     bit.
//
// Layout: per thread the staple accumulator lives in shared memory (18
// doubles per thread, conflict-free column layout) so the register budget
// holds three matrices at most and four 128-thread blocks fit per SM.
#include <cuda_runtime.h>

#include "su3_exp.cuh"
#include "ym_internal.hpp"

#ifndef YM_METRO_MIN_BLOCKS
#define YM_METRO_MIN_BLOCKS 4   // resident 128-thread blocks per SM the register budget targets
#endif

namespace ym {

namespace {

constexpr int T = kSweepThreads;

__device__ __forceinline__ cplx sa_get(const double (*sa)[T], int e) {
    return cmake(sa[2 * e][threadIdx.x], sa[2 * e + 1][threadIdx.x]);
}
__device__ __forceinline__ void sa_put(double (*sa)[T], int e, cplx v) {
    sa[2 * e][threadIdx.x] = v.re;
    sa[2 * e + 1][threadIdx.x] = v.im;
}

// Column i of A: A[0][i], A[1][i], A[2][i].
__device__ __forceinline__ void sa_col(const double (*sa)[T], int i, cplx col[3]) {
#pragma unroll
    for (int k = 0; k < 3; ++k) col[k] = sa_get(sa, 3 * k + i);
}

// The two staple terms of direction NU for link (x, MU):
//   forward  U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag
//   backward U_nu(x-nu+mu)^dag U_mu(x-nu)^dag U_nu(x-nu)
// P = first two factors (fma chains from zero), then A += P * third factor.
template <int MU, int NU>
__device__ __forceinline__ void add_staple(const double2 *__restrict__ links, const ChainInfo &c,
                                           const Coord &x, int par, const Nb &pm, double (*sa)[T]) {
    const Nb pn = step(c, x.x, x.lex, par, NU, +1);
    const Nb mn = step(c, x.x, x.lex, par, NU, -1);
    const Nb mnpm = step(c, x.x, mn.lex, mn.par, MU, +1);   // x-nu keeps x's mu coordinate
    {
        const m3 l2 = load_su3(links, c, storage_index(c, pn.lex, pn.par), MU);
        const m3 l1 = load_su3(links, c, storage_index(c, pm.lex, pm.par), NU);
        m3 p;
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                cplx v = cmake(0.0, 0.0);
#pragma unroll
                for (int j = 0; j < 3; ++j) cfma(v, l1.e[r][j], cconj(l2.e[k][j]));
                p.e[r][k] = v;
            }
        const m3 l3 = load_su3(links, c, storage_index(c, x.lex, par), NU);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int col = 0; col < 3; ++col) {
                cplx a = sa_get(sa, 3 * r + col);
#pragma unroll
                for (int k = 0; k < 3; ++k) cfma(a, p.e[r][k], cconj(l3.e[col][k]));
                sa_put(sa, 3 * r + col, a);
            }
    }
    {
        const m3 l2 = load_su3(links, c, storage_index(c, mn.lex, mn.par), MU);
        const m3 l1 = load_su3(links, c, storage_index(c, mnpm.lex, mnpm.par), NU);
        m3 p;
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                cplx v = cmake(0.0, 0.0);
#pragma unroll
                for (int j = 0; j < 3; ++j) cfma(v, cconj(l1.e[j][r]), cconj(l2.e[k][j]));
                p.e[r][k] = v;
            }
        const m3 l3 = load_su3(links, c, storage_index(c, mn.lex, mn.par), NU);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int col = 0; col < 3; ++col) {
                cplx a = sa_get(sa, 3 * r + col);
#pragma unroll
                for (int k = 0; k < 3; ++k) cfma(a, p.e[r][k], l3.e[k][col]);
                sa_put(sa, 3 * r + col, a);
            }
    }
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
__device__ __forceinline__ void hit_block(m3 &u, const double (*sa)[T], double rr[3], double &old_tr,
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

__device__ __forceinline__ void hit_diag(m3 &u, const double (*sa)[T], double rr[3], double &old_tr,
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

// Eight hits on u: generator h (ordered) or bits 52..54 of the hit's angle
// word (uniform).  Words 2h and 2h+1 of the link's stream.
__device__ __forceinline__ unsigned visit(m3 &u, const double (*sa)[T], double beta3,
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
            lambda8_rotation(theta, e1, e2);
            hit_diag(u, sa, rr, old_tr, e1, e2, beta3, unif, accepted);
        } else {
            double c, s;
            taylor_chain(0.5 * theta, c, s);   // |0.5 theta| < 0.5: no squaring
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

template <int MU>
__global__ void __launch_bounds__(T, YM_METRO_MIN_BLOCKS)
k_su3_metropolis(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                 double2 *__restrict__ links, int parity, double angle, int uniform,
                 const uint64_t *__restrict__ sweep_ptr, unsigned long long *__restrict__ accepts) {
    __shared__ double sa[18][T];
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t t = tile.start + threadIdx.x;
    unsigned accepted = 0;
    if (t < c.half) {
        const int64_t s = (int64_t)parity * c.half + t;
        const Coord x = decode_storage(c, s);
#pragma unroll
        for (int e = 0; e < 18; ++e) sa[e][threadIdx.x] = 0.0;
        const Nb pm = step(c, x.x, x.lex, parity, MU, +1);
        if (MU != 0) add_staple<MU, 0>(links, c, x, parity, pm, sa);
        if (MU != 1) add_staple<MU, 1>(links, c, x, parity, pm, sa);
        if (MU != 2) add_staple<MU, 2>(links, c, x, parity, pm, sa);
        if (MU != 3) add_staple<MU, 3>(links, c, x, parity, pm, sa);
        m3 u = load_su3_rw(links, c, s, MU);
        const uint64_t key = link_key(c.seed, *sweep_ptr, x.lex, MU);
        accepted = visit(u, sa, c.beta / 3.0, angle, key, uniform);
        store_su3(links, c, s, MU, u);
    }
    const unsigned warp_sum = __reduce_add_sync(0xffffffffu, accepted);
    if ((threadIdx.x & 31) == 0 && warp_sum)
        atomicAdd(accepts + tile.chain, (unsigned long long)warp_sum);
}

__global__ void k_advance_sweep(uint64_t *sweep) { *sweep += 1; }

}  // namespace

cudaError_t launch_su3_metropolis(ym_ensemble *e, int parity, int mu, double angle, int uniform) {
    const dim3 grid((unsigned)e->n_half_tiles), block(T);
    switch (mu) {
    case 0: k_su3_metropolis<0><<<grid, block, 0, e->stream>>>(e->d_chains, e->d_half_tiles, e->d_links, parity, angle, uniform, e->d_sweep, e->d_accepts); break;
    case 1: k_su3_metropolis<1><<<grid, block, 0, e->stream>>>(e->d_chains, e->d_half_tiles, e->d_links, parity, angle, uniform, e->d_sweep, e->d_accepts); break;
    case 2: k_su3_metropolis<2><<<grid, block, 0, e->stream>>>(e->d_chains, e->d_half_tiles, e->d_links, parity, angle, uniform, e->d_sweep, e->d_accepts); break;
    default: k_su3_metropolis<3><<<grid, block, 0, e->stream>>>(e->d_chains, e->d_half_tiles, e->d_links, parity, angle, uniform, e->d_sweep, e->d_accepts); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_advance_sweep(ym_ensemble *e) {
    k_advance_sweep<<<1, 1, 0, e->stream>>>(e->d_sweep);
    return cudaGetLastError();
}

}  // namespace ym
