// su3_metropolis.cu -- the SU(3) FP64 Metropolis sweeps with the
// reference's bits (compiled with -fmad=false): the tiled sub-sweep kernels
// of su3_tiled.cuh, the chain-resident kernel for small chains, and the
// dispatch to the fast form (su3_metropolis_fast.cu) for handles that ask
// for it.
#include "su3_tiled.cuh"

namespace ym {

namespace {

constexpr int T = kSweepThreads;

// ---------------------------------------------------------------------------
// Chain-resident sweeps for small lattices: one CTA per chain copies the
// chain's links into shared memory, runs n_meas x sweeps_per_meas whole
// sweeps there (sub-sweeps separated by block barriers) and writes the links
// back once.  A sweep over a small chain otherwise costs a launch per
// sub-sweep and a global-memory round trip per link; here neither.  Every
// link update is the tiled kernel's arithmetic on the same values, and the
// measured plaquette reproduces ym_average_plaquette's reduction (per-site
// sums, block_reduce per 128-site tile, then the chain reduction's shuffle
// tree over the tile partials), so both paths give the same bits.
// ---- latency-oriented link update for the chain-resident kernel ----------
// A resident launch has only a few hundred threads per sub-sweep, so the
// time of a sub-sweep is the dependent-operation depth of one link update.
// The functions below compute exactly the same values as staple_pipelined/visit
// with less depth: the staple sum stays in registers, the Taylor chains of
// all eight hits (independent of the link) run in lockstep before the
// first hit, the SU(2)-subgroup hits share one formula (so drawn
// generators do not split a warp four ways), and most accept decisions come
// from a bracket around exp(-m) instead of exp itself.

// staple_pipelined's two terms of direction NU, accumulated into a in registers
// (the same fma chains in the same order).
template <int MU, int NU>
__device__ __forceinline__ void add_staple_reg(const double2 *links, const ChainInfo &c,
                                               const Coord &x, int par, const Nb &pm, m3 &a) {
    const Nb pn = step(c, x.x, x.lex, par, NU, +1);
    const Nb mn = step(c, x.x, x.lex, par, NU, -1);
    const Nb mnpm = step(c, x.x, mn.lex, mn.par, MU, +1);
    {
        const m3 l2 = load_su3_rw(links, c, storage_index(c, pn.lex, pn.par), MU);
        const m3 l1 = load_su3_rw(links, c, storage_index(c, pm.lex, pm.par), NU);
        const m3 l3 = load_su3_rw(links, c, storage_index(c, x.lex, par), NU);
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
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int col = 0; col < 3; ++col)
#pragma unroll
                for (int k = 0; k < 3; ++k) cfma(a.e[r][col], p.e[r][k], cconj(l3.e[col][k]));
    }
    {
        const m3 l2 = load_su3_rw(links, c, storage_index(c, mn.lex, mn.par), MU);
        const m3 l1 = load_su3_rw(links, c, storage_index(c, mnpm.lex, mnpm.par), NU);
        const m3 l3 = load_su3_rw(links, c, storage_index(c, mn.lex, mn.par), NU);
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
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int col = 0; col < 3; ++col)
#pragma unroll
                for (int k = 0; k < 3; ++k) cfma(a.e[r][col], p.e[r][k], l3.e[k][col]);
    }
}

// u < exp(-m), m = max(dS, 0), decided as accept_step decides it.  For
// 0 < m <= 1 the alternating series puts exp(-m) between
// L = 1 - m + m^2/2 - m^3/6 and H = 1 - m + m^2/2; widened by 2^-45 (far
// beyond the rounding of L, H and of exp itself, which lies within a few
// ulps of the true value) the bracket decides every draw outside it exactly
// as u < exp(-m) would; exp is evaluated only inside it.
__device__ __forceinline__ bool accept_bracketed(double old_tr, double new_tr, double beta3,
                                                 double unif) {
    const double ds = beta3 * (old_tr - new_tr);
    const double m = fmax(ds, 0.0);
    if (m == 0.0) return true;
    if (m <= 1.0) {
        const double q = (1.0 - m) + 0.5 * (m * m);
        if (unif < q - (m * m) * m * (1.0 / 6.0) - 0x1p-45) return true;
        if (unif >= q + 0x1p-45) return false;
    }
    return unif < exp(-m);
}

__device__ __forceinline__ cplx sel(bool p, cplx a, cplx b) { return cmake(p ? a.re : b.re, p ? a.im : b.im); }

// An SU(2)-subgroup hit for any generator g < 7, rows and A columns picked by
// selects.  Every kind of hit_block writes its candidate entries as
// c*x + s*a with a one of the other entries or its negation
// (c*x - s*y == c*x + s*(-y) exactly), so one formula gives hit_block's bits.
__device__ __forceinline__ void hit_block_any(m3 &u, const m3 &a, double rr[3], double &old_tr,
                                              int g, double c, double s, double beta3, double unif,
                                              unsigned &accepted) {
    const int kind = (g == 2) ? 2 : ((g == 1 || g == 4 || g == 6) ? 1 : 0);
    const int i0 = g <= 4 ? 0 : 1, i1 = g <= 2 ? 1 : 2;
    cplx n0[3], n1[3], col0[3], col1[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const cplx r0 = sel(i0 == 0, u.e[0][k], u.e[1][k]);
        const cplx r1 = sel(i1 == 1, u.e[1][k], u.e[2][k]);
        const double x0 = r0.re, y0 = r0.im, x1 = r1.re, y1 = r1.im;
        const double a0 = kind == 0 ? -y1 : (kind == 1 ? x1 : -y0);
        const double b0 = kind == 0 ? x1 : (kind == 1 ? y1 : x0);
        const double a1 = kind == 0 ? -y0 : (kind == 1 ? -x0 : y1);
        const double b1 = kind == 0 ? x0 : (kind == 1 ? -y0 : -x1);
        n0[k] = cmake(c * x0 + s * a0, c * y0 + s * b0);
        n1[k] = cmake(c * x1 + s * a1, c * y1 + s * b1);
        col0[k] = sel(i0 == 0, a.e[k][0], a.e[k][1]);
        col1[k] = sel(i1 == 1, a.e[k][1], a.e[k][2]);
    }
    const double q0n = retr_row_fma(n0, col0), q1n = retr_row_fma(n1, col1);
    const double q0 = i0 == 0 ? q0n : rr[0];
    const double q1 = i0 == 1 ? q0n : (i1 == 1 ? q1n : rr[1]);
    const double q2 = i1 == 2 ? q1n : rr[2];
    const double new_tr = (q0 + q1) + q2;
    if (accept_bracketed(old_tr, new_tr, beta3, unif)) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            u.e[0][k] = sel(i0 == 0, n0[k], u.e[0][k]);
            u.e[1][k] = sel(i0 == 1, n0[k], sel(i1 == 1, n1[k], u.e[1][k]));
            u.e[2][k] = sel(i1 == 2, n1[k], u.e[2][k]);
        }
        rr[0] = q0;
        rr[1] = q1;
        rr[2] = q2;
        old_tr = new_tr;
        accepted++;
    }
}

__device__ __forceinline__ void hit_diag_reg(m3 &u, const m3 &a, double rr[3], double &old_tr,
                                             cplx e1, cplx e2, double beta3, double unif,
                                             unsigned &accepted) {
    cplx n[3][3];
    double q[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const cplx e = i < 2 ? e1 : e2;
        cplx col[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            n[i][k] = cmul(e, u.e[i][k]);
            col[k] = a.e[k][i];
        }
        q[i] = retr_row_fma(n[i], col);
    }
    const double new_tr = (q[0] + q[1]) + q[2];
    if (accept_bracketed(old_tr, new_tr, beta3, unif)) {
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

// visit()'s eight hits with every rotation computed first.  Chain h of the
// lockstep loop performs exactly taylor_chain's operations on 0.5 theta_h.
__device__ __forceinline__ unsigned visit_resident(m3 &u, const m3 &a, double beta3, double angle,
                                                   uint64_t key, int uniform) {
    int g[8];
    double c[8], s[8], t[8], hx[8], e2r[8], e2i[8];
    unsigned active = 0;
#pragma unroll
    for (int h = 0; h < 8; ++h) {
        const uint64_t w = splitmix_at(key, (uint64_t)(2 * h));
        g[h] = uniform ? (int)((w >> 52) & 7) : h;
        const double theta = grid_angle(w, angle);
        hx[h] = 0.5 * theta;
        t[h] = 1.0;
        c[h] = 1.0;
        s[h] = 0.0;
        e2r[h] = 0.0;
        e2i[h] = 0.0;
        if (g[h] != 7) {
            active |= 1u << h;
        } else {
            cplx e1, e2;
            lambda8_rotation(theta, e1, e2);
            c[h] = e1.re;
            s[h] = e1.im;
            e2r[h] = e2.re;
            e2i[h] = e2.im;
        }
    }
#pragma unroll 1
    for (int k = 1; k <= 64 && active; k += 4) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double inv = c_inv[k + q];
#pragma unroll
            for (int h = 0; h < 8; ++h) {
                if (active & (1u << h)) {
                    t[h] = (t[h] * hx[h]) * inv;
                    if (q == 0) s[h] = s[h] + t[h];
                    else if (q == 1) c[h] = c[h] - t[h];
                    else if (q == 2) s[h] = s[h] - t[h];
                    else c[h] = c[h] + t[h];
                    if (fabs(t[h]) <= kTermCutoff) active &= ~(1u << h);
                }
            }
        }
    }
    double rr[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const cplx col[3] = {a.e[0][i], a.e[1][i], a.e[2][i]};
        rr[i] = retr_row_fma(u.e[i], col);
    }
    double old_tr = (rr[0] + rr[1]) + rr[2];
    unsigned accepted = 0;
#pragma unroll
    for (int h = 0; h < 8; ++h) {
        const double unif = unit_from(splitmix_at(key, (uint64_t)(2 * h + 1)));
        if (g[h] == 7)
            hit_diag_reg(u, a, rr, old_tr, cmake(c[h], s[h]), cmake(e2r[h], e2i[h]), beta3, unif, accepted);
        else
            hit_block_any(u, a, rr, old_tr, g[h], c[h], s[h], beta3, unif, accepted);
    }
    return accepted;
}

template <int MU>
__device__ __forceinline__ unsigned resident_subsweep(const ChainInfo &cs, double2 *sl, int parity,
                                                      double angle, int uniform, uint64_t sweep) {
    unsigned accepted = 0;
    for (int64_t t = threadIdx.x; t < cs.half; t += T) {
        const int64_t s = (int64_t)parity * cs.half + t;
        const Coord x = decode_storage(cs, s);
        m3 a;
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int k = 0; k < 3; ++k) a.e[r][k] = cmake(0.0, 0.0);
        const Nb pm = step(cs, x.x, x.lex, parity, MU, +1);
        if (MU != 0) add_staple_reg<MU, 0>(sl, cs, x, parity, pm, a);
        if (MU != 1) add_staple_reg<MU, 1>(sl, cs, x, parity, pm, a);
        if (MU != 2) add_staple_reg<MU, 2>(sl, cs, x, parity, pm, a);
        if (MU != 3) add_staple_reg<MU, 3>(sl, cs, x, parity, pm, a);
        m3 u = load_su3_rw(sl, cs, s, MU);
        const uint64_t key = link_key(cs.seed, sweep, x.lex, MU);
        accepted += visit_resident(u, a, cs.beta / 3.0, angle, key, uniform);
        store_su3(sl, cs, s, MU, u);
    }
    return accepted;
}

__global__ void __launch_bounds__(T, 1)
k_su3_resident(const ChainInfo *__restrict__ chains, double2 *__restrict__ links, double angle,
               int uniform, const uint64_t *__restrict__ sweep_ptr, int64_t n_meas,
               int64_t sweeps_per_meas, double *__restrict__ series, int64_t n_chains,
               unsigned long long *__restrict__ accepts) {
    extern __shared__ __align__(16) double2 sl[];
    __shared__ double tile_sum[32];
    const int64_t chain = blockIdx.x;
    const ChainInfo c = chains[chain];
    ChainInfo cs = c;
    cs.offset = 0;
    const int64_t n = 36 * c.volume;
    for (int64_t i = threadIdx.x; i < n; i += T) sl[i] = links[c.offset + i];
    __syncthreads();
    const uint64_t sweep0 = *sweep_ptr;
    unsigned accepted = 0;
    for (int64_t m = 0; m < n_meas; ++m) {
        for (int64_t k = 0; k < sweeps_per_meas; ++k) {
            const uint64_t sweep = sweep0 + (uint64_t)(m * sweeps_per_meas + k);
            for (int parity = 0; parity < 2; ++parity) {
                accepted += resident_subsweep<0>(cs, sl, parity, angle, uniform, sweep);
                __syncthreads();
                accepted += resident_subsweep<1>(cs, sl, parity, angle, uniform, sweep);
                __syncthreads();
                accepted += resident_subsweep<2>(cs, sl, parity, angle, uniform, sweep);
                __syncthreads();
                accepted += resident_subsweep<3>(cs, sl, parity, angle, uniform, sweep);
                __syncthreads();
            }
        }
        if (series) {
            const int64_t n_tiles = (c.volume + T - 1) / T;   // at most 32 (resident chains are small)
            for (int64_t tile = 0; tile < n_tiles; ++tile) {
                const int64_t s = tile * T + threadIdx.x;
                double v = s < c.volume ? site_plaquette_sum<true>(sl, cs, s) : 0.0;
                v = block_reduce<false>(v);
                if (threadIdx.x == 0) tile_sum[tile] = v;
                __syncthreads();
            }
            if (threadIdx.x < 32) {
                double v = threadIdx.x < n_tiles ? tile_sum[threadIdx.x] : 0.0;
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
                if (threadIdx.x == 0) series[m * n_chains + chain] = v / (6.0 * (double)c.volume);
            }
            __syncthreads();
        }
    }
    for (int64_t i = threadIdx.x; i < n; i += T) links[c.offset + i] = sl[i];
    const unsigned warp_sum = __reduce_add_sync(0xffffffffu, accepted);
    if ((threadIdx.x & 31) == 0 && warp_sum)
        atomicAdd(accepts + chain, (unsigned long long)warp_sum);
}

__global__ void k_advance_sweep_by(uint64_t *sweep, int64_t n) { *sweep += (uint64_t)n; }

__global__ void k_advance_sweep(uint64_t *sweep) { *sweep += 1; }

}  // namespace

cudaError_t launch_su3_metropolis(ym_ensemble *e, int parity, int mu, double angle, int uniform) {
    if (e->fast_sweeps) return launch_su3_metropolis_fast(e, parity, mu, angle, uniform);
    return tiled_exact::tiled_launch(e, parity, mu, angle, uniform);
}

cudaError_t launch_su3_metropolis_measure(ym_ensemble *e, int mu, double angle, double *tr_partial) {
    if (e->fast_sweeps) return launch_su3_metropolis_measure_fast(e, mu, angle, tr_partial);
    return tiled_exact::tiled_launch_measure(e, mu, angle, tr_partial);
}

size_t resident_smem_bytes(const ym_ensemble *e) {
    int64_t vmax = 0;
    for (const ChainInfo &c : e->chains) vmax = c.volume > vmax ? c.volume : vmax;
    return (size_t)vmax * 36 * sizeof(double2);
}

bool resident_fits(const ym_ensemble *e) {
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return false;
    for (const ChainInfo &c : e->chains)
        if ((c.volume + T - 1) / T > 32) return false;
    // static shared memory of the kernel: tile sums and the reduction's warp
    // slots
    const size_t fixed = sizeof(double) * (32 + 32) + 1024;
    return resident_smem_bytes(e) + fixed <= (size_t)optin;
}

cudaError_t launch_su3_resident(ym_ensemble *e, double angle, int uniform, int64_t n_meas,
                                int64_t sweeps_per_meas, double *series) {
    const size_t smem = resident_smem_bytes(e);
    cudaError_t err = cudaFuncSetAttribute(k_su3_resident, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    k_su3_resident<<<(unsigned)e->n_chains, T, smem, e->stream>>>(e->d_chains, e->d_links, angle, uniform,
                                                                 e->d_sweep, n_meas, sweeps_per_meas,
                                                                 series, e->n_chains, e->d_accepts);
    err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    k_advance_sweep_by<<<1, 1, 0, e->stream>>>(e->d_sweep, n_meas * sweeps_per_meas);
    return cudaGetLastError();
}

cudaError_t launch_advance_sweep(ym_ensemble *e) {
    k_advance_sweep<<<1, 1, 0, e->stream>>>(e->d_sweep);
    return cudaGetLastError();
}

}  // namespace ym
