// su3_f64.cu -- SU(3) kernels of the FP64 path (compiled with -fmad=false).
//
//   k_su3_metropolis      one checkerboard sub-sweep (parity, mu) of every
//                         chain: staple sum -> eight Metropolis hits -> store
//                         (su3_ensemble.rs:342-391, update rule per link)
//   k_su3_plaquette       per-tile plaquette sums  (su3_ensemble.rs:228-259)
//   k_chain_sum/max       fixed-order per-chain reductions of tile partials
//   k_su3_residuals       unitarity / determinant residuals (su3_lattice.rs:285-297)
//   k_su3_reference_*     the reference's lexicographic single-stream sweep and
//                         sequential plaquette, one thread per chain
//   k_su3_{identity,from_aos,to_aos}  layout conversion, reference <-> SoA
//
// Each link visit draws from its own counter-based SplitMix64 stream (see
// ym_device.cuh); the proposal exponential is evaluated by the scalar Taylor
// recurrence the reference's dense series reduces to for one generator, so
// candidates are bitwise the reference's (su3.rs:409-450).
#include <cuda_runtime.h>

#include "ym_internal.hpp"

namespace ym {

// fl(1/k) for k = 0..67: the factors Mat3::scale_real(1.0 / order) applies
// (su3.rs:435); filled once from the host with IEEE division.
__constant__ double c_inv[68];

// ------------------------------------------------------------ exponential

constexpr double kTermCutoff = 1.0e-18;   // EXP_TERM_CUTOFF su3.rs:25

// Taylor recurrence of one generator: t_k = (t_{k-1} h) fl(1/k); the
// rotation block is c = 1 - t2 + t4 ..., s = t1 - t3 + ....  Stops after the
// first term with |t_k| <= 1e-18, at most 64 terms (su3.rs:434-440).
__device__ __forceinline__ void taylor_chain(double h, double &c, double &s) {
    double t = 1.0;
    c = 1.0;
    s = 0.0;
#pragma unroll 1
    for (int k = 1; k <= 64; k += 4) {
        t = (t * h) * c_inv[k];
        s = s + t;
        if (fabs(t) <= kTermCutoff) return;
        t = (t * h) * c_inv[k + 1];
        c = c - t;
        if (fabs(t) <= kTermCutoff) return;
        t = (t * h) * c_inv[k + 2];
        s = s - t;
        if (fabs(t) <= kTermCutoff) return;
        t = (t * h) * c_inv[k + 3];
        c = c + t;
        if (fabs(t) <= kTermCutoff) return;
    }
}

// Two diagonal chains advanced together (generator 8): the series stops on
// the larger term, as Mat3::max_abs_entry does.
__device__ __forceinline__ void taylor_chain2(double h1, double h2, double &c1, double &s1,
                                              double &c2, double &s2) {
    double t1 = 1.0, t2 = 1.0;
    c1 = 1.0; s1 = 0.0; c2 = 1.0; s2 = 0.0;
#pragma unroll 1
    for (int k = 1; k <= 64; k += 4) {
        t1 = (t1 * h1) * c_inv[k];     t2 = (t2 * h2) * c_inv[k];
        s1 = s1 + t1;                  s2 = s2 + t2;
        if (fmax(fabs(t1), fabs(t2)) <= kTermCutoff) return;
        t1 = (t1 * h1) * c_inv[k + 1]; t2 = (t2 * h2) * c_inv[k + 1];
        c1 = c1 - t1;                  c2 = c2 - t2;
        if (fmax(fabs(t1), fabs(t2)) <= kTermCutoff) return;
        t1 = (t1 * h1) * c_inv[k + 2]; t2 = (t2 * h2) * c_inv[k + 2];
        s1 = s1 - t1;                  s2 = s2 - t2;
        if (fmax(fabs(t1), fabs(t2)) <= kTermCutoff) return;
        t1 = (t1 * h1) * c_inv[k + 3]; t2 = (t2 * h2) * c_inv[k + 3];
        c1 = c1 + t1;                  c2 = c2 + t2;
        if (fmax(fabs(t1), fabs(t2)) <= kTermCutoff) return;
    }
}

// The (scaled) coefficient entries of i*theta*T^a: h = fl(0.5*theta) for the
// seven off-diagonal/sigma_3 generators; for T^8 the diagonal entries are
// fl((0.5/sqrt3)*theta) twice and fl((-1/sqrt3)*theta) (su3.rs:325-352,395-407).
constexpr double kInvSqrt3 = 0.5773502691896258;   // su3.rs:22

// Generator 8 rotation: diag(e1, e1, e2) with at most one squaring for
// |theta| <= 1 (1-norm |theta|/sqrt3 may exceed 0.5).
__device__ __forceinline__ void lambda8_rotation(double theta, cplx &e1, cplx &e2) {
    double d1 = (0.5 * kInvSqrt3) * theta;
    double d2 = (-kInvSqrt3) * theta;
    int sq = 0;
    double nrm = fmax(fabs(d1), fabs(d2));
    while (nrm > 0.5) {
        sq++;
        nrm *= 0.5;
    }
    double sc = ldexp(1.0, -sq);
    double c1, s1, c2, s2;
    taylor_chain2(d1 * sc, d2 * sc, c1, s1, c2, s2);
    e1 = cmake(c1, s1);
    e2 = cmake(c2, s2);
    for (int k = 0; k < sq; ++k) {
        e1 = cmul(e1, e1);
        e2 = cmul(e2, e2);
    }
}

// ------------------------------------------------------------ link visit

// Eight Metropolis hits on link u with staple sum a.  rr[i] caches row i of
// Re Tr(u a); old_tr = (rr0 + rr1) + rr2.  beta3 = beta / 3.
// Candidate rows follow Mat3::mul of the rotation with u: the block rotation
// [[r00, r01], [r10, r11]] enters in ascending index order; untouched rows are
// bitwise unchanged.  Returns the number of accepted hits.
template <int I0, int I1>
__device__ __forceinline__ void try_block(m3 &u, const m3 &a, double rr[3], double &old_tr,
                                          int kind, double c, double s, double beta3, double unif,
                                          unsigned &accepted) {
    cplx n0[3], n1[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double x0 = u.e[I0][k].re, y0 = u.e[I0][k].im;
        const double x1 = u.e[I1][k].re, y1 = u.e[I1][k].im;
        if (kind == 0) {          // i h sigma_1: [[c, i s], [i s, c]]
            n0[k] = cmake(c * x0 - s * y1, c * y0 + s * x1);
            n1[k] = cmake(c * x1 - s * y0, s * x0 + c * y1);
        } else if (kind == 1) {   // i h sigma_2: [[c, s], [-s, c]]
            n0[k] = cmake(c * x0 + s * x1, c * y0 + s * y1);
            n1[k] = cmake(c * x1 - s * x0, c * y1 - s * y0);
        } else {                  // i h sigma_3: diag(c + i s, c - i s)
            n0[k] = cmake(c * x0 - s * y0, c * y0 + s * x0);
            n1[k] = cmake(c * x1 + s * y1, c * y1 - s * x1);
        }
    }
    double q[3] = {rr[0], rr[1], rr[2]};
    q[I0] = retr_row(n0, a, I0);
    q[I1] = retr_row(n1, a, I1);
    const double new_tr = (q[0] + q[1]) + q[2];
    const double ds = beta3 * (old_tr - new_tr);
    const double m = fmax(ds, 0.0);
    const bool accept = (m == 0.0) ? true : (unif < exp(-m));
    if (accept) {
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

__device__ __forceinline__ void try_diag(m3 &u, const m3 &a, double rr[3], double &old_tr,
                                         cplx e1, cplx e2, double beta3, double unif,
                                         unsigned &accepted) {
    cplx n[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const cplx e = i < 2 ? e1 : e2;
#pragma unroll
        for (int k = 0; k < 3; ++k) n[i][k] = cmul(e, u.e[i][k]);
    }
    double q[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) q[i] = retr_row(n[i], a, i);
    const double new_tr = (q[0] + q[1]) + q[2];
    const double ds = beta3 * (old_tr - new_tr);
    const double m = fmax(ds, 0.0);
    const bool accept = (m == 0.0) ? true : (unif < exp(-m));
    if (accept) {
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

__device__ __forceinline__ unsigned visit_link(m3 &u, const m3 &a, double beta3, double angle,
                                               uint64_t key, int uniform) {
    double rr[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) rr[i] = retr_row(u.e[i], a, i);
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
            try_diag(u, a, rr, old_tr, e1, e2, beta3, unif, accepted);
        } else {
            double c, s;
            taylor_chain(0.5 * theta, c, s);   // |0.5 theta| < 0.5: no squaring
            const int kind = (g == 2) ? 2 : ((g == 1 || g == 4 || g == 6) ? 1 : 0);
            if (g <= 2)
                try_block<0, 1>(u, a, rr, old_tr, kind, c, s, beta3, unif, accepted);
            else if (g <= 4)
                try_block<0, 2>(u, a, rr, old_tr, kind, c, s, beta3, unif, accepted);
            else
                try_block<1, 2>(u, a, rr, old_tr, kind, c, s, beta3, unif, accepted);
        }
    }
    return accepted;
}

// Staple sum of link (x, mu): sum over nu != mu (ascending) of
//   U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag  +  U_nu(x-nu+mu)^dag U_mu(x-nu)^dag U_nu(x-nu),
// the SU(3) form of Lattice4::staple (lib.rs:507-546).  x has parity par.
__device__ __forceinline__ m3 staple_sum(const double2 *__restrict__ links, const ChainInfo &c,
                                         const Coord &x, int par, int mu) {
    m3 acc;
    bool first = true;
    const int opp = par ^ 1;
    const int64_t lex_pm = shift_lex(c, x.x, x.lex, mu, +1);
#pragma unroll 1
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == mu) continue;
        const int64_t lex_pn = shift_lex(c, x.x, x.lex, nu, +1);
        const int64_t lex_mn = shift_lex(c, x.x, x.lex, nu, -1);
        const int64_t lex_mnpm = shift_lex(c, x.x, lex_mn, mu, +1);
        {
            m3 p = mul_adj(load_su3(links, c, storage_index(c, lex_pm, opp), nu),
                           load_su3(links, c, storage_index(c, lex_pn, opp), mu));
            m3 f = mul_adj(p, load_su3(links, c, storage_index(c, x.lex, par), nu));
            if (first) {
                acc = f;
                first = false;
            } else {
                add_into(acc, f);
            }
        }
        {
            m3 p = adj_mul_adj(load_su3(links, c, storage_index(c, lex_mnpm, par), nu),
                               load_su3(links, c, storage_index(c, lex_mn, opp), mu));
            m3 b = mul(p, load_su3(links, c, storage_index(c, lex_mn, opp), nu));
            add_into(acc, b);
        }
    }
    return acc;
}

__global__ void __launch_bounds__(kSweepThreads)
k_su3_metropolis(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                 double2 *__restrict__ links, int parity, int mu, double angle, int uniform,
                 const uint64_t *__restrict__ sweep_ptr, unsigned long long *__restrict__ accepts) {
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t t = tile.start + threadIdx.x;
    unsigned accepted = 0;
    if (t < c.half) {
        const int64_t s = (int64_t)parity * c.half + t;
        const Coord x = decode_storage(c, s);
        const m3 a = staple_sum(links, c, x, parity, mu);
        m3 u = load_su3_rw(links, c, s, mu);
        const uint64_t key = link_key(c.seed, *sweep_ptr, x.lex, mu);
        accepted = visit_link(u, a, c.beta / 3.0, angle, key, uniform);
        store_su3(links, c, s, mu, u);
    }
    const unsigned warp_sum = __reduce_add_sync(0xffffffffu, accepted);
    if ((threadIdx.x & 31) == 0 && warp_sum) atomicAdd(accepts + tile.chain, (unsigned long long)warp_sum);
}

__global__ void k_advance_sweep(uint64_t *sweep) { *sweep += 1; }

// ------------------------------------------------------------ reductions

template <bool kMax>
__device__ __forceinline__ double block_reduce(double v) {
    __shared__ double warp_vals[32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const double o = __shfl_down_sync(0xffffffffu, v, off);
        v = kMax ? fmax(v, o) : v + o;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) warp_vals[warp] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    if (warp == 0) {
        v = lane < nw ? warp_vals[lane] : (kMax ? 0.0 : 0.0);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_down_sync(0xffffffffu, v, off);
            v = kMax ? fmax(v, o) : v + o;
        }
    }
    return v;   // valid in thread 0
}

// Sum of the six plaquette values (1/3) Re Tr P of each site, site order
// (mu, nu) = (0,1),(0,2),(0,3),(1,2),(1,3),(2,3), per tile.
__global__ void __launch_bounds__(kSiteThreads)
k_su3_plaquette(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                const double2 *__restrict__ links, double *__restrict__ partial) {
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t s = tile.start + threadIdx.x;
    double v = 0.0;
    if (s < c.volume) {
        const Coord x = decode_storage(c, s);
        bool first = true;
#pragma unroll 1
        for (int mu = 0; mu < 3; ++mu) {
            const m3 umu = load_su3(links, c, s, mu);
            const int64_t lex_pm = shift_lex(c, x.x, x.lex, mu, +1);
            const int opp = x.par ^ 1;
#pragma unroll 1
            for (int nu = mu + 1; nu < 4; ++nu) {
                const int64_t lex_pn = shift_lex(c, x.x, x.lex, nu, +1);
                m3 p = mul(umu, load_su3(links, c, storage_index(c, lex_pm, opp), nu));
                p = mul_adj(p, load_su3(links, c, storage_index(c, lex_pn, opp), mu));
                const double val = retrace_mul_adj(p, load_su3(links, c, s, nu)) / 3.0;
                v = first ? val : v + val;
                first = false;
            }
        }
    }
    v = block_reduce<false>(v);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
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

__device__ __forceinline__ m3 generator_rotation_dense(int g, double theta) {
    m3 r = identity3();
    if (g == 7) {
        cplx e1, e2;
        lambda8_rotation(theta, e1, e2);
        r.e[0][0] = e1;
        r.e[1][1] = e1;
        r.e[2][2] = e2;
        return r;
    }
    double c, s;
    taylor_chain(0.5 * theta, c, s);
    const int i0 = g <= 2 ? 0 : (g <= 4 ? 0 : 1);
    const int i1 = g <= 2 ? 1 : (g <= 4 ? 2 : 2);
    const int kind = (g == 2) ? 2 : ((g == 1 || g == 4 || g == 6) ? 1 : 0);
    cplx a, b, cc, d;
    if (kind == 0) { a = cmake(c, 0); b = cmake(0, s); cc = cmake(0, s); d = cmake(c, 0); }
    else if (kind == 1) { a = cmake(c, 0); b = cmake(s, 0); cc = cmake(-s, 0); d = cmake(c, 0); }
    else { a = cmake(c, s); b = cmake(0, 0); cc = cmake(0, 0); d = cmake(c, -s); }
    r.e[i0][i0] = a; r.e[i0][i1] = b; r.e[i1][i0] = cc; r.e[i1][i1] = d;
    return r;
}

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

// Haar-random SU(3) link from its own stream (no reference counterpart: the
// reference always starts cold).  Method: two rows of independent complex
// Gaussians (Box-Muller), Gram-Schmidt, third row the conjugate cross product
// of the first two, which fixes det = 1 -- the QR construction of Haar
// measure on U(3) (Mezzadri 2007) restricted to SU(3).
__device__ __forceinline__ m3 haar_su3(uint64_t key) {
    double g[12];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const double u1 = 1.0 - unit_from(splitmix_at(key, 2 * i));   // (0, 1]
        const double u2 = unit_from(splitmix_at(key, 2 * i + 1));
        const double r = sqrt(-2.0 * log(u1));
        double sn, cs;
        sincospi(2.0 * u2, &sn, &cs);
        g[2 * i] = r * cs;
        g[2 * i + 1] = r * sn;
    }
    m3 u;
    double n0 = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        u.e[0][k] = cmake(g[2 * k], g[2 * k + 1]);
        n0 += g[2 * k] * g[2 * k] + g[2 * k + 1] * g[2 * k + 1];
    }
    n0 = 1.0 / sqrt(n0);
#pragma unroll
    for (int k = 0; k < 3; ++k) u.e[0][k] = cmake(u.e[0][k].re * n0, u.e[0][k].im * n0);
    cplx dot = cmake(0.0, 0.0);   // <row0, row1> = sum conj(r0_k) r1_k
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        u.e[1][k] = cmake(g[6 + 2 * k], g[7 + 2 * k]);
        dot = cadd(dot, cmul(cconj(u.e[0][k]), u.e[1][k]));
    }
    double n1 = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        u.e[1][k] = csub(u.e[1][k], cmul(dot, u.e[0][k]));
        n1 += u.e[1][k].re * u.e[1][k].re + u.e[1][k].im * u.e[1][k].im;
    }
    n1 = 1.0 / sqrt(n1);
#pragma unroll
    for (int k = 0; k < 3; ++k) u.e[1][k] = cmake(u.e[1][k].re * n1, u.e[1][k].im * n1);
    // row2 = conj(row0 x row1)
    u.e[2][0] = cconj(csub(cmul(u.e[0][1], u.e[1][2]), cmul(u.e[0][2], u.e[1][1])));
    u.e[2][1] = cconj(csub(cmul(u.e[0][2], u.e[1][0]), cmul(u.e[0][0], u.e[1][2])));
    u.e[2][2] = cconj(csub(cmul(u.e[0][0], u.e[1][1]), cmul(u.e[0][1], u.e[1][0])));
    return u;
}

constexpr uint64_t kHotStartDomain = 0x484F5453544152ULL;   // "HOTSTAR"

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

__global__ void k_su3_identity(double2 *links, int64_t offset, int64_t volume) {
    const int64_t n = 36 * volume;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int entry = (int)((i / volume) % 9);
        links[offset + i] = make_double2((entry == 0 || entry == 4 || entry == 8) ? 1.0 : 0.0, 0.0);
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

// __constant__ memory is per device: fill it once on every device used.
static cudaError_t ensure_constants() {
    static bool done[128] = {};
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (dev < 0 || dev >= 128) return cudaErrorInvalidDevice;
    if (done[dev]) return cudaSuccess;
    double inv[68];
    inv[0] = 0.0;
    for (int k = 1; k < 68; ++k) inv[k] = 1.0 / (double)k;
    err = cudaMemcpyToSymbol(c_inv, inv, sizeof inv);
    if (err == cudaSuccess) done[dev] = true;
    return err;
}

static int grid_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b > 148 * 16) b = 148 * 16;
    return (int)(b < 1 ? 1 : b);
}

cudaError_t launch_su3_identity(ym_ensemble *e) {
    for (int64_t ch = 0; ch < e->n_chains; ++ch) {
        const ChainInfo &c = e->chains[ch];
        k_su3_identity<<<grid_for(36 * c.volume, 256), 256, 0, e->stream>>>(e->d_links, c.offset, c.volume);
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

cudaError_t launch_su3_metropolis(ym_ensemble *e, int parity, int mu, double angle, int uniform) {
    cudaError_t err = ensure_constants();
    if (err != cudaSuccess) return err;
    k_su3_metropolis<<<(unsigned)e->n_half_tiles, kSweepThreads, 0, e->stream>>>(
        e->d_chains, e->d_half_tiles, e->d_links, parity, mu, angle, uniform, e->d_sweep,
        e->d_accepts);
    return cudaGetLastError();
}

cudaError_t launch_advance_sweep(ym_ensemble *e) {
    k_advance_sweep<<<1, 1, 0, e->stream>>>(e->d_sweep);
    return cudaGetLastError();
}

cudaError_t launch_su3_plaquette(ym_ensemble *e) {
    k_su3_plaquette<<<(unsigned)e->n_site_tiles, kSiteThreads, 0, e->stream>>>(
        e->d_chains, e->d_site_tiles, e->d_links, e->d_partial);
    k_chain_reduce<<<(unsigned)e->n_chains, 256, 0, e->stream>>>(
        e->d_partial, e->d_site_tile_first, e->d_chains, e->d_result, 0, 6.0);
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
    cudaError_t err = ensure_constants();
    if (err != cudaSuccess) return err;
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
