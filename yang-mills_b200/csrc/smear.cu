// smear.cu -- spatial stout smearing and stride-2 spatial blocking of SU(3)
// lattices (compiled with -fmad=false; the reference's arithmetic).
//
// Stout, one synchronous level (glueball_smearing.rs:137-268): for every
// site and spatial mu,
//   C  = rho * sum_{nu spatial != mu} [ U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag
//                                      + U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu) ]
//   Om = C U^dag,  A = Om^dag - Om,
//   Q  = (i/2) A - (i/6) Tr(A) 1,           checked Hermitian and traceless,
//   c_a = Re Tr(Q lambda_a),                 checked |Im| <= 2e-12,
//   U' = exp(i sum_a c_a T^a) U             (dense scale-and-square Taylor,
//                                            su3.rs:395-450), checked in SU(3);
// temporal links are copied.  A failed gate sets the device error flag
// (the reference returns an error).  Levels ping-pong between two buffers.
//
// Blocking (glueball_blocking.rs:105-136): V_mu(y) = U_mu(2y) U_mu(2y+mu)
// for spatial mu, V_3(y) = U_3(2y), fine site 2y = (2y0, 2y1, 2y2, y3).
#include <cuda_runtime.h>

#include "ym_internal.hpp"

namespace ym {

namespace {

constexpr int T = kSiteThreads;
constexpr double kAlgebraTol = 2.0e-12;   // ALGEBRA_RESIDUAL_TOLERANCE glueball_smearing.rs:26
constexpr double kSu3Tol = 5.0e-12;       // SU3_ACCEPTANCE_TOLERANCE su3.rs:20
constexpr double kInvSqrt3d = 0.5773502691896258;

constexpr unsigned kErrProjection = 4u;
constexpr unsigned kErrGroup = 8u;
constexpr unsigned kErrNonFiniteStaple = 16u;

__device__ __forceinline__ double cabs(cplx z) { return hypot(z.re, z.im); }

__device__ __forceinline__ double max_abs(const m3 &m) {
    double r = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r = fmax(r, cabs(m.e[i][j]));
    return r;
}

__device__ __forceinline__ bool finite3(const m3 &m) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            if (!isfinite(m.e[i][j].re) || !isfinite(m.e[i][j].im)) return false;
    return true;
}

__device__ __forceinline__ m3 sub3(const m3 &a, const m3 &b) {
    m3 o;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) o.e[i][j] = csub(a.e[i][j], b.e[i][j]);
    return o;
}

__device__ __forceinline__ m3 scale_c(const m3 &a, cplx f) {
    m3 o;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) o.e[i][j] = cmul(a.e[i][j], f);
    return o;
}

__device__ __forceinline__ m3 scale_r(const m3 &a, double f) {
    m3 o;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) o.e[i][j] = cmake(a.e[i][j].re * f, a.e[i][j].im * f);
    return o;
}

__device__ __forceinline__ cplx trace3(const m3 &a) { return cadd(cadd(a.e[0][0], a.e[1][1]), a.e[2][2]); }

__device__ __forceinline__ m3 gell_mann(int a) {
    m3 g;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) g.e[i][j] = cmake(0.0, 0.0);
    switch (a) {   // su3.rs:325-348
    case 0: g.e[0][1] = cmake(1, 0); g.e[1][0] = cmake(1, 0); break;
    case 1: g.e[0][1] = cmake(0, -1); g.e[1][0] = cmake(0, 1); break;
    case 2: g.e[0][0] = cmake(1, 0); g.e[1][1] = cmake(-1, 0); break;
    case 3: g.e[0][2] = cmake(1, 0); g.e[2][0] = cmake(1, 0); break;
    case 4: g.e[0][2] = cmake(0, -1); g.e[2][0] = cmake(0, 1); break;
    case 5: g.e[1][2] = cmake(1, 0); g.e[2][1] = cmake(1, 0); break;
    case 6: g.e[1][2] = cmake(0, -1); g.e[2][1] = cmake(0, 1); break;
    default:
        g.e[0][0] = cmake(kInvSqrt3d, 0);
        g.e[1][1] = cmake(kInvSqrt3d, 0);
        g.e[2][2] = cmake(-2.0 * kInvSqrt3d, 0);
        break;
    }
    return g;
}

// Mat3::unitarity_residual / determinant_residual (su3.rs:219-229).
__device__ __forceinline__ double unitarity_res(const m3 &u) {
    m3 a = adj_mul(u, u), b = mul_adj(u, u);
    double r = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const cplx id = cmake(i == j ? 1.0 : 0.0, 0.0);
            r = fmax(r, fmax(cabs(csub(a.e[i][j], id)), cabs(csub(b.e[i][j], id))));
        }
    return r;
}

__device__ __forceinline__ cplx det3(const m3 &m) {
    const cplx t1 = cmul(m.e[0][0], csub(cmul(m.e[1][1], m.e[2][2]), cmul(m.e[1][2], m.e[2][1])));
    const cplx t2 = cmul(m.e[0][1], csub(cmul(m.e[1][0], m.e[2][2]), cmul(m.e[1][2], m.e[2][0])));
    const cplx t3 = cmul(m.e[0][2], csub(cmul(m.e[1][0], m.e[2][1]), cmul(m.e[1][1], m.e[2][0])));
    return cadd(csub(t1, t2), t3);
}

__device__ __forceinline__ bool in_su3(const m3 &u) {
    if (!finite3(u)) return false;
    if (unitarity_res(u) > kSu3Tol) return false;
    const double dd = cabs(csub(det3(u), cmake(1.0, 0.0)));
    const double dg = cabs(csub(det3(adj(u)), cmake(1.0, 0.0)));
    return fmax(dd, dg) <= kSu3Tol;
}

// Su3::from_algebra_coefficients (su3.rs:255-262, 395-450), all eight
// coefficients: algebra matrix accumulated in generator order, times i,
// scale-and-square to 1-norm <= 0.5, Taylor until max |term| <= 1e-18.
__device__ bool from_algebra(const double coef[8], m3 &out) {
    m3 h;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) h.e[i][j] = cmake(0.0, 0.0);
    for (int a = 0; a < 8; ++a) {
        if (!isfinite(coef[a]) || fabs(coef[a]) > 64.0) return false;
        const m3 g = scale_r(scale_r(gell_mann(a), 0.5), coef[a]);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) h.e[i][j] = cadd(h.e[i][j], g.e[i][j]);
    }
    const m3 m = scale_c(h, cmake(0.0, 1.0));
    double norm = 0.0;
    for (int col = 0; col < 3; ++col) {
        double s = 0.0;
        for (int row = 0; row < 3; ++row) s += cabs(m.e[row][col]);
        norm = fmax(norm, s);
    }
    if (!isfinite(norm)) return false;
    int squarings = 0;
    double scaled_norm = norm;
    while (scaled_norm > 0.5) {
        squarings++;
        if (squarings > 32) return false;
        scaled_norm *= 0.5;
    }
    const m3 scaled = scale_r(m, ldexp(1.0, -squarings));
    m3 sum = identity3(), term = identity3();
    for (int order = 1; order <= 64; ++order) {
        term = scale_r(mul(term, scaled), 1.0 / (double)order);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) sum.e[i][j] = cadd(sum.e[i][j], term.e[i][j]);
        if (max_abs(term) <= 1.0e-18) break;
    }
    for (int k = 0; k < squarings; ++k) sum = mul(sum, sum);
    if (!finite3(sum)) return false;
    out = sum;
    return true;
}

__device__ __forceinline__ m3 lk(const double2 *links, const ChainInfo &c, const Nb &n, int mu) {
    return load_su3(links, c, storage_index(c, n.lex, n.par), mu);
}

__global__ void __launch_bounds__(T)
k_stout_level(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
              const double2 *__restrict__ in, double2 *__restrict__ out, double rho,
              unsigned *__restrict__ err) {
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t s = tile.start + threadIdx.x;
    if (s >= c.volume) return;
    const Coord x = decode_storage(c, s);
    const Nb self{x.lex, x.par};
    store_su3(out, c, s, 3, load_su3(in, c, s, 3));           // temporal copied
    for (int mu = 0; mu < 3; ++mu) {
        const m3 old = load_su3(in, c, s, mu);
        const Nb pm = step(c, x.x, x.lex, x.par, mu, +1);
        m3 sum;
        bool first = true;
        for (int nu = 0; nu < 3; ++nu) {
            if (nu == mu) continue;
            const Nb pn = step(c, x.x, x.lex, x.par, nu, +1);
            const Nb mn = step(c, x.x, x.lex, x.par, nu, -1);
            const Nb mnpm = step(c, x.x, mn.lex, mn.par, mu, +1);
            const m3 f = mul_adj(mul(lk(in, c, self, nu), lk(in, c, pn, mu)), lk(in, c, pm, nu));
            if (first) {
                // Mat3::ZERO + f is f entry for entry
                sum = f;
                first = false;
            } else {
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) sum.e[i][j] = cadd(sum.e[i][j], f.e[i][j]);
            }
            const m3 b = mul(adj_mul(lk(in, c, mn, nu), lk(in, c, mn, mu)), lk(in, c, mnpm, nu));
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) sum.e[i][j] = cadd(sum.e[i][j], b.e[i][j]);
        }
        const m3 staple = scale_r(sum, rho);
        if (!finite3(staple)) { atomicOr(err, kErrNonFiniteStaple); continue; }
        // stout_q (glueball_smearing.rs:174-193)
        const m3 omega = mul_adj(staple, old);
        if (!finite3(omega)) { atomicOr(err, kErrNonFiniteStaple); continue; }
        const m3 anti = sub3(adj(omega), omega);
        const m3 firstq = scale_c(anti, cmake(0.0, 0.5));
        const cplx tc = cmul(trace3(anti), cmake(0.0, 1.0));
        const cplx tcs = cmake(tc.re * (1.0 / 6.0), tc.im * (1.0 / 6.0));
        const m3 q = sub3(firstq, scale_c(identity3(), tcs));
        if (!finite3(q)) { atomicOr(err, kErrNonFiniteStaple); continue; }
        if (max_abs(sub3(q, adj(q))) > kAlgebraTol || cabs(trace3(q)) > kAlgebraTol) {
            atomicOr(err, kErrProjection);
            continue;
        }
        // q_coefficients (glueball_smearing.rs:195-205)
        double coef[8];
        bool ok = true;
        for (int a = 0; a < 8; ++a) {
            const cplx p = trace3(mul(q, gell_mann(a)));
            if (!isfinite(p.re) || !isfinite(p.im) || fabs(p.im) > kAlgebraTol) ok = false;
            coef[a] = p.re;
        }
        if (!ok) { atomicOr(err, kErrProjection); continue; }
        m3 rot;
        if (!from_algebra(coef, rot) || !in_su3(rot)) { atomicOr(err, kErrGroup); continue; }
        const m3 upd = mul(rot, old);
        if (!in_su3(upd)) { atomicOr(err, kErrGroup); continue; }
        store_su3(out, c, s, mu, upd);
    }
}

// Coarse chain table entry `cc` of the destination; fine table `fc`.
__global__ void __launch_bounds__(T)
k_block(const ChainInfo *__restrict__ fine_chains, const ChainInfo *__restrict__ coarse_chains,
        const Tile *__restrict__ coarse_tiles, const double2 *__restrict__ fine,
        double2 *__restrict__ coarse, unsigned *__restrict__ err) {
    const Tile tile = coarse_tiles[blockIdx.x];
    const ChainInfo cc = coarse_chains[tile.chain];
    const ChainInfo fc = fine_chains[tile.chain];
    const int64_t s = tile.start + threadIdx.x;
    if (s >= cc.volume) return;
    const Coord y = decode_storage(cc, s);
    int32_t x[4] = {2 * y.x[0], 2 * y.x[1], 2 * y.x[2], y.x[3]};
    const int64_t lex = (((int64_t)x[0] * fc.n[1] + x[1]) * fc.n[2] + x[2]) * fc.n[3] + x[3];
    const int par = (x[0] + x[1] + x[2] + x[3]) & 1;
    for (int mu = 0; mu < 3; ++mu) {
        const Nb pm = step(fc, x, lex, par, mu, +1);
        const m3 b = mul(load_su3(fine, fc, storage_index(fc, lex, par), mu),
                         load_su3(fine, fc, storage_index(fc, pm.lex, pm.par), mu));
        if (!in_su3(b)) {
            atomicOr(err, kErrGroup);
            continue;
        }
        store_su3(coarse, cc, s, mu, b);
    }
    store_su3(coarse, cc, s, 3, load_su3(fine, fc, storage_index(fc, lex, par), 3));
}

}  // namespace

cudaError_t launch_stout_level(ym_ensemble *e, const double2 *in, double2 *out, double rho) {
    k_stout_level<<<(unsigned)e->n_site_tiles, T, 0, e->stream>>>(e->d_chains, e->d_site_tiles, in, out,
                                                                 rho, e->d_error);
    return cudaGetLastError();
}

cudaError_t launch_block(ym_ensemble *fine, ym_ensemble *coarse) {
    k_block<<<(unsigned)coarse->n_site_tiles, T, 0, coarse->stream>>>(
        fine->d_chains, coarse->d_chains, coarse->d_site_tiles, fine->d_links, coarse->d_links,
        coarse->d_error);
    return cudaGetLastError();
}

}  // namespace ym
