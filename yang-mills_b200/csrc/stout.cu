// stout.cu -- spatial stout smearing of SU(3) lattices, one synchronous
// level per launch (glueball_smearing.rs:137-268): for every site and
// spatial mu,
//   C  = rho * sum_{nu spatial != mu} [ U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag
//                                      + U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu) ]
//   Om = C U^dag,  A = Om^dag - Om,
//   Q  = (i/2) A - (i/6) Tr(A) 1,           checked Hermitian and traceless,
//   c_a = Re Tr(Q lambda_a),                 checked |Im| <= 2e-12,
//   U' = exp(i sum_a c_a T^a) U             (scale-and-square exponential,
//                                            su3.rs:395-450), checked in SU(3);
// temporal links are copied.  A failed gate sets the device error flag
// (the reference returns an error).  Levels ping-pong between two buffers.
//
// Results are held to a tolerance (1e-14 against the oracle per level, the
// reference goldens' 1e-12), not bitwise, so this unit is compiled with
// fused multiply-adds.
#include <cuda_runtime.h>

#include "su3_checks.cuh"
#include "ym_internal.hpp"

namespace ym {

namespace {

constexpr int T = kSiteThreads;

// 1/k for k = 0..22 (entry 0 unused), correctly rounded.
__constant__ double kInvInt[23] = {
    0.0, 1.0 / 1, 1.0 / 2, 1.0 / 3, 1.0 / 4, 1.0 / 5, 1.0 / 6, 1.0 / 7, 1.0 / 8, 1.0 / 9, 1.0 / 10,
    1.0 / 11, 1.0 / 12, 1.0 / 13, 1.0 / 14, 1.0 / 15, 1.0 / 16, 1.0 / 17, 1.0 / 18, 1.0 / 19,
    1.0 / 20, 1.0 / 21, 1.0 / 22};
constexpr int kMaxOrder = 22;

// Su3::from_algebra_coefficients (su3.rs:255-262, 395-450): algebra matrix
// M = i sum_a c_a T^a accumulated in generator order, scaled by 2^-k to
// 1-norm <= 0.5 (the reference's rule), exponentiated, squared k times.
// The reference sums the dense Taylor series until a term's largest entry
// is <= 1e-18; here the same series runs on three scalars: for a traceless
// 3x3 X, X^3 = h X + d 1 (Cayley-Hamilton, h = Tr(X^2)/2, d = det X), so a
// polynomial in X is a 1 + b X + c X^2 and exp(X) = f0 1 + f1 X + f2 X^2.
// The order N is fixed before summing, as the first n with
// ||X||_1^n / n! <= 1e-18 (a bound on every entry of the n-th term, so N is
// at least the reference's stopping order and each extra term is below
// 1e-18), and the series is evaluated by Horner's rule.  With the scaled
// 1-norm <= 0.5, N <= 16 on every coefficient range the gate admits
// (|c_a| <= 64), so the 22-entry table is never exhausted.  The result
// agrees with the dense series to rounding (1e-16 per level at the
// coefficient sizes smearing produces).
__device__ __forceinline__ bool from_algebra(const double coef[8], m3 &out) {
#pragma unroll
    for (int a = 0; a < 8; ++a)
        if (!isfinite(coef[a]) || fabs(coef[a]) > 64.0) return false;
    // M = i * sum_a c_a lambda_a / 2, entries written out
    const double h3 = 0.5 * coef[2], h8 = 0.5 * kInvSqrt3d * coef[7];
    m3 hm;
    hm.e[0][0] = cmake(h3 + h8, 0.0);
    hm.e[1][1] = cmake(-h3 + h8, 0.0);
    hm.e[2][2] = cmake(-2.0 * h8, 0.0);
    hm.e[0][1] = cmake(0.5 * coef[0], -0.5 * coef[1]);
    hm.e[1][0] = cmake(0.5 * coef[0], 0.5 * coef[1]);
    hm.e[0][2] = cmake(0.5 * coef[3], -0.5 * coef[4]);
    hm.e[2][0] = cmake(0.5 * coef[3], 0.5 * coef[4]);
    hm.e[1][2] = cmake(0.5 * coef[5], -0.5 * coef[6]);
    hm.e[2][1] = cmake(0.5 * coef[5], 0.5 * coef[6]);
    const m3 m = scale_c(hm, cmake(0.0, 1.0));
    // 1-norm (max column sum of |m_rc|); m is i times a Hermitian matrix, so
    // |m_rc| = |m_cr| and three square roots cover the off-diagonal entries
    const double o01 = sqrt(norm2(m.e[0][1])), o02 = sqrt(norm2(m.e[0][2])),
                 o12 = sqrt(norm2(m.e[1][2]));
    const double d0 = fabs(m.e[0][0].im), d1 = fabs(m.e[1][1].im), d2 = fabs(m.e[2][2].im);
    const double norm = fmax(fmax((d0 + o01) + o02, (o01 + d1) + o12), (o02 + o12) + d2);
    if (!isfinite(norm)) return false;
    int squarings = 0;
    double scaled_norm = norm;
    while (scaled_norm > 0.5) {
        squarings++;
        if (squarings > 32) return false;
        scaled_norm *= 0.5;
    }
    const m3 x = scale_r(m, ldexp(1.0, -squarings));
    const m3 x2 = mul_fma(x, x);
    const cplx h = cmake(0.5 * trace3(x2).re, 0.5 * trace3(x2).im);
    const cplx d = det3(x);
    // Terms through order N, N the first order whose term is below 1e-18
    // by the a-priori bound |(X^n / n!)_ij| <= ||X||_1^n / n! (so at least
    // the terms the running test would sum; every extra term is below
    // 1e-18), then Horner's rule on the three scalars:
    // F_k = 1 + (X / k) F_{k+1}, X (a + b X + c X^2) = c d + (a + c h) X + b X^2.
    int order = 0;
    for (double t = 1.0; t > 1.0e-18 && order < kMaxOrder;) {
        ++order;
        t *= scaled_norm * kInvInt[order];
    }
    cplx fa = cmake(1.0, 0.0), fb = cmake(0.0, 0.0), fc = cmake(0.0, 0.0);
    for (int k = order; k >= 1; --k) {
        const double inv = kInvInt[k];
        const cplx na = cmul(fc, d), nb = cadd(fa, cmul(fc, h)), nc = fb;
        fa = cmake(1.0 + na.re * inv, na.im * inv);
        fb = cmake(nb.re * inv, nb.im * inv);
        fc = cmake(nc.re * inv, nc.im * inv);
    }
    const cplx f0 = fa, f1 = fb, f2 = fc;
    m3 sum;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            cplx v = cadd(cmul(f1, x.e[i][j]), cmul(f2, x2.e[i][j]));
            if (i == j) v = cadd(v, f0);
            sum.e[i][j] = v;
        }
    for (int k = 0; k < squarings; ++k) sum = mul_fma(sum, sum);
    if (!finite3(sum)) return false;
    out = sum;
    return true;
}

// a^dagger b, every entry one chain of cfma() over k = 0, 1, 2 from zero.
__device__ __forceinline__ m3 adj_mul_fma(const m3 &a, const m3 &b) {
    m3 o;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            cplx v = cmake(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < 3; ++k) cfma(v, cconj(a.e[k][r]), b.e[k][c]);
            o.e[r][c] = v;
        }
    return o;
}

__device__ __forceinline__ m3 lk(const double2 *links, const ChainInfo &c, const Nb &n, int mu) {
    return load_su3(links, c, storage_index(c, n.lex, n.par), mu);
}

// Three blocks per SM: 168 registers (56 bytes spilled) measured 10 %
// faster than two blocks at 254.
__global__ void __launch_bounds__(T, 3)
k_stout_level(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
              const double2 *__restrict__ in, double2 *__restrict__ out, double rho,
              unsigned *__restrict__ err, int reverse) {
    const Tile tile = tiles[reverse ? gridDim.x - 1 - blockIdx.x : blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t s = tile.start + threadIdx.x;
    if (s >= c.volume) return;
    const Coord x = decode_storage(c, s);
    const Nb self{x.lex, x.par};
    store_su3(out, c, s, 3, load_su3(in, c, s, 3));           // temporal copied
    for (int mu = 0; mu < 3; ++mu) {
        const Nb pm = step_any(c, x.x, x.lex, x.par, mu, +1);
        m3 sum;
        bool first = true;
        for (int nu = 0; nu < 3; ++nu) {
            if (nu == mu) continue;
            const Nb pn = step_any(c, x.x, x.lex, x.par, nu, +1);
            const Nb mn = step_any(c, x.x, x.lex, x.par, nu, -1);
            const Nb mnpm = step_any(c, x.x, mn.lex, mn.par, mu, +1);
            const m3 f = mul_adj_fma(mul_fma(lk(in, c, self, nu), lk(in, c, pn, mu)), lk(in, c, pm, nu));
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
            const m3 b = mul_fma(adj_mul_fma(lk(in, c, mn, nu), lk(in, c, mn, mu)), lk(in, c, mnpm, nu));
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) sum.e[i][j] = cadd(sum.e[i][j], b.e[i][j]);
        }
        const m3 staple = scale_r(sum, rho);
        if (!finite3(staple)) { atomicOr(err, kErrNonFiniteStaple); continue; }
        // stout_q (glueball_smearing.rs:174-193)
        const m3 old = load_su3(in, c, s, mu);
        const m3 omega = mul_adj_fma(staple, old);
        if (!finite3(omega)) { atomicOr(err, kErrNonFiniteStaple); continue; }
        const m3 anti = sub3(adj(omega), omega);
        const m3 firstq = scale_c(anti, cmake(0.0, 0.5));
        const cplx tc = cmul(trace3(anti), cmake(0.0, 1.0));
        const cplx tcs = cmake(tc.re * (1.0 / 6.0), tc.im * (1.0 / 6.0));
        const m3 q = sub3(firstq, scale_c(identity3(), tcs));
        if (!finite3(q)) { atomicOr(err, kErrNonFiniteStaple); continue; }
        if (max_abs(sub3(q, adj(q))) > kAlgebraTol || norm2(trace3(q)) > kAlgebraTol * kAlgebraTol) {
            atomicOr(err, kErrProjection);
            continue;
        }
        // q_coefficients (glueball_smearing.rs:195-205)
        // Tr(Q lambda_a) = sum_{i,k} Q_ik (lambda_a)_ki, written out
        const cplx I1 = cmake(0.0, 1.0);
        cplx pa[8];
        pa[0] = cadd(q.e[0][1], q.e[1][0]);
        pa[1] = csub(cmul(q.e[0][1], I1), cmul(q.e[1][0], I1));
        pa[2] = csub(q.e[0][0], q.e[1][1]);
        pa[3] = cadd(q.e[0][2], q.e[2][0]);
        pa[4] = csub(cmul(q.e[0][2], I1), cmul(q.e[2][0], I1));
        pa[5] = cadd(q.e[1][2], q.e[2][1]);
        pa[6] = csub(cmul(q.e[1][2], I1), cmul(q.e[2][1], I1));
        {
            const cplx s01 = cadd(q.e[0][0], q.e[1][1]);
            pa[7] = csub(cmake(s01.re * kInvSqrt3d, s01.im * kInvSqrt3d),
                         cmake(q.e[2][2].re * (2.0 * kInvSqrt3d), q.e[2][2].im * (2.0 * kInvSqrt3d)));
        }
        double coef[8];
        bool ok = true;
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            const cplx p = pa[a];
            if (!isfinite(p.re) || !isfinite(p.im) || fabs(p.im) > kAlgebraTol) ok = false;
            coef[a] = p.re;
        }
        if (!ok) { atomicOr(err, kErrProjection); continue; }
        m3 rot;
        if (!from_algebra(coef, rot) || !in_su3(rot)) { atomicOr(err, kErrGroup); continue; }
        const m3 upd = mul_fma(rot, old);
        if (!in_su3(upd)) { atomicOr(err, kErrGroup); continue; }
        store_su3(out, c, s, mu, upd);
    }
}

}  // namespace

cudaError_t launch_stout_level(ym_ensemble *e, const double2 *in, double2 *out, double rho, int reverse) {
    k_stout_level<<<(unsigned)e->n_site_tiles, T, 0, e->stream>>>(e->d_chains, e->d_mixed_tiles, in, out,
                                                                 rho, e->d_error, reverse);
    return cudaGetLastError();
}

}  // namespace ym
