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

// 1/n! for n = 0..22: each n! is an exact binary64 integer, so each entry is
// the correctly rounded reciprocal.
__constant__ double kInvFactorial[23] = {
    1.0 / 1.0, 1.0 / 1.0, 1.0 / 2.0, 1.0 / 6.0,
    1.0 / 24.0, 1.0 / 120.0, 1.0 / 720.0, 1.0 / 5040.0,
    1.0 / 40320.0, 1.0 / 362880.0, 1.0 / 3628800.0, 1.0 / 39916800.0,
    1.0 / 479001600.0, 1.0 / 6227020800.0, 1.0 / 87178291200.0, 1.0 / 1307674368000.0,
    1.0 / 20922789888000.0, 1.0 / 355687428096000.0, 1.0 / 6402373705728000.0, 1.0 / 121645100408832000.0,
    1.0 / 2432902008176640000.0, 1.0 / 51090942171709440000.0, 1.0 / 1124000727777607680000.0};
constexpr int kMaxOrder = 22;

// Su3::from_algebra_coefficients (su3.rs:255-262, 395-450): algebra matrix
// M = i sum_a c_a T^a accumulated in generator order, scaled by 2^-k to
// 1-norm <= 0.5 (the reference's rule), exponentiated, squared k times.
// The reference sums the dense Taylor series; here the same series runs on
// three scalars: for a traceless 3x3 X, X^3 = h X + d 1 (Cayley-Hamilton,
// h = Tr(X^2)/2, d = det X), so X^n = a_n 1 + b_n X + c_n X^2 with
// (a, b, c)_{n+1} = (d c_n, a_n + h c_n, b_n), and exp(X) = f0 1 + f1 X + f2 X^2.
// Terms stop once a bound on the term matrix's largest entry is <= 1e-18
// (the reference's rule on the dense term; the bound is never below the
// entry, so at most a term more is summed).  With the scaled 1-norm <= 0.5
// the rule fires by order 16 on every coefficient range the gate admits
// (|c_a| <= 64), so the 22-term table is never exhausted.  The result agrees
// with the dense series to rounding (1e-16 per level at the coefficient
// sizes smearing produces).
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
    const m3 x2 = mul(x, x);
    const cplx h = cmake(0.5 * trace3(x2).re, 0.5 * trace3(x2).im);
    const cplx d = det3(x);
    const double nx = max_abs(x), nx2 = max_abs(x2);
    cplx an = cmake(1.0, 0.0), bn = cmake(0.0, 0.0), cn = cmake(0.0, 0.0);
    cplx f0 = an, f1 = bn, f2 = cn;
    for (int order = 1; order <= kMaxOrder; ++order) {
        const cplx a1 = cmul(d, cn), b1 = cadd(an, cmul(h, cn)), c1 = bn;
        an = a1;
        bn = b1;
        cn = c1;
        const double fact = kInvFactorial[order];
        const cplx ta = cmake(an.re * fact, an.im * fact), tb = cmake(bn.re * fact, bn.im * fact),
                   tc = cmake(cn.re * fact, cn.im * fact);
        f0 = cadd(f0, ta);
        f1 = cadd(f1, tb);
        f2 = cadd(f2, tc);
        // |z| <= |re| + |im|: a bound on the largest entry of the term matrix
        const double bound = (fabs(ta.re) + fabs(ta.im)) + (fabs(tb.re) + fabs(tb.im)) * nx +
                             (fabs(tc.re) + fabs(tc.im)) * nx2;
        if (bound <= 1.0e-18) break;
    }
    m3 sum;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            cplx v = cadd(cmul(f1, x.e[i][j]), cmul(f2, x2.e[i][j]));
            if (i == j) v = cadd(v, f0);
            sum.e[i][j] = v;
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
        const m3 old = load_su3(in, c, s, mu);
        const m3 omega = mul_adj(staple, old);
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
        const m3 upd = mul(rot, old);
        if (!in_su3(upd)) { atomicOr(err, kErrGroup); continue; }
        store_su3(out, c, s, mu, upd);
    }
}

}  // namespace

cudaError_t launch_stout_level(ym_ensemble *e, const double2 *in, double2 *out, double rho) {
    k_stout_level<<<(unsigned)e->n_site_tiles, T, 0, e->stream>>>(e->d_chains, e->d_mixed_tiles, in, out,
                                                                 rho, e->d_error);
    return cudaGetLastError();
}

}  // namespace ym
