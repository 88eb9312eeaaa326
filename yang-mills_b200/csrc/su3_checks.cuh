// su3_checks.cuh -- the gauge-observable units' dense 3x3 helpers and the
// reference's acceptance gates (finite entries, unitarity and determinant
// residuals) shared by stout smearing and blocking.
#pragma once

#include "ym_device.cuh"

namespace ym {

namespace {

constexpr double kAlgebraTol = 2.0e-12;   // ALGEBRA_RESIDUAL_TOLERANCE glueball_smearing.rs:26
constexpr double kSu3Tol = 5.0e-12;       // SU3_ACCEPTANCE_TOLERANCE su3.rs:20
constexpr double kInvSqrt3d = 0.5773502691896258;

constexpr unsigned kErrProjection = 4u;
constexpr unsigned kErrGroup = 8u;
constexpr unsigned kErrNonFiniteStaple = 16u;

__device__ __forceinline__ double cabs(cplx z) { return hypot(z.re, z.im); }

__device__ __forceinline__ double norm2(cplx z) { return z.re * z.re + z.im * z.im; }

// max |m_ij|, compared through squared magnitudes (one sqrt at the end)
__device__ __forceinline__ double max_abs(const m3 &m) {
    double r = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r = fmax(r, norm2(m.e[i][j]));
    return sqrt(r);
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

__device__ __forceinline__ cplx det3(const m3 &m) {
    const cplx t1 = cmul(m.e[0][0], csub(cmul(m.e[1][1], m.e[2][2]), cmul(m.e[1][2], m.e[2][1])));
    const cplx t2 = cmul(m.e[0][1], csub(cmul(m.e[1][0], m.e[2][2]), cmul(m.e[1][2], m.e[2][0])));
    const cplx t3 = cmul(m.e[0][2], csub(cmul(m.e[1][0], m.e[2][1]), cmul(m.e[1][1], m.e[2][0])));
    return cadd(csub(t1, t2), t3);
}

// Square of Mat3::unitarity_residual (su3.rs:219-223): max |U^dag U - 1|^2
// and |U U^dag - 1|^2 over all entries.  Both products are Hermitian, so
// the upper triangle (diagonal included) carries every distinct magnitude;
// only those six entries of each are formed.
__device__ __forceinline__ double unitarity_res2(const m3 &u) {
    double r = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const double dl = norm2(u.e[0][i]) + norm2(u.e[1][i]) + norm2(u.e[2][i]) - 1.0;
        const double dr = norm2(u.e[i][0]) + norm2(u.e[i][1]) + norm2(u.e[i][2]) - 1.0;
        r = fmax(r, fmax(dl * dl, dr * dr));
#pragma unroll
        for (int j = i + 1; j < 3; ++j) {
            cplx l = cmul(cconj(u.e[0][i]), u.e[0][j]);
            l = cadd(l, cmul(cconj(u.e[1][i]), u.e[1][j]));
            l = cadd(l, cmul(cconj(u.e[2][i]), u.e[2][j]));
            cplx g = cmul(u.e[i][0], cconj(u.e[j][0]));
            g = cadd(g, cmul(u.e[i][1], cconj(u.e[j][1])));
            g = cadd(g, cmul(u.e[i][2], cconj(u.e[j][2])));
            r = fmax(r, fmax(norm2(l), norm2(g)));
        }
    }
    return r;
}

// Su3::from_checked_matrix gate (su3.rs:20, 241-252): finite, unitarity residual
// and |det U - 1| within 5e-12.  The reference also takes |det(U^dag) - 1|,
// which is the same number (det U^dag is the conjugate of det U).
__device__ __forceinline__ bool in_su3(const m3 &u) {
    if (!finite3(u)) return false;
    if (unitarity_res2(u) > kSu3Tol * kSu3Tol) return false;
    return norm2(csub(det3(u), cmake(1.0, 0.0))) <= kSu3Tol * kSu3Tol;
}

}  // namespace

}  // namespace ym
