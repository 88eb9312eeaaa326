// su3_exp.cuh -- exp(i theta T^a) for a single Gell-Mann generator with the
// reference's arithmetic (reference/rust/src/su3.rs:325-450).
//
// For one generator the reference's dense scale-and-square Taylor series
// only ever multiplies a term by one non-zero entry per column, so every
// non-zero entry of every term follows the scalar recurrence
// t_k = (t_{k-1} * h) * fl(1/k) (h the scaled coefficient entry) and the
// zero entries only add exact zeros.  Evaluating that recurrence reproduces
// the reference rotation's non-zero entries bit for bit at a fraction of the
// dense cost.  Include only from translation units built with -fmad=false.
#pragma once

#include "ym_device.cuh"

namespace ym {

#define YM_INV4(k) 1.0 / (k), 1.0 / ((k) + 1), 1.0 / ((k) + 2), 1.0 / ((k) + 3)
// fl(1/k), k = 0..67 (entry 0 unused): the factors Mat3::scale_real(1.0 /
// order) applies (su3.rs:435).  Constant-folded IEEE divisions.
static __constant__ double c_inv[68] = {
    0.0, 1.0, 1.0 / 2, 1.0 / 3, YM_INV4(4), YM_INV4(8), YM_INV4(12), YM_INV4(16),
    YM_INV4(20), YM_INV4(24), YM_INV4(28), YM_INV4(32), YM_INV4(36), YM_INV4(40),
    YM_INV4(44), YM_INV4(48), YM_INV4(52), YM_INV4(56), YM_INV4(60), YM_INV4(64)};
#undef YM_INV4

constexpr double kTermCutoff = 1.0e-18;           // EXP_TERM_CUTOFF su3.rs:25
constexpr double kInvSqrt3 = 0.5773502691896258;  // su3.rs:22

// c = 1 - t2 + t4 ..., s = t1 - t3 + ..., stopping after the first term with
// |t_k| <= 1e-18, at most 64 terms (su3.rs:434-440).  Fully unrolled, so
// every fl(1/k) is an immediate constant operand and the loop carries no
// counter (about 2% of the FP64 sub-sweep).
__device__ __forceinline__ void taylor_chain(double h, double &c, double &s) {
    double t = 1.0;
    c = 1.0;
    s = 0.0;
#pragma unroll
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
#pragma unroll
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

// Generator 8: diag(e1, e1, e2).  The entries of i theta T^8 are
// fl((0.5/sqrt3) theta) twice and fl((-1/sqrt3) theta); the 1-norm
// |theta|/sqrt3 may exceed 0.5 for |theta| > 0.866, giving one squaring.
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

// Dense 3x3 form of the rotation (zeros +0), for the reference-order path.
// Generators 1..7 (indices 0..6): h = fl(0.5 theta) < 0.5 for |theta| <= 1,
// so no squaring; the block is [[c, i s],[i s, c]] (sigma_1 type),
// [[c, s],[-s, c]] (sigma_2 type) or diag(c + i s, c - i s) (sigma_3).
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
    const int i0 = g <= 4 ? 0 : 1;
    const int i1 = g <= 2 ? 1 : 2;
    const int kind = (g == 2) ? 2 : ((g == 1 || g == 4 || g == 6) ? 1 : 0);
    cplx a, b, cc, d;
    if (kind == 0) { a = cmake(c, 0); b = cmake(0, s); cc = cmake(0, s); d = cmake(c, 0); }
    else if (kind == 1) { a = cmake(c, 0); b = cmake(s, 0); cc = cmake(-s, 0); d = cmake(c, 0); }
    else { a = cmake(c, s); b = cmake(0, 0); cc = cmake(0, 0); d = cmake(c, -s); }
    r.e[i0][i0] = a; r.e[i0][i1] = b; r.e[i1][i0] = cc; r.e[i1][i1] = d;
    return r;
}

}  // namespace ym
