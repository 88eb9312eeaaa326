// su2_quat.cuh -- SU(2) links as unit quaternions (a0, a1, a2, a3),
// U = a0 I - i a.sigma (reference/rust/src/lib.rs:7-13), stored as two
// double2 planes per direction: (a0, a1) and (a2, a3).  Every product is
// re-normalised exactly as Su2::mul does (lib.rs:106-130, 212-224): divide by
// the largest magnitude, then by the Euclidean norm.  Shared by the sweep
// kernels (su2.cu) and the lattice queries (lattice_ops.cu); include only
// from translation units built with -fmad=false.
#pragma once

#include "ym_device.cuh"

namespace ym {

namespace {

struct q4 {
    double c[4];
};

// normalize_scaled (lib.rs:106-130) for N = 4 or 3 entries.
template <int N>
__device__ __forceinline__ bool normalize_scaled(const double *v, double *out) {
    double scale = 0.0;
#pragma unroll
    for (int i = 0; i < N; ++i) scale = fmax(scale, fabs(v[i]));
    if (scale == 0.0 || !isfinite(scale)) return false;
    double s[N];
#pragma unroll
    for (int i = 0; i < N; ++i) s[i] = v[i] / scale;
    double ss = s[0] * s[0];
#pragma unroll
    for (int i = 1; i < N; ++i) ss = ss + s[i] * s[i];
    const double norm = sqrt(ss);
    if (norm == 0.0 || !isfinite(norm)) return false;
#pragma unroll
    for (int i = 0; i < N; ++i) out[i] = s[i] / norm;
    return true;
}

// Su2::mul (lib.rs:212-224); the raw product is kept if normalisation fails,
// which cannot happen for finite unit inputs (the reference panics there).
__device__ __forceinline__ q4 qmul(const q4 &a, const q4 &b) {
    const double a0 = a.c[0], a1 = a.c[1], a2 = a.c[2], a3 = a.c[3];
    const double b0 = b.c[0], b1 = b.c[1], b2 = b.c[2], b3 = b.c[3];
    double raw[4];
    raw[0] = a0 * b0 - a1 * b1 - a2 * b2 - a3 * b3;
    raw[1] = a0 * b1 + a1 * b0 + a2 * b3 - a3 * b2;
    raw[2] = a0 * b2 - a1 * b3 + a2 * b0 + a3 * b1;
    raw[3] = a0 * b3 + a1 * b2 - a2 * b1 + a3 * b0;
    q4 o;
    if (!normalize_scaled<4>(raw, o.c)) {
#pragma unroll
        for (int i = 0; i < 4; ++i) o.c[i] = raw[i];
    }
    return o;
}

__device__ __forceinline__ q4 qdag(const q4 &a) { return q4{{a.c[0], -a.c[1], -a.c[2], -a.c[3]}}; }

__device__ __forceinline__ q4 load_q(const double2 *__restrict__ links, const ChainInfo &c,
                                     int64_t s, int mu) {
    const double2 *p = links + c.offset + (int64_t)(mu * 2) * c.volume + s;
    const double2 lo = __ldg(p), hi = __ldg(p + c.volume);
    return q4{{lo.x, lo.y, hi.x, hi.y}};
}

__device__ __forceinline__ q4 load_q_rw(const double2 *links, const ChainInfo &c, int64_t s, int mu) {
    const double2 *p = links + c.offset + (int64_t)(mu * 2) * c.volume + s;
    const double2 lo = p[0], hi = p[c.volume];
    return q4{{lo.x, lo.y, hi.x, hi.y}};
}

__device__ __forceinline__ void store_q(double2 *links, const ChainInfo &c, int64_t s, int mu,
                                        const q4 &q) {
    double2 *p = links + c.offset + (int64_t)(mu * 2) * c.volume + s;
    p[0] = make_double2(q.c[0], q.c[1]);
    p[c.volume] = make_double2(q.c[2], q.c[3]);
}

__device__ __forceinline__ q4 link_q(const double2 *links, const ChainInfo &c, const Nb &n, int mu) {
    return load_q(links, c, storage_index(c, n.lex, n.par), mu);
}

}  // namespace

}  // namespace ym
