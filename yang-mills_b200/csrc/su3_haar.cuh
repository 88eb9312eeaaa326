// su3_haar.cuh -- Haar-random SU(3) links for hot starts.
#pragma once

#include "ym_device.cuh"

namespace ym {

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

// Stream key of link (lex, mu) of a chain's hot start.
__device__ __forceinline__ uint64_t hot_start_key(uint64_t chain_seed, int64_t lex, int mu) {
    return splitmix_at(splitmix_at(chain_seed ^ kHotStartDomain, 0), (uint64_t)(4 * lex + mu));
}

}  // namespace ym
