// su3_sites.cuh -- per-site SU(3) FP64 measurement pieces shared by the
// tiled measurement kernels (su3_f64.cu) and the chain-resident sweep kernel
// (su3_metropolis.cu), so both produce the same bits.  Include only from
// translation units built with -fmad=false.
#pragma once

#include "ym_device.cuh"

namespace ym {

// A link from global memory (read-only path) or, RESIDENT, from a chain copy
// in shared memory (generic loads).
template <bool RESIDENT>
__device__ __forceinline__ m3 link_at(const double2 *links, const ChainInfo &c, int64_t s, int mu) {
    return RESIDENT ? load_su3_rw(links, c, s, mu) : load_su3(links, c, s, mu);
}

// Fixed-shape block reduction: a shuffle-down tree within each warp, then
// the warp results (zeros past the last warp) by the same tree in warp 0.
// The result is valid in thread 0.
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

// Sum over the six planes of (1/3) Re Tr of the site's plaquettes, in the
// order (mu, nu) = (0,1),(0,2),(0,3),(1,2),(1,3),(2,3); each product in the
// reference's orientation U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag, its
// two matrix products as fma() chains (within 1e-12 relative of the
// reference's plaquette; the tiled and chain-resident paths share this code
// and so agree bitwise).
template <bool RESIDENT>
__device__ __forceinline__ double site_plaquette_sum(const double2 *links, const ChainInfo &c,
                                                     int64_t s) {
    const Coord x = decode_storage(c, s);
    double v = 0.0;
    bool first = true;
#pragma unroll 1
    for (int mu = 0; mu < 3; ++mu) {
        const m3 umu = link_at<RESIDENT>(links, c, s, mu);
        const Nb pm = step(c, x.x, x.lex, x.par, mu, +1);
#pragma unroll 1
        for (int nu = mu + 1; nu < 4; ++nu) {
            const Nb pn = step(c, x.x, x.lex, x.par, nu, +1);
            m3 p = mul_fma(umu, link_at<RESIDENT>(links, c, storage_index(c, pm.lex, pm.par), nu));
            p = mul_adj_fma(p, link_at<RESIDENT>(links, c, storage_index(c, pn.lex, pn.par), mu));
            const double val = retrace_mul_adj(p, link_at<RESIDENT>(links, c, s, nu)) / 3.0;
            v = first ? val : v + val;
            first = false;
        }
    }
    return v;
}

}  // namespace ym
