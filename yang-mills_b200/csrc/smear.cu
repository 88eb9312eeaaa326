// smear.cu -- stride-2 spatial blocking of SU(3) lattices (compiled with
// -fmad=false: the product is the reference's arithmetic, bit for bit).
//
// Blocking (glueball_blocking.rs:105-136): V_mu(y) = U_mu(2y) U_mu(2y+mu)
// for spatial mu, V_3(y) = U_3(2y), fine site 2y = (2y0, 2y1, 2y2, y3).
#include <cuda_runtime.h>

#include "su3_checks.cuh"
#include "ym_internal.hpp"

namespace ym {

namespace {

constexpr int T = kSiteThreads;

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

cudaError_t launch_block(ym_ensemble *fine, ym_ensemble *coarse) {
    k_block<<<(unsigned)coarse->n_site_tiles, T, 0, coarse->stream>>>(
        fine->d_chains, coarse->d_chains, coarse->d_site_tiles, fine->d_links, coarse->d_links,
        coarse->d_error);
    return cudaGetLastError();
}

}  // namespace ym
