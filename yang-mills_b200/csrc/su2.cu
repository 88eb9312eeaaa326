// su2.cu -- SU(2) kernels (compiled with -fmad=false): checkerboard
// heat-bath and overrelaxation sub-sweeps, plaquette, unit residual, layout.
//
// Links are unit quaternions (a0, a1, a2, a3), U = a0 I - i a.sigma
// (reference/rust/src/lib.rs:7-13), stored as two double2 planes per
// direction: (a0, a1) and (a2, a3).  Every quaternion product is
// re-normalised exactly as Su2::mul does (lib.rs:106-130, 212-224): divide by
// the largest magnitude, then by the Euclidean norm.
//
// Heat-bath: the reference's sampler (su2_ensemble.rs:220-281) -- r0 from
// the truncated exponential by inverse CDF (exp_m1, ln_1p), the Haar factor
// sqrt(1 - r0^2) by rejection, a uniform direction on S^2, U = R Vhat^dag --
// or, as an alternative, the Kennedy-Pendleton sampler for the same density.
// The attempt loop is bounded; a link that exhausts it keeps its value and
// raises the ensemble's error flag (HeatbathAttemptLimitExceeded).
// Overrelaxation: U <- Vhat^dag U^dag Vhat^dag (su2_ensemble.rs:283-299).
#include <cuda_runtime.h>

#include "su2_quat.cuh"
#include "ym_internal.hpp"

namespace ym {

namespace {

constexpr int T = kSweepThreads;
constexpr double kAlphaZeroLimit = 1.0e-300;   // su2_ensemble.rs:22
constexpr double kTau = 6.283185307179586;     // core::f64::consts::TAU

// Lattice4::staple (lib.rs:507-546): the unnormalised sum of six products,
// nu ascending, forward then backward, components added in order (one
// thread per link).
template <int MU>
__device__ __forceinline__ void su2_staple(const double2 *__restrict__ links, const ChainInfo &c,
                                           const Coord &x, int par, double comp[4]) {
    comp[0] = comp[1] = comp[2] = comp[3] = 0.0;
    const Nb self{x.lex, par};
    const Nb pm = step(c, x.x, x.lex, par, MU, +1);
#pragma unroll
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == MU) continue;
        const Nb pn = step(c, x.x, x.lex, par, nu, +1);
        const Nb mn = step(c, x.x, x.lex, par, nu, -1);
        const Nb mnpm = step(c, x.x, mn.lex, mn.par, MU, +1);
        const q4 fwd = qmul(qmul(link_q(links, c, pm, nu), qdag(link_q(links, c, pn, MU))),
                            qdag(link_q(links, c, self, nu)));
        const q4 bwd = qmul(qmul(qdag(link_q(links, c, mnpm, nu)), qdag(link_q(links, c, mn, MU))),
                            link_q(links, c, mn, nu));
#pragma unroll
        for (int i = 0; i < 4; ++i) comp[i] += fwd.c[i];
#pragma unroll
        for (int i = 0; i < 4; ++i) comp[i] += bwd.c[i];
    }
}

// The same staple for a link updated by a group of kGroup lanes: lane j < 6
// computes term j (the (j/2)-th direction nu != MU, forward for even j,
// backward for odd j) and every lane of the group then adds the six terms in
// that order, so the sum has the one-thread staple's bits while its twelve
// normalised products run on six lanes at once.
constexpr int kGroup = 8;
constexpr int kGroupLinks = T / kGroup;   // links per 128-thread block

__device__ __forceinline__ q4 qdag_if(const q4 &a, bool d) {
    const double s = d ? -1.0 : 1.0;   // exact sign flip
    return q4{{a.c[0], s * a.c[1], s * a.c[2], s * a.c[3]}};
}

// Term j of the staple of link (x, MU):
//   forward  U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag
//   backward U_nu(x-nu+mu)^dag U_mu(x-nu)^dag U_nu(x-nu)
template <int MU>
__device__ __forceinline__ q4 su2_staple_term(const double2 *__restrict__ links, const ChainInfo &c,
                                              const Coord &x, int par, int j) {
    const int k = j >> 1;
    const int nu = k < MU ? k : k + 1;
    const bool fwd = (j & 1) == 0;
    const Nb pm = step(c, x.x, x.lex, par, MU, +1);
    const Nb pn = step_any(c, x.x, x.lex, par, nu, +1);
    const Nb mn = step_any(c, x.x, x.lex, par, nu, -1);
    const Nb mnpm = step(c, x.x, mn.lex, mn.par, MU, +1);   // x - nu keeps x's mu coordinate
    const Nb sa = fwd ? pm : mnpm, sb = fwd ? pn : mn, sc = fwd ? Nb{x.lex, par} : mn;
    const q4 a = qdag_if(link_q(links, c, sa, nu), !fwd);
    const q4 b = qdag(link_q(links, c, sb, MU));
    const q4 cc = qdag_if(link_q(links, c, sc, nu), fwd);
    return qmul(qmul(a, b), cc);
}

// The group's staple sum (every lane of the group gets it): terms computed
// by lanes 0..5 of the group (`active` false: the group's lanes load nothing
// and the sum is meaningless), added in term order.
template <int MU>
__device__ __forceinline__ void su2_staple_group(const double2 *__restrict__ links, const ChainInfo &c,
                                                 const Coord &x, int par, bool active, double comp[4]) {
    const int lane = threadIdx.x & 31, j = lane & (kGroup - 1), base = lane - j;
    q4 term{{0.0, 0.0, 0.0, 0.0}};
    if (active && j < 6) term = su2_staple_term<MU>(links, c, x, par, j);
    comp[0] = comp[1] = comp[2] = comp[3] = 0.0;
#pragma unroll
    for (int jj = 0; jj < 6; ++jj)
#pragma unroll
        for (int i = 0; i < 4; ++i) comp[i] += __shfl_sync(0xffffffffu, term.c[i], base + jj);
}

// staple_norm (su2_ensemble.rs:194-202): sum of squares from -0.0, sqrt.
__device__ __forceinline__ double staple_norm(const double comp[4]) {
    double ss = comp[0] * comp[0];
    ss = ss + comp[1] * comp[1];
    ss = ss + comp[2] * comp[2];
    ss = ss + comp[3] * comp[3];
    return sqrt(ss);
}

// The reference sampler (su2_ensemble.rs:220-254) on the link's stream:
// words 2k, 2k+1 for attempt k+1, then two for the S^2 direction.
__device__ __forceinline__ bool sample_reference(double alpha, uint64_t key, int max_attempts,
                                                 q4 &out, int &attempts) {
    uint64_t j = 0;
    const double mass = alpha <= kAlphaZeroLimit ? 0.0 : -expm1(-2.0 * alpha);
    for (int a = 1; a <= max_attempts; ++a) {
        const double pu = unit_from(splitmix_at(key, j++));
        double r0;
        if (alpha <= kAlphaZeroLimit) {
            r0 = 2.0 * pu - 1.0;
        } else {
            const double y = -log1p(-pu * mass) / alpha;
            r0 = 1.0 - y;
            r0 = r0 < -1.0 ? -1.0 : (r0 > 1.0 ? 1.0 : r0);
        }
        const double radial = sqrt(fmax(1.0 - r0 * r0, 0.0));
        if (unit_from(splitmix_at(key, j++)) <= radial) {
            const double z = 2.0 * unit_from(splitmix_at(key, j++)) - 1.0;
            const double phi = kTau * unit_from(splitmix_at(key, j++));
            const double planar = sqrt(fmax(1.0 - z * z, 0.0));
            const double v[4] = {r0, radial * (planar * cos(phi)), radial * (planar * sin(phi)),
                                 radial * z};
            if (!normalize_scaled<4>(v, out.c)) return false;
            attempts = a;
            return true;
        }
    }
    attempts = max_attempts;
    return false;
}

// Kennedy-Pendleton (Phys. Lett. B 156 (1985) 393) for the same density
// exp(alpha r0) sqrt(1 - r0^2): x = -(ln u1 + cos^2(2 pi u2) ln u3)/alpha,
// accept if u4^2 <= 1 - x/2, r0 = 1 - x.  Uniforms in (0, 1].
__device__ __forceinline__ bool sample_kp(double alpha, uint64_t key, int max_attempts, q4 &out,
                                          int &attempts) {
    uint64_t j = 0;
    if (alpha <= kAlphaZeroLimit) return sample_reference(alpha, key, max_attempts, out, attempts);
    for (int a = 1; a <= max_attempts; ++a) {
        const double u1 = 1.0 - unit_from(splitmix_at(key, j++));
        const double u2 = unit_from(splitmix_at(key, j++));
        const double u3 = 1.0 - unit_from(splitmix_at(key, j++));
        const double u4 = unit_from(splitmix_at(key, j++));
        const double cs = cospi(2.0 * u2);
        const double x = -(log(u1) + cs * cs * log(u3)) / alpha;
        if (u4 * u4 <= 1.0 - 0.5 * x) {
            const double r0 = 1.0 - x;
            const double radial = sqrt(fmax(1.0 - r0 * r0, 0.0));
            const double z = 2.0 * unit_from(splitmix_at(key, j++)) - 1.0;
            double sn, cn;
            sincospi(2.0 * unit_from(splitmix_at(key, j++)), &sn, &cn);
            const double planar = sqrt(fmax(1.0 - z * z, 0.0));
            const double v[4] = {r0, radial * (planar * cn), radial * (planar * sn), radial * z};
            if (!normalize_scaled<4>(v, out.c)) return false;
            attempts = a;
            return true;
        }
    }
    attempts = max_attempts;
    return false;
}

// Error flag bits.
constexpr unsigned kErrAttempts = 1u;
constexpr unsigned kErrNonFinite = 2u;

// One thread per link (large sub-sweeps, throughput-bound).
template <int MU>
__global__ void __launch_bounds__(T)
k_su2_heatbath_thread(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
               double2 *__restrict__ links, int parity, int max_attempts, int kp,
               const uint64_t *__restrict__ sweep_ptr, unsigned long long *__restrict__ proposals,
               unsigned *__restrict__ err) {
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t t = tile.start + threadIdx.x;
    unsigned attempts_used = 0;
    if (t < c.half) {
        const int64_t s = (int64_t)parity * c.half + t;
        const Coord x = decode_storage(c, s);
        double comp[4];
        su2_staple<MU>(links, c, x, parity, comp);
        const double norm = staple_norm(comp);
        const double alpha = c.beta * norm;
        if (!isfinite(norm) || !isfinite(alpha)) {
            atomicOr(err, kErrNonFinite);
        } else {
            const uint64_t key = link_key(c.seed, *sweep_ptr, x.lex, MU);
            q4 r;
            int att = 0;
            const bool ok = kp ? sample_kp(alpha, key, max_attempts, r, att)
                               : sample_reference(alpha, key, max_attempts, r, att);
            attempts_used = (unsigned)att;
            if (!ok) {
                atomicOr(err, kErrAttempts);
            } else {
                q4 next = r;
                if (norm != 0.0) {
                    q4 vhat;
                    normalize_scaled<4>(comp, vhat.c);
                    next = qmul(r, qdag(vhat));
                }
                store_q(links, c, s, MU, next);
            }
        }
    }
    const unsigned warp_sum = __reduce_add_sync(0xffffffffu, attempts_used);
    if ((threadIdx.x & 31) == 0 && warp_sum)
        atomicAdd(proposals + tile.chain, (unsigned long long)warp_sum);
}

template <int MU>
__global__ void __launch_bounds__(T)
k_su2_overrelax_thread(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                double2 *__restrict__ links, int parity, unsigned *__restrict__ err) {
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t t = tile.start + threadIdx.x;
    if (t >= c.half) return;
    const int64_t s = (int64_t)parity * c.half + t;
    const Coord x = decode_storage(c, s);
    double comp[4];
    su2_staple<MU>(links, c, x, parity, comp);
    const double norm = staple_norm(comp);
    if (!isfinite(norm)) {
        atomicOr(err, kErrNonFinite);
        return;
    }
    if (norm == 0.0) return;
    q4 vhat;
    normalize_scaled<4>(comp, vhat.c);
    const q4 nd = qdag(vhat);
    store_q(links, c, s, MU, qmul(qmul(nd, qdag(load_q_rw(links, c, s, MU))), nd));
}

// Grouped form (small sub-sweeps, latency-bound: a 10^4 lattice updates
// 5,000 links per launch, about one warp per SM with one thread per link).
// One block: kGroupLinks links of the tile blockIdx.x / kGroup (sub-block
// blockIdx.x % kGroup), kGroup lanes per link; the update is evaluated by
// every lane of the group alike and written by its first lane.
template <int MU>
__global__ void __launch_bounds__(T)
k_su2_heatbath_group(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
               double2 *__restrict__ links, int parity, int max_attempts, int kp,
               const uint64_t *__restrict__ sweep_ptr, unsigned long long *__restrict__ proposals,
               unsigned *__restrict__ err) {
    const Tile tile = tiles[blockIdx.x / kGroup];
    const ChainInfo c = chains[tile.chain];
    const int64_t t = tile.start + (int64_t)(blockIdx.x % kGroup) * kGroupLinks + threadIdx.x / kGroup;
    const bool leader = (threadIdx.x & (kGroup - 1)) == 0;
    const bool active = t < c.half;
    const int64_t s = (int64_t)parity * c.half + (active ? t : 0);
    const Coord x = decode_storage(c, s);
    double comp[4];
    su2_staple_group<MU>(links, c, x, parity, active, comp);
    unsigned attempts_used = 0;
    if (active) {
        const double norm = staple_norm(comp);
        const double alpha = c.beta * norm;
        if (!isfinite(norm) || !isfinite(alpha)) {
            if (leader) atomicOr(err, kErrNonFinite);
        } else {
            const uint64_t key = link_key(c.seed, *sweep_ptr, x.lex, MU);
            q4 r;
            int att = 0;
            const bool ok = kp ? sample_kp(alpha, key, max_attempts, r, att)
                               : sample_reference(alpha, key, max_attempts, r, att);
            attempts_used = leader ? (unsigned)att : 0u;
            if (!ok) {
                if (leader) atomicOr(err, kErrAttempts);
            } else {
                q4 next = r;
                if (norm != 0.0) {
                    q4 vhat;
                    normalize_scaled<4>(comp, vhat.c);
                    next = qmul(r, qdag(vhat));
                }
                if (leader) store_q(links, c, s, MU, next);
            }
        }
    }
    const unsigned warp_sum = __reduce_add_sync(0xffffffffu, attempts_used);
    if ((threadIdx.x & 31) == 0 && warp_sum)
        atomicAdd(proposals + tile.chain, (unsigned long long)warp_sum);
}

template <int MU>
__global__ void __launch_bounds__(T)
k_su2_overrelax_group(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                double2 *__restrict__ links, int parity, unsigned *__restrict__ err) {
    const Tile tile = tiles[blockIdx.x / kGroup];
    const ChainInfo c = chains[tile.chain];
    const int64_t t = tile.start + (int64_t)(blockIdx.x % kGroup) * kGroupLinks + threadIdx.x / kGroup;
    const bool leader = (threadIdx.x & (kGroup - 1)) == 0;
    const bool active = t < c.half;
    const int64_t s = (int64_t)parity * c.half + (active ? t : 0);
    const Coord x = decode_storage(c, s);
    double comp[4];
    su2_staple_group<MU>(links, c, x, parity, active, comp);
    if (!active) return;
    const double norm = staple_norm(comp);
    if (!isfinite(norm)) {
        if (leader) atomicOr(err, kErrNonFinite);
        return;
    }
    if (norm == 0.0) return;
    q4 vhat;
    normalize_scaled<4>(comp, vhat.c);
    const q4 nd = qdag(vhat);
    const q4 next = qmul(qmul(nd, qdag(load_q_rw(links, c, s, MU))), nd);
    if (leader) store_q(links, c, s, MU, next);
}

// Plaquette half real trace per site, (mu, nu) order as the reference.
__global__ void __launch_bounds__(kSiteThreads)
k_su2_plaquette(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                const double2 *__restrict__ links, double *__restrict__ partial) {
    __shared__ double warp_vals[32];
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t s = tile.start + threadIdx.x;
    double v = 0.0;
    if (s < c.volume) {
        const Coord x = decode_storage(c, s);
        const Nb self{x.lex, x.par};
        bool first = true;
#pragma unroll 1
        for (int mu = 0; mu < 3; ++mu) {
            const Nb pm = step(c, x.x, x.lex, x.par, mu, +1);
#pragma unroll 1
            for (int nu = mu + 1; nu < 4; ++nu) {
                const Nb pn = step(c, x.x, x.lex, x.par, nu, +1);
                q4 p = qmul(link_q(links, c, self, mu), link_q(links, c, pm, nu));
                p = qmul(p, qdag(link_q(links, c, pn, mu)));
                p = qmul(p, qdag(link_q(links, c, self, nu)));
                v = first ? p.c[0] : v + p.c[0];
                first = false;
            }
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) warp_vals[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < (blockDim.x >> 5) ? warp_vals[threadIdx.x] : 0.0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (threadIdx.x == 0) partial[blockIdx.x] = v;
    }
}

// max |norm^2 - 1| per tile (Lattice4::max_link_unit_residual lib.rs:726-740).
__global__ void __launch_bounds__(kSiteThreads)
k_su2_unit_residual(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                    const double2 *__restrict__ links, double *__restrict__ partial) {
    __shared__ double warp_vals[32];
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t s = tile.start + threadIdx.x;
    double r = 0.0;
    if (s < c.volume) {
        for (int mu = 0; mu < 4; ++mu) {
            const q4 q = load_q(links, c, s, mu);
            double n2 = q.c[0] * q.c[0];
            n2 = n2 + q.c[1] * q.c[1];
            n2 = n2 + q.c[2] * q.c[2];
            n2 = n2 + q.c[3] * q.c[3];
            const double res = isfinite(n2) ? fabs(n2 - 1.0) : INFINITY;
            r = isfinite(res) ? fmax(r, res) : INFINITY;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) r = fmax(r, __shfl_down_sync(0xffffffffu, r, off));
    if ((threadIdx.x & 31) == 0) warp_vals[threadIdx.x >> 5] = r;
    __syncthreads();
    if (threadIdx.x < 32) {
        r = threadIdx.x < (blockDim.x >> 5) ? warp_vals[threadIdx.x] : 0.0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) r = fmax(r, __shfl_down_sync(0xffffffffu, r, off));
        if (threadIdx.x == 0) partial[blockIdx.x] = r;
    }
}

// Every chain at once: blockIdx.y picks the chain.
__global__ void k_su2_identity(const ChainInfo *__restrict__ chains, double2 *links) {
    const ChainInfo c = chains[blockIdx.y];
    const int64_t n = 8 * c.volume;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t plane = i / c.volume;
        links[c.offset + i] = make_double2((plane % 2 == 0) ? 1.0 : 0.0, 0.0);
    }
}

__global__ void k_su2_from_aos(const ChainInfo *__restrict__ chains, int chain, double2 *links,
                               const double2 *__restrict__ staging) {
    const ChainInfo c = chains[chain];
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < c.volume;
         s += (int64_t)gridDim.x * blockDim.x) {
        const Coord x = decode_storage(c, s);
        for (int mu = 0; mu < 4; ++mu) {
            const double2 *src = staging + (x.lex * 4 + mu) * 2;
            double2 *dst = links + c.offset + (int64_t)(mu * 2) * c.volume + s;
            dst[0] = src[0];
            dst[c.volume] = src[1];
        }
    }
}

__global__ void k_su2_to_aos(const ChainInfo *__restrict__ chains, int chain,
                             const double2 *__restrict__ links, double2 *staging) {
    const ChainInfo c = chains[chain];
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < c.volume;
         s += (int64_t)gridDim.x * blockDim.x) {
        const Coord x = decode_storage(c, s);
        for (int mu = 0; mu < 4; ++mu) {
            double2 *dst = staging + (x.lex * 4 + mu) * 2;
            const double2 *src = links + c.offset + (int64_t)(mu * 2) * c.volume + s;
            dst[0] = src[0];
            dst[1] = src[c.volume];
        }
    }
}

int grid_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b > 148 * 16) b = 148 * 16;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace

// The grouped kernels give each link kGroup lanes; they win while a
// sub-sweep has too few links to hide the one-thread kernels' latency
// (measured on B200: 5,000 links per launch 15.5 vs 24.5 us heat-bath,
// 32,768 links 35.4 vs 25.2 us, crossover near 17,000), so up to 96 links
// per SM.
static bool su2_grouped(const ym_ensemble *e) {
    static thread_local int sms = 0, dev_seen = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != dev_seen) {
        sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        dev_seen = dev;
    }
    return e->n_half_tiles * (int64_t)T <= (int64_t)sms * 96;
}

cudaError_t launch_su2_heatbath(ym_ensemble *e, int parity, int mu, int max_attempts, int kp) {
    auto *ch = e->d_chains;
    auto *tl = e->d_half_tiles;
    const dim3 b(T);
    if (su2_grouped(e)) {
        const dim3 g((unsigned)(e->n_half_tiles * kGroup));
        switch (mu) {
        case 0: k_su2_heatbath_group<0><<<g, b, 0, e->stream>>>(ch, tl, e->d_links, parity, max_attempts, kp, e->d_sweep, e->d_accepts, e->d_error); break;
        case 1: k_su2_heatbath_group<1><<<g, b, 0, e->stream>>>(ch, tl, e->d_links, parity, max_attempts, kp, e->d_sweep, e->d_accepts, e->d_error); break;
        case 2: k_su2_heatbath_group<2><<<g, b, 0, e->stream>>>(ch, tl, e->d_links, parity, max_attempts, kp, e->d_sweep, e->d_accepts, e->d_error); break;
        default: k_su2_heatbath_group<3><<<g, b, 0, e->stream>>>(ch, tl, e->d_links, parity, max_attempts, kp, e->d_sweep, e->d_accepts, e->d_error); break;
        }
        return cudaGetLastError();
    }
    const dim3 g((unsigned)e->n_half_tiles);
    switch (mu) {
    case 0: k_su2_heatbath_thread<0><<<g, b, 0, e->stream>>>(ch, tl, e->d_links, parity, max_attempts, kp, e->d_sweep, e->d_accepts, e->d_error); break;
    case 1: k_su2_heatbath_thread<1><<<g, b, 0, e->stream>>>(ch, tl, e->d_links, parity, max_attempts, kp, e->d_sweep, e->d_accepts, e->d_error); break;
    case 2: k_su2_heatbath_thread<2><<<g, b, 0, e->stream>>>(ch, tl, e->d_links, parity, max_attempts, kp, e->d_sweep, e->d_accepts, e->d_error); break;
    default: k_su2_heatbath_thread<3><<<g, b, 0, e->stream>>>(ch, tl, e->d_links, parity, max_attempts, kp, e->d_sweep, e->d_accepts, e->d_error); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_su2_overrelax(ym_ensemble *e, int parity, int mu) {
    auto *ch = e->d_chains;
    auto *tl = e->d_half_tiles;
    const dim3 b(T);
    if (su2_grouped(e)) {
        const dim3 g((unsigned)(e->n_half_tiles * kGroup));
        switch (mu) {
        case 0: k_su2_overrelax_group<0><<<g, b, 0, e->stream>>>(ch, tl, e->d_links, parity, e->d_error); break;
        case 1: k_su2_overrelax_group<1><<<g, b, 0, e->stream>>>(ch, tl, e->d_links, parity, e->d_error); break;
        case 2: k_su2_overrelax_group<2><<<g, b, 0, e->stream>>>(ch, tl, e->d_links, parity, e->d_error); break;
        default: k_su2_overrelax_group<3><<<g, b, 0, e->stream>>>(ch, tl, e->d_links, parity, e->d_error); break;
        }
        return cudaGetLastError();
    }
    const dim3 g((unsigned)e->n_half_tiles);
    switch (mu) {
    case 0: k_su2_overrelax_thread<0><<<g, b, 0, e->stream>>>(ch, tl, e->d_links, parity, e->d_error); break;
    case 1: k_su2_overrelax_thread<1><<<g, b, 0, e->stream>>>(ch, tl, e->d_links, parity, e->d_error); break;
    case 2: k_su2_overrelax_thread<2><<<g, b, 0, e->stream>>>(ch, tl, e->d_links, parity, e->d_error); break;
    default: k_su2_overrelax_thread<3><<<g, b, 0, e->stream>>>(ch, tl, e->d_links, parity, e->d_error); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_su2_plaquette_partials(ym_ensemble *e) {
    k_su2_plaquette<<<(unsigned)e->n_site_tiles, kSiteThreads, 0, e->stream>>>(
        e->d_chains, e->d_site_tiles, e->d_links, e->d_partial);
    return cudaGetLastError();
}

cudaError_t launch_su2_unit_residual_partials(ym_ensemble *e) {
    k_su2_unit_residual<<<(unsigned)e->n_site_tiles, kSiteThreads, 0, e->stream>>>(
        e->d_chains, e->d_site_tiles, e->d_links, e->d_partial);
    return cudaGetLastError();
}

cudaError_t launch_su2_identity(ym_ensemble *e) {
    int64_t vmax = 0;
    for (const ChainInfo &c : e->chains) vmax = c.volume > vmax ? c.volume : vmax;
    for (int64_t first = 0; first < e->n_chains; first += 65535) {   // the grid's y limit
        const int64_t count = e->n_chains - first < 65535 ? e->n_chains - first : 65535;
        const int64_t bx = (grid_for(8 * vmax, 256) + count - 1) / count;
        k_su2_identity<<<dim3((unsigned)(bx < 1 ? 1 : bx), (unsigned)count), 256, 0, e->stream>>>(
            e->d_chains + first, e->d_links);
    }
    return cudaGetLastError();
}

cudaError_t launch_su2_from_aos(ym_ensemble *e, int64_t chain) {
    k_su2_from_aos<<<grid_for(e->chains[chain].volume, 128), 128, 0, e->stream>>>(
        e->d_chains, (int)chain, e->d_links, reinterpret_cast<const double2 *>(e->d_staging));
    return cudaGetLastError();
}

cudaError_t launch_su2_to_aos(ym_ensemble *e, int64_t chain) {
    k_su2_to_aos<<<grid_for(e->chains[chain].volume, 128), 128, 0, e->stream>>>(
        e->d_chains, (int)chain, e->d_links, reinterpret_cast<double2 *>(e->d_staging));
    return cudaGetLastError();
}

}  // namespace ym
