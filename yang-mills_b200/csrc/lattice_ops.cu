// lattice_ops.cu -- per-site and per-link lattice queries of the reference's
// Su3Lattice4 / Lattice4 / path_holonomy API on device-resident chains
// (compiled with -fmad=false: every product below is the reference's, in
// its order, with no fused multiply-add).
//
//   path_holonomy / wilson_loop (path_holonomy.rs:132-181, lib.rs:384-436)
//       every start site of a chain in one launch, or one start;
//   polyakov_loop (su3_lattice.rs:185-212, lib.rs:483-505) per start site;
//   plaquette(x, mu, nu) (su3_lattice.rs:168-181, lib.rs:348-361);
//   wilson_action(beta) (su3_lattice.rs:214-242, lib.rs:363-382): per-site
//       plaquette terms in parallel, then one warp per chain sums them in
//       the reference's sequential order, so the action is bit for bit;
//   gauge_transform (su3_lattice.rs:244-283) with per-site gauges;
//   local_link_action / local_action_difference (su3_ensemble.rs:261-334);
//   SU(2) staple (lib.rs:507-546);
//   link / set_link (su3_lattice.rs:153-166) moving one link.
//
// SU(3) products are the reference's checked ones (Su3::mul, su3.rs:286-288
// and 242-253): after each product the result must be finite, unitary and of
// determinant one within 5e-12; a failure sets an error bit that the host
// turns into the reference's Su3Error variant.  SU(2) products re-normalise
// as Su2::mul does.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "su2_quat.cuh"
#include "su3_checks.cuh"
#include "ym_internal.hpp"

namespace ym {

namespace {

constexpr int kThreads = 128;
constexpr int64_t kMaxPathSteps = int64_t(1) << 20;   // MAX_PATH_STEPS path_holonomy.rs:17, lib.rs:22
constexpr double kMaxSu3Beta = 12.0;                   // MAX_REFERENCE_BETA su3_ensemble.rs:24

// Error bits of a query launch.
constexpr unsigned kQNonFiniteMatrix = 1u;
constexpr unsigned kQNonUnitary = 2u;
constexpr unsigned kQDeterminant = 4u;
constexpr unsigned kQNonFiniteStatistic = 8u;
constexpr unsigned kQNonFiniteAction = 16u;

// Su3::from_checked_matrix (su3.rs:242-253) as an error bit, in the
// reference's order of checks.
__device__ __forceinline__ unsigned su3_gate(const m3 &u) {
    if (!finite3(u)) return kQNonFiniteMatrix;
    if (unitarity_res2(u) > kSu3Tol * kSu3Tol) return kQNonUnitary;
    if (norm2(csub(det3(u), cmake(1.0, 0.0))) > kSu3Tol * kSu3Tol) return kQDeterminant;
    return 0u;
}

// Checked product a*b; the first failure of a thread is kept in *bits.
__device__ __forceinline__ m3 mul_checked(const m3 &a, const m3 &b, unsigned &bits) {
    const m3 p = mul(a, b);
    if (!bits) bits = su3_gate(p);
    return p;
}

__device__ __forceinline__ int32_t xget(const int32_t x[4], int d) { return coord_of(x, d); }

__device__ __forceinline__ void xset(int32_t x[4], int d, int32_t v) {
    if (d == 0) x[0] = v;
    else if (d == 1) x[1] = v;
    else if (d == 2) x[2] = v;
    else x[3] = v;
}

__device__ __forceinline__ int64_t lex_of(const ChainInfo &c, const int32_t x[4]) {
    return (((int64_t)x[0] * c.n[1] + x[1]) * c.n[2] + x[2]) * c.n[3] + x[3];
}

// Storage slot of site x (checkerboard or lexicographic order).
__device__ __forceinline__ int64_t slot_of(const ChainInfo &c, const int32_t x[4]) {
    return storage_index(c, lex_of(c, x), (x[0] + x[1] + x[2] + x[3]) & 1);
}

__device__ __forceinline__ void lex_decode(const ChainInfo &c, int64_t lex, int32_t x[4]) {
    x[3] = (int32_t)(lex % c.n[3]);
    int64_t r = lex / c.n[3];
    x[2] = (int32_t)(r % c.n[2]);
    r /= c.n[2];
    x[1] = (int32_t)(r % c.n[1]);
    x[0] = (int32_t)(r / c.n[1]);
}

// neighbor_plus / neighbor_minus (periodic) along d, in place.
__device__ __forceinline__ void move(const ChainInfo &c, int32_t x[4], int d, int dir) {
    const int32_t v = xget(x, d), n = coord_of(c.n, d);
    xset(x, d, dir > 0 ? (v + 1 == n ? 0 : v + 1) : (v == 0 ? n - 1 : v - 1));
}

__device__ __forceinline__ m3 su3_at(const double2 *links, const ChainInfo &c, const int32_t x[4], int mu) {
    return load_su3(links, c, slot_of(c, x), mu);
}

__device__ __forceinline__ q4 su2_at(const double2 *links, const ChainInfo &c, const int32_t x[4], int mu) {
    return load_q(links, c, slot_of(c, x), mu);
}

__device__ __forceinline__ m3 m3_from(const double *p) {
    m3 o;
#pragma unroll
    for (int e = 0; e < 9; ++e) o.e[e / 3][e % 3] = cmake(p[2 * e], p[2 * e + 1]);
    return o;
}

__device__ __forceinline__ void m3_to(const m3 &u, double *p) {
#pragma unroll
    for (int e = 0; e < 9; ++e) {
        p[2 * e] = u.e[e / 3][e % 3].re;
        p[2 * e + 1] = u.e[e / 3][e % 3].im;
    }
}

// ---------------------------------------------------------------- paths

// The closed or open path `steps` (+(d+1) forward along d, -(d+1) backward)
// from each start site lex = first + i, i < count: holonomy = 1, then
// holonomy = holonomy * segment for every step, a forward step taking the
// link at the current site, a backward step the dagger of the link at the
// site it moves to (path_holonomy.rs:132-161, lib.rs:384-414).  out[i]
// receives (1/3) Tr (SU(3), Complex64::scale(1/3), path_holonomy.rs:172-181)
// or ((1/2) Re Tr, 0) (SU(2)); hol (optional) the first start's holonomy.
template <int GROUP>
__global__ void __launch_bounds__(kThreads)
k_path_sites(const ChainInfo *__restrict__ chains, int chain, const double2 *__restrict__ links,
             const int32_t *__restrict__ steps, int64_t n_steps, int64_t first, int64_t count,
             double2 *__restrict__ out, double *__restrict__ hol, unsigned *__restrict__ err) {
    const int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (i >= count) return;
    const ChainInfo c = chains[chain];
    int32_t x[4];
    lex_decode(c, first + i, x);
    unsigned bits = 0;
    if (GROUP == 3) {
        m3 h = identity3();
#pragma unroll 1
        for (int64_t k = 0; k < n_steps; ++k) {
            const int32_t st = __ldg(steps + k);
            const int d = st > 0 ? st - 1 : -st - 1;
            m3 seg;
            if (st > 0) {
                seg = su3_at(links, c, x, d);
                move(c, x, d, +1);
            } else {
                move(c, x, d, -1);
                seg = adj(su3_at(links, c, x, d));
            }
            h = mul_checked(h, seg, bits);
        }
        const cplx t = trace3(h);
        const double third = 1.0 / 3.0;
        out[i] = make_double2(t.re * third, t.im * third);
        if (hol && i == 0) m3_to(h, hol);
    } else {
        q4 h{{1.0, 0.0, 0.0, 0.0}};
#pragma unroll 1
        for (int64_t k = 0; k < n_steps; ++k) {
            const int32_t st = __ldg(steps + k);
            const int d = st > 0 ? st - 1 : -st - 1;
            q4 seg;
            if (st > 0) {
                seg = su2_at(links, c, x, d);
                move(c, x, d, +1);
            } else {
                move(c, x, d, -1);
                seg = qdag(su2_at(links, c, x, d));
            }
            h = qmul(h, seg);
        }
        out[i] = make_double2(h.c[0], 0.0);
        if (hol && i == 0)
            for (int k = 0; k < 4; ++k) hol[k] = h.c[k];
    }
    if (bits) atomicOr(err, bits);
}

// ---------------------------------------------------------------- action

// Plaquette of site x in plane (mu, nu), the reference's product order:
// U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag, each product checked.
__device__ __forceinline__ m3 su3_plaquette_at(const double2 *links, const ChainInfo &c,
                                               const int32_t x[4], int mu, int nu, unsigned &bits) {
    int32_t xm[4] = {x[0], x[1], x[2], x[3]}, xn[4] = {x[0], x[1], x[2], x[3]};
    move(c, xm, mu, +1);
    move(c, xn, nu, +1);
    m3 p = mul_checked(su3_at(links, c, x, mu), su3_at(links, c, xm, nu), bits);
    p = mul_checked(p, adj(su3_at(links, c, xn, mu)), bits);
    return mul_checked(p, adj(su3_at(links, c, x, nu)), bits);
}

__device__ __forceinline__ q4 su2_plaquette_at(const double2 *links, const ChainInfo &c,
                                               const int32_t x[4], int mu, int nu) {
    int32_t xm[4] = {x[0], x[1], x[2], x[3]}, xn[4] = {x[0], x[1], x[2], x[3]};
    move(c, xm, mu, +1);
    move(c, xn, nu, +1);
    q4 p = qmul(su2_at(links, c, x, mu), su2_at(links, c, xm, nu));
    p = qmul(p, qdag(su2_at(links, c, xn, mu)));
    return qmul(p, qdag(su2_at(links, c, x, nu)));
}

// terms[lex * 6 + plane] = 1 - (1/3) Re Tr P (SU(3), normalized_real_trace
// su3_lattice.rs:80-82) or 1 - (1/2) Re Tr P (SU(2)) for every site of a
// chain, planes (0,1),(0,2),(0,3),(1,2),(1,3),(2,3).
template <int GROUP>
__global__ void __launch_bounds__(kThreads)
k_action_terms(const ChainInfo *__restrict__ chains, int chain, const double2 *__restrict__ links,
               double *__restrict__ terms, unsigned *__restrict__ err) {
    const ChainInfo c = chains[chain];
    const int64_t lex = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (lex >= c.volume) return;
    int32_t x[4];
    lex_decode(c, lex, x);
    unsigned bits = 0;
    int plane = 0;
#pragma unroll 1
    for (int mu = 0; mu < 4; ++mu)
#pragma unroll 1
        for (int nu = mu + 1; nu < 4; ++nu, ++plane) {
            double v;
            if (GROUP == 3) {
                const m3 p = su3_plaquette_at(links, c, x, mu, nu, bits);
                v = 1.0 - trace3(p).re / 3.0;
            } else {
                v = 1.0 - su2_plaquette_at(links, c, x, mu, nu).c[0];
            }
            terms[lex * 6 + plane] = v;
        }
    if (bits) atomicOr(err, bits);
}

// sum = 0; sum += terms[k] for k = 0..n-1 in order (the reference's
// sequential sum), then out = beta * sum.  One warp per chain: the lanes
// load 32 consecutive terms and every lane adds them in order through
// shuffles, so the result is the sequential sum's bits.
__global__ void k_sequential_action(const double *__restrict__ terms, int64_t n, double beta,
                                    double *__restrict__ out) {
    const int lane = threadIdx.x & 31;
    double sum = 0.0;
    double next = lane < n ? terms[lane] : 0.0;
    for (int64_t base = 0; base < n; base += 32) {
        const double cur = next;
        const int64_t k = base + 32 + lane;
        next = k < n ? terms[k] : 0.0;
        const int64_t m = n - base < 32 ? n - base : 32;
        for (int j = 0; j < 32; ++j) {
            const double t = __shfl_sync(0xffffffffu, cur, j);
            if (j < m) sum = sum + t;
        }
    }
    if (lane == 0) {
        out[0] = sum;
        out[1] = beta * sum;
    }
}

// ---------------------------------------------------------------- gauge

// dst link (x, mu) = g(x) U_mu(x) g(x+mu)^dag, both products checked
// (su3_lattice.rs:262-271); gauges[lex] are 9 double2 (row-major).
__global__ void __launch_bounds__(kThreads)
k_gauge_transform(const ChainInfo *__restrict__ src_chains, int src_chain,
                  const double2 *__restrict__ src, const ChainInfo *__restrict__ dst_chains,
                  int dst_chain, double2 *__restrict__ dst, const double2 *__restrict__ gauges,
                  unsigned *__restrict__ err) {
    const ChainInfo c = src_chains[src_chain];
    const ChainInfo d = dst_chains[dst_chain];
    const int64_t lex = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (lex >= c.volume) return;
    int32_t x[4];
    lex_decode(c, lex, x);
    const int64_t s = slot_of(c, x);
    m3 gx;
#pragma unroll
    for (int e = 0; e < 9; ++e) {
        const double2 v = gauges[lex * 9 + e];
        gx.e[e / 3][e % 3] = cmake(v.x, v.y);
    }
    unsigned bits = 0;
    m3 out[4];
#pragma unroll 1
    for (int mu = 0; mu < 4; ++mu) {
        int32_t xp[4] = {x[0], x[1], x[2], x[3]};
        move(c, xp, mu, +1);
        const int64_t lp = lex_of(c, xp);
        m3 gxp;
#pragma unroll
        for (int e = 0; e < 9; ++e) {
            const double2 v = gauges[lp * 9 + e];
            gxp.e[e / 3][e % 3] = cmake(v.x, v.y);
        }
        const m3 v = mul_checked(gx, load_su3_rw(src, c, s, mu), bits);
        out[mu] = mul_checked(v, adj(gxp), bits);
    }
    // every link is read before any is written (src may be dst)
#pragma unroll 1
    for (int mu = 0; mu < 4; ++mu) store_su3(dst, d, s, mu, out[mu]);
    if (bits) atomicOr(err, bits);
}

// ---------------------------------------------------------------- one link

// local_link_action_with_value (su3_ensemble.rs:261-309) for link (x, mu)
// with the value `val`: for each nu != mu the forward plaquette
// val U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag and the backward one
// U_mu(x-nu) U_nu(x-nu+mu) val^dag U_nu(x-nu)^dag, sum += 1 - ntr each.
__device__ double su3_local_action(const double2 *links, const ChainInfo &c, const int32_t x[4],
                                   int mu, const m3 &val, double beta, unsigned &bits) {
    double sum = 0.0;
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == mu) continue;
        int32_t xm[4] = {x[0], x[1], x[2], x[3]}, xn[4] = {x[0], x[1], x[2], x[3]};
        move(c, xm, mu, +1);
        move(c, xn, nu, +1);
        m3 f = mul_checked(val, su3_at(links, c, xm, nu), bits);
        f = mul_checked(f, adj(su3_at(links, c, xn, mu)), bits);
        f = mul_checked(f, adj(su3_at(links, c, x, nu)), bits);
        int32_t bx[4] = {x[0], x[1], x[2], x[3]};
        move(c, bx, nu, -1);
        int32_t bxm[4] = {bx[0], bx[1], bx[2], bx[3]};
        move(c, bxm, mu, +1);
        m3 b = mul_checked(su3_at(links, c, bx, mu), su3_at(links, c, bxm, nu), bits);
        b = mul_checked(b, adj(val), bits);
        b = mul_checked(b, adj(su3_at(links, c, bx, nu)), bits);
        if (bits) return 0.0;
        sum += 1.0 - trace3(f).re / 3.0;
        sum += 1.0 - trace3(b).re / 3.0;
        if (!isfinite(sum)) {
            bits = kQNonFiniteStatistic;
            return 0.0;
        }
    }
    const double action = beta * sum;
    if (!isfinite(action)) bits = kQNonFiniteStatistic;
    return action;
}

// mode 0: out[0] = local_link_action; mode 1: out[0] =
// local_action_difference with the candidate cand (18 doubles).
__global__ void k_local_action(const ChainInfo *__restrict__ chains, int chain,
                               const double2 *__restrict__ links, int x0, int x1, int x2, int x3,
                               int mu, const double *__restrict__ cand, double beta, int mode,
                               double *__restrict__ out, unsigned *__restrict__ err) {
    const ChainInfo c = chains[chain];
    const int32_t x[4] = {x0, x1, x2, x3};
    unsigned bits = 0;
    const m3 old = su3_at(links, c, x, mu);
    const double a_old = su3_local_action(links, c, x, mu, old, beta, bits);
    double result = a_old;
    if (!bits && mode == 1) {
        const double a_new = su3_local_action(links, c, x, mu, m3_from(cand), beta, bits);
        const double diff = a_new - a_old;
        if (!bits && !isfinite(diff)) bits = kQNonFiniteStatistic;
        result = diff;
    }
    out[0] = result;
    if (bits) atomicOr(err, bits);
}

// SU(3) plaquette matrix (18 doubles) or SU(2) plaquette quaternion (4).
template <int GROUP>
__global__ void k_plaquette_at(const ChainInfo *__restrict__ chains, int chain,
                               const double2 *__restrict__ links, int x0, int x1, int x2, int x3,
                               int mu, int nu, double *__restrict__ out, unsigned *__restrict__ err) {
    const ChainInfo c = chains[chain];
    const int32_t x[4] = {x0, x1, x2, x3};
    if (GROUP == 3) {
        unsigned bits = 0;
        m3_to(su3_plaquette_at(links, c, x, mu, nu, bits), out);
        if (bits) atomicOr(err, bits);
    } else {
        const q4 p = su2_plaquette_at(links, c, x, mu, nu);
        for (int k = 0; k < 4; ++k) out[k] = p.c[k];
    }
}

// Lattice4::staple (lib.rs:507-546): for nu != mu ascending, the forward
// term U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag and the backward term
// U_nu(x-nu+mu)^dag U_mu(x-nu)^dag U_nu(x-nu), components added in order.
__global__ void k_su2_staple_at(const ChainInfo *__restrict__ chains, int chain,
                                const double2 *__restrict__ links, int x0, int x1, int x2, int x3,
                                int mu, double *__restrict__ out) {
    const ChainInfo c = chains[chain];
    const int32_t x[4] = {x0, x1, x2, x3};
    double comp[4] = {0.0, 0.0, 0.0, 0.0};
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == mu) continue;
        int32_t xpm[4] = {x[0], x[1], x[2], x[3]}, xpn[4] = {x[0], x[1], x[2], x[3]};
        move(c, xpm, mu, +1);
        move(c, xpn, nu, +1);
        const q4 fwd = qmul(qmul(su2_at(links, c, xpm, nu), qdag(su2_at(links, c, xpn, mu))),
                            qdag(su2_at(links, c, x, nu)));
        int32_t xmn[4] = {x[0], x[1], x[2], x[3]};
        move(c, xmn, nu, -1);
        int32_t xmnpm[4] = {xmn[0], xmn[1], xmn[2], xmn[3]};
        move(c, xmnpm, mu, +1);
        const q4 bwd = qmul(qmul(qdag(su2_at(links, c, xmnpm, nu)), qdag(su2_at(links, c, xmn, mu))),
                            su2_at(links, c, xmn, nu));
        for (int i = 0; i < 4; ++i) comp[i] += fwd.c[i];
        for (int i = 0; i < 4; ++i) comp[i] += bwd.c[i];
    }
    for (int i = 0; i < 4; ++i) out[i] = comp[i];
}

// One link (binary64 storage) to / from a small buffer: SU(3) 9 double2,
// SU(2) 2 double2 (its quaternion).
__global__ void k_link_get(const ChainInfo *__restrict__ chains, int chain, const double2 *links,
                           int64_t s, int mu, int entries, double2 *out) {
    const ChainInfo c = chains[chain];
    const int e = threadIdx.x;
    if (e < entries) out[e] = links[c.offset + (int64_t)(mu * entries + e) * c.volume + s];
}

__global__ void k_link_set(const ChainInfo *__restrict__ chains, int chain, double2 *links,
                           int64_t s, int mu, int entries, const double2 *in) {
    const ChainInfo c = chains[chain];
    const int e = threadIdx.x;
    if (e < entries) links[c.offset + (int64_t)(mu * entries + e) * c.volume + s] = in[e];
}

unsigned grid_of(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// ------------------------------------------------ SU(2) lattice averages

__device__ __forceinline__ double block_sum_q(double v, double *red) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double a = red[0];
    for (int w = 1; w < kThreads / 32; ++w) a += red[w];
    __syncthreads();
    return a;
}

// Lattice4::rectangular_wilson_loop (lib.rs:471-481) from every site of a
// tile, plane (mu, nu) = blockIdx.y in the order (0,1),(0,2),(0,3),(1,2),
// (1,3),(2,3), every R <= rmax along mu and T <= tmax along nu: the
// reference's single left-to-right product of the 2(R+T) steps of
// rectangular_path (lib.rs:438-469), re-normalised after every product,
// half real trace.  partial[(tile * 6 + plane) * 16 + (R-1)*4 + (T-1)] =
// tile sum (fixed order).
__global__ void __launch_bounds__(kThreads)
k_su2_wilson_tiles(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                   const double2 *__restrict__ links, int rmax, int tmax, double *__restrict__ partial) {
    __shared__ double red[kThreads / 32];
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int plane = blockIdx.y;
    const int mu = plane < 3 ? 0 : (plane < 5 ? 1 : 2);
    const int nu = plane < 3 ? plane + 1 : (plane < 5 ? plane - 1 : 3);
    const int64_t s = tile.start + threadIdx.x;
    const bool live = s < c.volume;
    int32_t x0[4] = {0, 0, 0, 0};
    if (live) {
        const Coord k = decode_storage(c, s);
        for (int d = 0; d < 4; ++d) x0[d] = k.x[d];
    }
    for (int r = 1; r <= 4; ++r)
        for (int t = 1; t <= 4; ++t) {
            double v = 0.0;
            if (live && r <= rmax && t <= tmax) {
                int32_t x[4] = {x0[0], x0[1], x0[2], x0[3]};
                q4 h{{1.0, 0.0, 0.0, 0.0}};
                for (int i = 0; i < r; ++i) {
                    h = qmul(h, su2_at(links, c, x, mu));
                    move(c, x, mu, +1);
                }
                for (int i = 0; i < t; ++i) {
                    h = qmul(h, su2_at(links, c, x, nu));
                    move(c, x, nu, +1);
                }
                for (int i = 0; i < r; ++i) {
                    move(c, x, mu, -1);
                    h = qmul(h, qdag(su2_at(links, c, x, mu)));
                }
                for (int i = 0; i < t; ++i) {
                    move(c, x, nu, -1);
                    h = qmul(h, qdag(su2_at(links, c, x, nu)));
                }
                v = h.c[0];
            }
            const double sum = block_sum_q(v, red);
            if (threadIdx.x == 0)
                partial[((int64_t)blockIdx.x * 6 + plane) * 16 + (r - 1) * 4 + (t - 1)] = sum;
        }
}

// Lattice4::polyakov_loop (lib.rs:483-505) along dir from every site with
// x_dir = 0 (line l = the l-th such site in lexicographic order of the other
// coordinates, taken by the chain's first site tiles): the ordered product
// of the n_dir links, half real trace.  partial[tile*2] = tile sum,
// partial[tile*2 + 1] = 0 (no imaginary part).
__global__ void __launch_bounds__(kThreads)
k_su2_polyakov_tiles(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
                     const double2 *__restrict__ links, int dir, double *__restrict__ partial) {
    __shared__ double red[kThreads / 32];
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t line = tile.start + threadIdx.x;
    double v = 0.0;
    if (line < c.volume / coord_of(c.n, dir)) {
        int32_t x[4];
        int64_t q = line;
        for (int d = 3; d >= 0; --d) {
            if (d == dir) {
                xset(x, d, 0);
            } else {
                xset(x, d, (int32_t)(q % coord_of(c.n, d)));
                q /= coord_of(c.n, d);
            }
        }
        q4 h{{1.0, 0.0, 0.0, 0.0}};
        for (int k = 0; k < coord_of(c.n, dir); ++k) {
            h = qmul(h, su2_at(links, c, x, dir));
            move(c, x, dir, +1);
        }
        v = h.c[0];
    }
    const double sum = block_sum_q(v, red);
    if (threadIdx.x == 0) {
        partial[(int64_t)blockIdx.x * 2] = sum;
        partial[(int64_t)blockIdx.x * 2 + 1] = 0.0;
    }
}

}  // namespace

cudaError_t launch_su2_wilson_loops(ym_ensemble *e, int rmax, int tmax, double *d_partial, double *d_out) {
    k_su2_wilson_tiles<<<dim3((unsigned)e->n_site_tiles, 6), kThreads, 0, e->stream>>>(
        e->d_chains, e->d_site_tiles, e->d_links, rmax, tmax, d_partial);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    return launch_tile_mean(e, d_partial, 96, -1, d_out);
}

cudaError_t launch_su2_polyakov(ym_ensemble *e, int dir, double *d_partial, double *d_out) {
    k_su2_polyakov_tiles<<<(unsigned)e->n_site_tiles, kThreads, 0, e->stream>>>(
        e->d_chains, e->d_site_tiles, e->d_links, dir, d_partial);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    return launch_tile_mean(e, d_partial, 2, dir, d_out);
}

}  // namespace ym

// ======================================================================= host

using ym::ChainInfo;

namespace {

constexpr int64_t kQueryDoubles = 64;

cudaError_t ensure_query(ym_ensemble *e) {
    cudaError_t err = cudaSuccess;
    if (!e->d_query_error) err = ym::dev_alloc(reinterpret_cast<void **>(&e->d_query_error), 16);
    if (err == cudaSuccess && !e->d_query)
        err = ym::dev_alloc(reinterpret_cast<void **>(&e->d_query), kQueryDoubles * sizeof(double));
    if (err == cudaSuccess) err = cudaMemsetAsync(e->d_query_error, 0, sizeof(unsigned), e->stream);
    return err;
}

cudaError_t ensure_steps(ym_ensemble *e, int64_t n) {
    if (e->steps_capacity >= n) return cudaSuccess;
    if (e->d_steps) ym::dev_free(e->d_steps);
    e->d_steps = nullptr;
    e->steps_capacity = 0;
    cudaError_t err = ym::dev_alloc(reinterpret_cast<void **>(&e->d_steps), (size_t)n * sizeof(int32_t));
    if (err == cudaSuccess) e->steps_capacity = n;
    return err;
}

cudaError_t ensure_terms(ym_ensemble *e, int64_t n) {
    if (e->terms_capacity >= n) return cudaSuccess;
    if (e->d_terms) ym::dev_free(e->d_terms);
    e->d_terms = nullptr;
    e->terms_capacity = 0;
    cudaError_t err = ym::dev_alloc(reinterpret_cast<void **>(&e->d_terms), (size_t)n * sizeof(double));
    if (err == cudaSuccess) e->terms_capacity = n;
    return err;
}

#define YM_Q(call)                                                   \
    do {                                                             \
        cudaError_t err__ = (call);                                  \
        if (err__ != cudaSuccess) return ym::record_cuda_status(err__); \
    } while (0)

// Reads and clears the query error bits; maps them onto the reference's
// variants (Su3Error for group gates, the statistic / action variants).
int32_t take_query_error(ym_ensemble *e, int32_t action_status) {
    unsigned bits = 0;
    YM_Q(cudaMemcpyAsync(&bits, e->d_query_error, sizeof bits, cudaMemcpyDeviceToHost, e->stream));
    YM_Q(cudaStreamSynchronize(e->stream));
    if (!bits) return YM_OK;
    if (bits & ym::kQNonFiniteMatrix) return YM_ERR_NON_FINITE_MATRIX;
    if (bits & ym::kQNonUnitary) return YM_ERR_NON_UNITARY_MATRIX;
    if (bits & ym::kQDeterminant) return YM_ERR_DETERMINANT_NOT_ONE;
    if (bits & ym::kQNonFiniteAction) return action_status;
    return YM_ERR_NON_FINITE_STATISTIC;
}

int32_t open_chain(ym_ensemble *e, int64_t chain) {
    if (chain < 0 || chain >= e->n_chains) return YM_ERR_INVALID_ARGUMENT;
    return ym::record_cuda_status(cudaSetDevice(e->device));
}

// Queries read full binary64 links.
int32_t require_f64(const ym_ensemble *e) {
    return e->precision == YM_PREC_F64 ? YM_OK : YM_ERR_UNSUPPORTED_PRECISION;
}

bool coord_ok(const ChainInfo &c, const int64_t *x) {
    for (int d = 0; d < 4; ++d)
        if (x[d] < 0 || x[d] >= c.n[d]) return false;
    return true;
}

int64_t lex_host(const ChainInfo &c, const int64_t *x) {
    return ((x[0] * c.n[1] + x[1]) * c.n[2] + x[2]) * c.n[3] + x[3];
}

int64_t slot_host(const ChainInfo &c, const int64_t *x) {
    const int64_t lex = lex_host(c, x);
    const int par = (int)((x[0] + x[1] + x[2] + x[3]) & 1);
    return c.eo ? (int64_t)par * c.half + (lex >> 1) : lex;
}

// validate_steps (path_holonomy.rs:86-99): empty, too long, then any
// direction out of range.
int32_t validate_steps(const int32_t *steps, int64_t n) {
    if (n <= 0) return YM_ERR_EMPTY_PATH;
    if (n > ym::kMaxPathSteps) return YM_ERR_PATH_TOO_LONG;
    if (!steps) return YM_ERR_NULL_ARGUMENT;
    for (int64_t i = 0; i < n; ++i)
        if (steps[i] == 0 || steps[i] > 4 || steps[i] < -4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
    return YM_OK;
}

// Net displacement of a path on the chain's periodic lattice: every start
// site ends at start + disp (mod extents).
void path_displacement(const ChainInfo &c, const int32_t *steps, int64_t n, int64_t disp[4]) {
    for (int d = 0; d < 4; ++d) disp[d] = 0;
    for (int64_t i = 0; i < n; ++i) {
        const int d = steps[i] > 0 ? steps[i] - 1 : -steps[i] - 1;
        disp[d] += steps[i] > 0 ? 1 : -1;
    }
    for (int d = 0; d < 4; ++d) disp[d] = ((disp[d] % c.n[d]) + c.n[d]) % c.n[d];
}

// Runs the path kernel over [first, first + count) of one chain.
int32_t run_path(ym_ensemble *e, int64_t chain, const int32_t *steps, int64_t n_steps,
                 int64_t first, int64_t count, double *out2, double *hol) {
    const ChainInfo &c = e->chains[chain];
    YM_Q(ensure_query(e));
    YM_Q(ensure_steps(e, n_steps));
    YM_Q(cudaMemcpyAsync(e->d_steps, steps, (size_t)n_steps * sizeof(int32_t), cudaMemcpyHostToDevice,
                         e->stream));
    double2 *d_out = nullptr;
    const bool big = count > 16;
    if (big) {
        YM_Q(cudaMallocAsync(reinterpret_cast<void **>(&d_out), (size_t)count * sizeof(double2), e->stream));
    } else {
        d_out = reinterpret_cast<double2 *>(e->d_query);
    }
    double *d_hol = hol ? e->d_query + 40 : nullptr;
    if (e->group == YM_GROUP_SU3)
        ym::k_path_sites<3><<<ym::grid_of(count), ym::kThreads, 0, e->stream>>>(
            e->d_chains, (int)chain, e->d_links, e->d_steps, n_steps, first, count, d_out, d_hol,
            e->d_query_error);
    else
        ym::k_path_sites<2><<<ym::grid_of(count), ym::kThreads, 0, e->stream>>>(
            e->d_chains, (int)chain, e->d_links, e->d_steps, n_steps, first, count, d_out, d_hol,
            e->d_query_error);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(out2, d_out, (size_t)count * sizeof(double2), cudaMemcpyDeviceToHost, e->stream);
    if (err == cudaSuccess && hol)
        err = cudaMemcpyAsync(hol, d_hol, (e->group == YM_GROUP_SU3 ? 18 : 4) * sizeof(double),
                              cudaMemcpyDeviceToHost, e->stream);
    if (big) {
        const cudaError_t f = cudaFreeAsync(d_out, e->stream);
        if (err == cudaSuccess) err = f;
    }
    if (err != cudaSuccess) return ym::record_cuda_status(err);
    (void)c;
    return take_query_error(e, YM_ERR_NON_FINITE_ACTION);
}

int32_t copy_small(ym_ensemble *e, double *host, int64_t n) {
    YM_Q(cudaMemcpyAsync(host, e->d_query, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    YM_Q(cudaStreamSynchronize(e->stream));
    return YM_OK;
}

}  // namespace

extern "C" {

int32_t ym_rectangular_path(int32_t mu, int32_t nu, int64_t r, int64_t t, int32_t *steps,
                            int64_t capacity, int64_t *n_steps) {
    if (!steps || !n_steps) return YM_ERR_NULL_ARGUMENT;
    if (mu < 0 || mu >= 4 || nu < 0 || nu >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
    if (mu == nu) return YM_ERR_DIRECTIONS_MUST_DIFFER;
    if (r <= 0 || t <= 0) return YM_ERR_ZERO_RECTANGLE_EXTENT;
    if (r > ym::kMaxPathSteps || t > ym::kMaxPathSteps || 2 * (r + t) > ym::kMaxPathSteps)
        return YM_ERR_PATH_TOO_LONG;
    const int64_t per = 2 * (r + t);
    if (per > capacity) return YM_ERR_INVALID_ARGUMENT;
    int64_t k = 0;
    for (int64_t i = 0; i < r; ++i) steps[k++] = mu + 1;
    for (int64_t i = 0; i < t; ++i) steps[k++] = nu + 1;
    for (int64_t i = 0; i < r; ++i) steps[k++] = -(mu + 1);
    for (int64_t i = 0; i < t; ++i) steps[k++] = -(nu + 1);
    *n_steps = per;
    return YM_OK;
}

int32_t ym_path_holonomy(ym_ensemble *e, int64_t chain, const int64_t *start, const int32_t *steps,
                         int64_t n_steps, double *holonomy, int64_t *end) {
    if (!e || !start || !holonomy) return YM_ERR_NULL_ARGUMENT;
    int32_t st = open_chain(e, chain);
    if (st) return st;
    if ((st = require_f64(e))) return st;
    const ChainInfo &c = e->chains[chain];
    if (e->group == YM_GROUP_SU3) {      // path_holonomy.rs:132-135: steps, then start
        if ((st = validate_steps(steps, n_steps))) return st;
        if (!coord_ok(c, start)) return YM_ERR_COORDINATE_OUT_OF_RANGE;
    } else {                              // lib.rs:389-395: start, then steps
        if (!coord_ok(c, start)) return YM_ERR_COORDINATE_OUT_OF_RANGE;
        if ((st = validate_steps(steps, n_steps))) return st;
    }
    double out2[2];
    st = run_path(e, chain, steps, n_steps, lex_host(c, start), 1, out2, holonomy);
    if (st) return st;
    if (end) {
        int64_t disp[4];
        path_displacement(c, steps, n_steps, disp);
        for (int d = 0; d < 4; ++d) end[d] = (start[d] + disp[d]) % c.n[d];
    }
    return YM_OK;
}

int32_t ym_wilson_loop(ym_ensemble *e, int64_t chain, const int64_t *start, const int32_t *steps,
                       int64_t n_steps, double *out2) {
    if (!e || !start || !out2) return YM_ERR_NULL_ARGUMENT;
    int32_t st = open_chain(e, chain);
    if (st) return st;
    if ((st = require_f64(e))) return st;
    const ChainInfo &c = e->chains[chain];
    if (e->group == YM_GROUP_SU3) {
        if ((st = validate_steps(steps, n_steps))) return st;
        if (!coord_ok(c, start)) return YM_ERR_COORDINATE_OUT_OF_RANGE;
    } else {
        if (!coord_ok(c, start)) return YM_ERR_COORDINATE_OUT_OF_RANGE;
        if ((st = validate_steps(steps, n_steps))) return st;
    }
    double v[2];
    st = run_path(e, chain, steps, n_steps, lex_host(c, start), 1, v, nullptr);
    if (st) return st;
    int64_t disp[4];
    path_displacement(c, steps, n_steps, disp);
    for (int d = 0; d < 4; ++d)
        if (disp[d]) return YM_ERR_PATH_NOT_CLOSED;
    out2[0] = v[0];
    out2[1] = v[1];
    return YM_OK;
}

int32_t ym_wilson_loop_sites(ym_ensemble *e, int64_t chain, const int32_t *steps, int64_t n_steps,
                             double *out) {
    if (!e || !out) return YM_ERR_NULL_ARGUMENT;
    int32_t st = open_chain(e, chain);
    if (st) return st;
    if ((st = require_f64(e))) return st;
    if ((st = validate_steps(steps, n_steps))) return st;
    const ChainInfo &c = e->chains[chain];
    int64_t disp[4];
    path_displacement(c, steps, n_steps, disp);
    for (int d = 0; d < 4; ++d)
        if (disp[d]) return YM_ERR_PATH_NOT_CLOSED;
    return run_path(e, chain, steps, n_steps, 0, c.volume, out, nullptr);
}

int32_t ym_polyakov_loop_sites(ym_ensemble *e, int64_t chain, int32_t direction, double *out) {
    if (!e || !out) return YM_ERR_NULL_ARGUMENT;
    int32_t st = open_chain(e, chain);
    if (st) return st;
    if ((st = require_f64(e))) return st;
    if (direction < 0 || direction >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
    const ChainInfo &c = e->chains[chain];
    const int64_t winding = c.n[direction];
    if (e->group == YM_GROUP_SU2 && winding > ym::kMaxPathSteps) return YM_ERR_PATH_TOO_LONG;
    std::vector<int32_t> steps((size_t)winding, direction + 1);
    return run_path(e, chain, steps.data(), winding, 0, c.volume, out, nullptr);
}

int32_t ym_polyakov_loop(ym_ensemble *e, int64_t chain, const int64_t *start, int32_t direction,
                         double *out2) {
    if (!e || !start || !out2) return YM_ERR_NULL_ARGUMENT;
    int32_t st = open_chain(e, chain);
    if (st) return st;
    if ((st = require_f64(e))) return st;
    if (direction < 0 || direction >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
    const ChainInfo &c = e->chains[chain];
    if (!coord_ok(c, start)) return YM_ERR_COORDINATE_OUT_OF_RANGE;
    const int64_t winding = c.n[direction];
    if (e->group == YM_GROUP_SU2 && winding > ym::kMaxPathSteps) return YM_ERR_PATH_TOO_LONG;
    std::vector<int32_t> steps((size_t)winding, direction + 1);
    return run_path(e, chain, steps.data(), winding, lex_host(c, start), 1, out2, nullptr);
}

int32_t ym_plaquette(ym_ensemble *e, int64_t chain, const int64_t *x, int32_t mu, int32_t nu,
                     double *out) {
    if (!e || !x || !out) return YM_ERR_NULL_ARGUMENT;
    int32_t st = open_chain(e, chain);
    if (st) return st;
    if ((st = require_f64(e))) return st;
    if (mu < 0 || mu >= 4 || nu < 0 || nu >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
    if (mu == nu) return YM_ERR_DIRECTIONS_MUST_DIFFER;
    const ChainInfo &c = e->chains[chain];
    if (!coord_ok(c, x)) return YM_ERR_COORDINATE_OUT_OF_RANGE;
    YM_Q(ensure_query(e));
    if (e->group == YM_GROUP_SU3)
        ym::k_plaquette_at<3><<<1, 1, 0, e->stream>>>(e->d_chains, (int)chain, e->d_links, (int)x[0],
                                                      (int)x[1], (int)x[2], (int)x[3], mu, nu,
                                                      e->d_query, e->d_query_error);
    else
        ym::k_plaquette_at<2><<<1, 1, 0, e->stream>>>(e->d_chains, (int)chain, e->d_links, (int)x[0],
                                                      (int)x[1], (int)x[2], (int)x[3], mu, nu,
                                                      e->d_query, e->d_query_error);
    YM_Q(cudaGetLastError());
    if ((st = copy_small(e, out, e->group == YM_GROUP_SU3 ? 18 : 4))) return st;
    return take_query_error(e, YM_ERR_NON_FINITE_ACTION);
}

int32_t ym_wilson_action(ym_ensemble *e, double beta, double *per_chain) {
    if (!e || !per_chain) return YM_ERR_NULL_ARGUMENT;
    int32_t st = open_chain(e, 0);
    if (st) return st;
    if ((st = require_f64(e))) return st;
    if (!std::isfinite(beta)) return YM_ERR_NON_FINITE_BETA;   // validate_beta lib.rs:132-140
    if (beta < 0.0) return YM_ERR_NEGATIVE_BETA;
    YM_Q(ensure_query(e));
    for (int64_t ch = 0; ch < e->n_chains; ++ch) {
        const ChainInfo &c = e->chains[ch];
        YM_Q(ensure_terms(e, 6 * c.volume));
        if (e->group == YM_GROUP_SU3)
            ym::k_action_terms<3><<<ym::grid_of(c.volume), ym::kThreads, 0, e->stream>>>(
                e->d_chains, (int)ch, e->d_links, e->d_terms, e->d_query_error);
        else
            ym::k_action_terms<2><<<ym::grid_of(c.volume), ym::kThreads, 0, e->stream>>>(
                e->d_chains, (int)ch, e->d_links, e->d_terms, e->d_query_error);
        YM_Q(cudaGetLastError());
        ym::k_sequential_action<<<1, 32, 0, e->stream>>>(e->d_terms, 6 * c.volume, beta, e->d_query);
        YM_Q(cudaGetLastError());
        double r[2];
        if ((st = copy_small(e, r, 2))) return st;
        if ((st = take_query_error(e, YM_ERR_NON_FINITE_ACTION))) return st;
        if (!std::isfinite(r[0]) || !std::isfinite(r[1])) return YM_ERR_NON_FINITE_ACTION;
        per_chain[ch] = r[1];
    }
    return YM_OK;
}

int32_t ym_su2_staple(ym_ensemble *e, int64_t chain, const int64_t *x, int32_t mu, double *comp4,
                      int64_t *terms) {
    if (!e || !x || !comp4) return YM_ERR_NULL_ARGUMENT;
    int32_t st = open_chain(e, chain);
    if (st) return st;
    if (e->group != YM_GROUP_SU2) return YM_ERR_WRONG_GROUP;
    if (mu < 0 || mu >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;   // lib.rs:508-509
    if (!coord_ok(e->chains[chain], x)) return YM_ERR_COORDINATE_OUT_OF_RANGE;
    YM_Q(ensure_query(e));
    ym::k_su2_staple_at<<<1, 1, 0, e->stream>>>(e->d_chains, (int)chain, e->d_links, (int)x[0],
                                                (int)x[1], (int)x[2], (int)x[3], mu, e->d_query);
    YM_Q(cudaGetLastError());
    if ((st = copy_small(e, comp4, 4))) return st;
    if (terms) *terms = 6;
    return YM_OK;
}

static int32_t local_action(ym_ensemble *e, int64_t chain, const int64_t *x, int32_t mu,
                            const double *cand, double beta, int mode, double *out) {
    if (!e || !x || !out || (mode == 1 && !cand)) return YM_ERR_NULL_ARGUMENT;
    int32_t st = open_chain(e, chain);
    if (st) return st;
    if (e->group != YM_GROUP_SU3) return YM_ERR_WRONG_GROUP;
    if ((st = require_f64(e))) return st;
    // local_action_difference (su3_ensemble.rs:319-334): lattice.link(x, mu)
    // first (direction, then coordinate), then the beta gate of the action.
    if (mu < 0 || mu >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
    if (!coord_ok(e->chains[chain], x)) return YM_ERR_COORDINATE_OUT_OF_RANGE;
    if (!std::isfinite(beta) || beta < 0.0 || beta > ym::kMaxSu3Beta)
        return YM_ERR_BETA_OUTSIDE_REFERENCE_RANGE;
    if (mode == 1) {
        // a candidate must be an Su3 (Su3::from_checked_matrix gates,
        // su3.rs:242-253), as the reference's type guarantees
        for (int i = 0; i < 18; ++i)
            if (!std::isfinite(cand[i])) return YM_ERR_NON_FINITE_MATRIX;
    }
    YM_Q(ensure_query(e));
    if (mode == 1)
        YM_Q(cudaMemcpyAsync(e->d_query + 32, cand, 18 * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    ym::k_local_action<<<1, 1, 0, e->stream>>>(e->d_chains, (int)chain, e->d_links, (int)x[0],
                                               (int)x[1], (int)x[2], (int)x[3], mu,
                                               e->d_query + 32, beta, mode, e->d_query,
                                               e->d_query_error);
    YM_Q(cudaGetLastError());
    if ((st = copy_small(e, out, 1))) return st;
    return take_query_error(e, YM_ERR_NON_FINITE_STATISTIC);
}

int32_t ym_su3_local_link_action(ym_ensemble *e, int64_t chain, const int64_t *x, int32_t mu,
                                 double beta, double *out) {
    return local_action(e, chain, x, mu, nullptr, beta, 0, out);
}

int32_t ym_su3_local_action_difference(ym_ensemble *e, int64_t chain, const int64_t *x, int32_t mu,
                                       const double *candidate, double beta, double *out) {
    return local_action(e, chain, x, mu, candidate, beta, 1, out);
}

int32_t ym_su3_gauge_transform(ym_ensemble *src, int64_t chain, const double *site_gauges,
                               ym_ensemble *dst, int64_t dst_chain) {
    if (!src || !dst || !site_gauges) return YM_ERR_NULL_ARGUMENT;
    int32_t st = open_chain(src, chain);
    if (st) return st;
    if (dst_chain < 0 || dst_chain >= dst->n_chains) return YM_ERR_INVALID_ARGUMENT;
    if (src->group != YM_GROUP_SU3 || dst->group != YM_GROUP_SU3) return YM_ERR_WRONG_GROUP;
    if ((st = require_f64(src)) || (st = require_f64(dst))) return st;
    if (src->device != dst->device) return YM_ERR_INVALID_ARGUMENT;
    const ChainInfo &c = src->chains[chain];
    const ChainInfo &d = dst->chains[dst_chain];
    for (int k = 0; k < 4; ++k)
        if (c.n[k] != d.n[k]) return YM_ERR_LATTICE_EXTENTS_MISMATCH;
    for (int64_t i = 0; i < c.volume * 18; ++i)
        if (!std::isfinite(site_gauges[i])) return YM_ERR_NON_FINITE_MATRIX;
    YM_Q(ensure_query(src));
    double2 *d_g = nullptr;
    const size_t bytes = (size_t)c.volume * 9 * sizeof(double2);
    YM_Q(cudaMallocAsync(reinterpret_cast<void **>(&d_g), bytes, src->stream));
    cudaError_t err = cudaMemcpyAsync(d_g, site_gauges, bytes, cudaMemcpyHostToDevice, src->stream);
    if (err == cudaSuccess && dst != src) {
        // dst's stream waits for src's work (the gauge upload) and src's
        // stream waits for the transform before the buffer is released
        err = cudaStreamSynchronize(dst->stream);
    }
    if (err == cudaSuccess) {
        ym::k_gauge_transform<<<ym::grid_of(c.volume), ym::kThreads, 0, src->stream>>>(
            src->d_chains, (int)chain, src->d_links, dst->d_chains, (int)dst_chain, dst->d_links, d_g,
            src->d_query_error);
        err = cudaGetLastError();
    }
    const cudaError_t f = cudaFreeAsync(d_g, src->stream);
    if (err == cudaSuccess) err = f;
    if (err != cudaSuccess) return ym::record_cuda_status(err);
    return take_query_error(src, YM_ERR_NON_FINITE_ACTION);
}

// Su3Lattice4::link / set_link (su3_lattice.rs:153-166), Lattice4::link /
// set_link: one link in the reference layout (18 or 4 doubles).
int32_t ym_ensemble_get_link(ym_ensemble *e, int64_t chain, const int64_t *x, int32_t mu, double *out) {
    if (!e || !x || !out) return YM_ERR_NULL_ARGUMENT;
    int32_t st = open_chain(e, chain);
    if (st) return st;
    if (mu < 0 || mu >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
    const ChainInfo &c = e->chains[chain];
    if (!coord_ok(c, x)) return YM_ERR_COORDINATE_OUT_OF_RANGE;
    YM_Q(ensure_query(e));
    const int64_t s = slot_host(c, x);
    if (e->precision == YM_PREC_F32_TWO_ROW) {
        YM_Q(ym::launch_f32_get_link(e, chain, s, mu, reinterpret_cast<double2 *>(e->d_query)));
    } else {
        const int entries = e->group == YM_GROUP_SU3 ? 9 : 2;
        ym::k_link_get<<<1, 32, 0, e->stream>>>(e->d_chains, (int)chain, e->d_links, s, mu, entries,
                                                reinterpret_cast<double2 *>(e->d_query));
        YM_Q(cudaGetLastError());
    }
    return copy_small(e, out, e->group == YM_GROUP_SU3 ? 18 : 4);
}

int32_t ym_ensemble_set_link(ym_ensemble *e, int64_t chain, const int64_t *x, int32_t mu,
                             const double *value) {
    if (!e || !x || !value) return YM_ERR_NULL_ARGUMENT;
    int32_t st = open_chain(e, chain);
    if (st) return st;
    if (mu < 0 || mu >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
    const ChainInfo &c = e->chains[chain];
    if (!coord_ok(c, x)) return YM_ERR_COORDINATE_OUT_OF_RANGE;
    const int n = e->group == YM_GROUP_SU3 ? 18 : 4;
    YM_Q(ensure_query(e));
    YM_Q(cudaMemcpyAsync(e->d_query, value, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    const int64_t s = slot_host(c, x);
    if (e->precision == YM_PREC_F32_TWO_ROW) {
        YM_Q(ym::launch_f32_set_link(e, chain, s, mu, reinterpret_cast<const double2 *>(e->d_query)));
    } else {
        ym::k_link_set<<<1, 32, 0, e->stream>>>(e->d_chains, (int)chain, e->d_links, s, mu, n / 2,
                                                reinterpret_cast<const double2 *>(e->d_query));
        YM_Q(cudaGetLastError());
    }
    YM_Q(cudaStreamSynchronize(e->stream));
    return YM_OK;
}

}  // extern "C"
