// learned.cu -- the learned SU(3) Metropolis proposal on the fifth-generation
// tensor cores (no reference counterpart; the definition of features,
// network, objective and proposal is in include/ym_learned.h).
//
// Every kernel here works on tiles of 128 rows (links or training records),
// one thread per row, four warps.  The network runs as a chain of
// tcgen05.mma (kind::f16, BF16 operands from shared memory, FP32
// accumulators in tensor memory): thread 0 issues, tcgen05.commit arrives on
// an mbarrier, all threads wait (time-bounded), read their row back with
// tcgen05.ld 32x32b (warp w owns lanes 32w..32w+31), apply bias and ReLU in
// FP32, round to BF16 and write the next layer's operand tile.
//
//   k_lp_records   staple, features and M = U A of one sub-sweep's links
//   k_lp_forward   y = net(x) for host-supplied features
//   k_lp_grad      forward + objective + backward of one tile: weight
//                  gradients as M=64 MMAs over the tile's 128 rows,
//                  per-tile partial sums written for a fixed-order reduction
//   k_lp_adam      fixed-order reduction of the partials, Adam step, BF16
//                  weight image for the next launch
//   k_lp_sweep     the learned sub-sweep: staple -> features -> network ->
//                  eight hits, fused in one kernel
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "su3_f32.cuh"
#include "umma.cuh"
#include "ym_internal.hpp"

namespace ym {
namespace lp {

constexpr int kRows = 128;
constexpr uint32_t kOffW1 = 0, kOffW2 = 2048, kOffW3 = 10240, kImageBytes = 12288;
constexpr uint32_t kTileX = 128 * 16 * 2;   // 4096
constexpr uint32_t kTileH = 128 * 64 * 2;   // 16384
constexpr uint64_t kWaitNs = 200000000ull;  // 0.2 s per MMA group
constexpr unsigned kErrWait = 1u;

// Shared-memory layouts (bytes from the 1024-aligned base).
struct FwdLayout {   // forward-only kernels: H2 overwrites H1
    static constexpr uint32_t X = kImageBytes, H1 = X + kTileX, H2 = H1, BIAS = H1 + kTileH,
                              MBAR = BIAS + 144 * 4, SLOT = MBAR + 8, BYTES = SLOT + 56;
};
struct GradLayout {
    static constexpr uint32_t X = kImageBytes, H1 = X + kTileX, H2 = H1 + kTileH, DY = H2 + kTileH,
                              DZ2 = DY + kTileX, DZ1 = DZ2 + kTileH, BIAS = DZ1 + kTileH,
                              MBAR = BIAS + 144 * 4, SLOT = MBAR + 8, BYTES = SLOT + 56;
};
static_assert(FwdLayout::BYTES % 16 == 0 && GradLayout::BYTES % 16 == 0, "layout");

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ float bf16_at(const uint8_t *tile, int r, int c, int cols) {
    const __nv_bfloat16 v = *reinterpret_cast<const __nv_bfloat16 *>(tile + umma::tile_offset(r, c, cols));
    return __bfloat162float(v);
}

// Eight consecutive columns c0..c0+7 of row r, rounded to BF16, as one
// 16-byte store.
__device__ __forceinline__ void store8(uint8_t *tile, int r, int c0, int cols, const float *v) {
    uint4 q;
    q.x = pack_bf16x2(v[0], v[1]);
    q.y = pack_bf16x2(v[2], v[3]);
    q.z = pack_bf16x2(v[4], v[5]);
    q.w = pack_bf16x2(v[6], v[7]);
    *reinterpret_cast<uint4 *>(tile + umma::tile_offset(r, c0, cols)) = q;
}

// Weight image and biases into shared memory (all threads).
__device__ __forceinline__ void stage_weights(uint8_t *sm, const uint4 *__restrict__ image,
                                              const float *__restrict__ params, float *bias) {
    uint4 *dst = reinterpret_cast<uint4 *>(sm);
    for (int i = threadIdx.x; i < (int)(kImageBytes / 16); i += kRows) dst[i] = image[i];
    for (int i = threadIdx.x; i < 144; i += kRows) {
        const int src = i < 64 ? YM_LP_OFF_B1 + i : (i < 128 ? YM_LP_OFF_B2 + i - 64 : YM_LP_OFF_B3 + i - 128);
        bias[i] = params[src];
    }
}

// Block-uniform wait for the next MMA group; on a timeout the error bit is
// set, one more bounded wait lets the group drain, and false is returned.
__device__ __forceinline__ bool wait_group(uint64_t *mbar, uint32_t &phase, unsigned *err) {
    bool ok = umma::mbar_wait(mbar, phase, kWaitNs);
    ok = __syncthreads_and(ok) != 0;
    if (!ok) {
        if (threadIdx.x == 0) atomicOr(err, kErrWait);
        umma::mbar_wait(mbar, phase, kWaitNs);
    }
    phase ^= 1u;
    umma::fence_after();
    return ok;
}

// Make this thread's shared-memory writes and tensor-memory reads ordered
// before the next MMA group, then let thread 0 issue.
__device__ __forceinline__ void sync_for_mma() {
    umma::fence_proxy_async();
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
}

// K-step loop of one MMA group member: D += A_k B_k^T over ksteps steps.
__device__ __forceinline__ void mma_chain(uint32_t d, uint32_t a, uint32_t a_lbo, uint32_t a_sbo,
                                          uint32_t a_step, uint32_t b, uint32_t b_lbo, uint32_t b_sbo,
                                          uint32_t b_step, int ksteps, uint32_t idesc) {
    for (int k = 0; k < ksteps; ++k)
        umma::mma_bf16(d, umma::sdesc(a + k * a_step, a_lbo, a_sbo),
                       umma::sdesc(b + k * b_step, b_lbo, b_sbo), idesc, k > 0 ? 1u : 0u);
}

__device__ __forceinline__ uint32_t lane_base(uint32_t tmem) {
    return tmem + ((uint32_t)((threadIdx.x >> 5) * 32) << 16);
}

// Forward pass of the tile whose features are already in X (and weights,
// biases staged, shared memory fenced and synchronised).  d1, d2, d3 are
// tensor-memory column offsets of the three accumulators.  y receives the
// 16 outputs of this thread's row.  Returns false on a wait timeout.
template <class L>
__device__ __forceinline__ bool forward_tile(uint8_t *sm, uint32_t tmem, uint64_t *mbar,
                                             uint32_t &phase, uint32_t d1, uint32_t d2, uint32_t d3,
                                             unsigned *err, float y[16]) {
    const uint32_t base = umma::smem_u32(sm);
    const float *bias = reinterpret_cast<const float *>(sm + L::BIAS);
    const int r = threadIdx.x;
    if (threadIdx.x == 0) {
        mma_chain(tmem + d1, base + L::X, 128, 256, 0, base + kOffW1, 128, 256, 0, 1,
                  umma::idesc_bf16(128, 64, 0, 0));
        umma::commit(mbar);
    }
    if (!wait_group(mbar, phase, err)) return false;
#pragma unroll 1
    for (int c = 0; c < 64; c += 16) {
        float v[16];
        umma::tmem_ld16(lane_base(tmem) + d1 + c, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = fmaxf(v[i] + bias[c + i], 0.f);
        store8(sm + L::H1, r, c, 64, v);
        store8(sm + L::H1, r, c + 8, 64, v + 8);
    }
    sync_for_mma();
    if (threadIdx.x == 0) {
        mma_chain(tmem + d2, base + L::H1, 128, 1024, 256, base + kOffW2, 128, 1024, 256, 4,
                  umma::idesc_bf16(128, 64, 0, 0));
        umma::commit(mbar);
    }
    if (!wait_group(mbar, phase, err)) return false;
#pragma unroll 1
    for (int c = 0; c < 64; c += 16) {
        float v[16];
        umma::tmem_ld16(lane_base(tmem) + d2 + c, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = fmaxf(v[i] + bias[64 + c + i], 0.f);
        store8(sm + L::H2, r, c, 64, v);
        store8(sm + L::H2, r, c + 8, 64, v + 8);
    }
    sync_for_mma();
    if (threadIdx.x == 0) {
        mma_chain(tmem + d3, base + L::H2, 128, 1024, 256, base + kOffW3, 128, 1024, 256, 4,
                  umma::idesc_bf16(128, 16, 0, 0));
        umma::commit(mbar);
    }
    if (!wait_group(mbar, phase, err)) return false;
    umma::tmem_ld16(lane_base(tmem) + d3, y);
#pragma unroll
    for (int i = 0; i < 16; ++i) y[i] += bias[128 + i];
    return true;
}

__device__ __forceinline__ void write_x_row(uint8_t *x_tile, int r, const float f[16]) {
    store8(x_tile, r, 0, 16, f);
    store8(x_tile, r, 8, 16, f + 8);
}

// Generator probabilities (cumulative, first seven) and half width.
__device__ __forceinline__ void proposal_from(const float y[16], float cum[7], float &scale) {
    float mx = y[0];
#pragma unroll
    for (int a = 1; a < 8; ++a) mx = fmaxf(mx, y[a]);
    float e[8], z = 0.f;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        e[a] = __expf(y[a] - mx);
        z += e[a];
    }
    const float iz = (1.f - (float)YM_LP_GENERATOR_FLOOR) / z;
    const float base = (float)YM_LP_GENERATOR_FLOOR * 0.125f;
    float c = 0.f;
#pragma unroll
    for (int a = 0; a < 7; ++a) {
        c += base + e[a] * iz;
        cum[a] = c;
    }
    const float sig = 1.f / (1.f + __expf(-y[8]));
    scale = (float)YM_LP_SCALE_MIN + (float)(YM_LP_SCALE_MAX - YM_LP_SCALE_MIN) * sig;
}

// ReTr(R_g(theta) M) and d/dtheta (closed forms of the header's definition).
__device__ __forceinline__ void retr_rotated(int g, const float *m, float tr, float th, float &f,
                                             float &df) {
    // m: row-major re/im of M; element (i, j) at 2 * (3 i + j)
    if (g < 7) {
        const int i = (g <= 4) ? 0 : 1, j = (g <= 2) ? 1 : 2;
        const int kind = (g == 2) ? 2 : ((g == 1 || g == 4 || g == 6) ? 1 : 0);
        const float mii_r = m[2 * (4 * i)], mjj_r = m[2 * (4 * j)];
        const float c1 = mii_r + mjj_r;
        float c2;
        if (kind == 0) c2 = -(m[2 * (3 * i + j) + 1] + m[2 * (3 * j + i) + 1]);
        else if (kind == 1) c2 = m[2 * (3 * j + i)] - m[2 * (3 * i + j)];
        else c2 = m[2 * (4 * j) + 1] - m[2 * (4 * i) + 1];
        float s, c;
        sincosf(0.5f * th, &s, &c);
        f = (tr - c1) + c1 * c + c2 * s;
        df = 0.5f * (-c1 * s + c2 * c);
    } else {
        const float k = 0.28867513459481287f;
        const float mr = m[0] + m[8], mi = m[1] + m[9];
        float s, c, s2, c2;
        sincosf(k * th, &s, &c);
        sincosf(2.f * k * th, &s2, &c2);
        f = c * mr - s * mi + c2 * m[16] + s2 * m[17];
        df = k * (-s * mr - c * mi) + 2.f * k * (-s2 * m[16] + c2 * m[17]);
    }
}

// Objective O = E + w H(q) of one record and dO/dy (outputs 0..8).
__device__ __forceinline__ float objective_row(const float y[16], const float *m, float b3, float dy[9]) {
    float mx = y[0];
#pragma unroll
    for (int a = 1; a < 8; ++a) mx = fmaxf(mx, y[a]);
    float q[8], p[8], z = 0.f;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        q[a] = expf(y[a] - mx);
        z += q[a];
    }
    constexpr float F = (float)YM_LP_GENERATOR_FLOOR;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        q[a] /= z;
        p[a] = F * 0.125f + (1.f - F) * q[a];
    }
    const float sig = 1.f / (1.f + expf(-y[8]));
    const float s = (float)YM_LP_SCALE_MIN + (float)(YM_LP_SCALE_MAX - YM_LP_SCALE_MIN) * sig;
    const float tr = m[0] + m[8] + m[16];
    constexpr int K = YM_LP_QUADRATURE;
    float J[8], E = 0.f, dEs = 0.f;
#pragma unroll 1
    for (int a = 0; a < 8; ++a) {
        float j = 0.f, dj = 0.f;
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const float gk = (q + 0.5f) / K;
#pragma unroll
            for (int sg = -1; sg <= 1; sg += 2) {
                const float dth = sg * gk, th = s * dth;
                float f, df;
                retr_rotated(a, m, tr, th, f, df);
                const float ds = b3 * (tr - f), dds = -b3 * df;
                const float al = ds > 0.f ? expf(-ds) : 1.f;
                const float dal = ds > 0.f ? -al * dds : 0.f;
                j += al * ds * ds;
                dj += (dal * ds * ds + 2.f * al * ds * dds) * dth;
            }
        }
        J[a] = j / (2.f * K);
        E += p[a] * J[a];
        dEs += p[a] * (dj / (2.f * K));
    }
    float Eq = 0.f, H = 0.f;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        Eq += q[a] * J[a];
        H -= q[a] * logf(q[a]);
    }
    constexpr float W = (float)YM_LP_ENTROPY_WEIGHT;
#pragma unroll
    for (int a = 0; a < 8; ++a) dy[a] = (1.f - F) * q[a] * (J[a] - Eq) - W * q[a] * (logf(q[a]) + H);
    dy[8] = dEs * (float)(YM_LP_SCALE_MAX - YM_LP_SCALE_MIN) * sig * (1.f - sig);
    return E + W * H;
}

__device__ __forceinline__ void setup_block(uint8_t *sm, uint32_t slot_off, uint32_t mbar_off,
                                            uint32_t ncols) {
    if (threadIdx.x < 32) umma::tmem_alloc(reinterpret_cast<uint32_t *>(sm + slot_off), ncols);
    if (threadIdx.x == 0) umma::mbar_init(reinterpret_cast<uint64_t *>(sm + mbar_off), 1);
}

__device__ __forceinline__ void teardown_block(uint32_t tmem, uint32_t ncols) {
    umma::fence_before();
    __syncthreads();
    if (threadIdx.x < 32) umma::tmem_dealloc(tmem, ncols);
}

// ------------------------------------------------------------------ kernels

template <int MU>
__global__ void __launch_bounds__(kRows)
k_lp_records(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles,
             const float2 *__restrict__ links, int parity, float *__restrict__ feat,
             float *__restrict__ mrec, float *__restrict__ b3rec) {
    using namespace f32;
    const Tile tile = tiles[blockIdx.x];
    const ChainInfo c = chains[tile.chain];
    const int64_t t = tile.start + threadIdx.x;
    const int64_t rec = (int64_t)blockIdx.x * kRows + threadIdx.x;
    float f[16], m[18];
#pragma unroll
    for (int i = 0; i < 16; ++i) f[i] = 0.f;
#pragma unroll
    for (int i = 0; i < 18; ++i) m[i] = 0.f;
    float b3 = -1.f;   // padding row
    if (t < c.half) {
        const int64_t s = (int64_t)parity * c.half + t;
        const Coord x = decode_storage(c, s);
        const m3f a = staple_f<MU>(links, c, x, parity);
        const m3f u = load_f(links, c, s, MU);
        staple_features(a, (float)c.beta, f);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                cf v = cfm(0.f, 0.f);
#pragma unroll
                for (int k = 0; k < 3; ++k) cffma(v, u.e[i][k], a.e[k][j]);
                m[2 * (3 * i + j)] = v.re;
                m[2 * (3 * i + j) + 1] = v.im;
            }
        b3 = (float)(c.beta / 3.0);
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) feat[rec * 16 + i] = f[i];
#pragma unroll
    for (int i = 0; i < 18; ++i) mrec[rec * 18 + i] = m[i];
    b3rec[rec] = b3;
}

__global__ void __launch_bounds__(kRows)
k_lp_forward(const float *__restrict__ feat, int64_t n, const uint4 *__restrict__ image,
             const float *__restrict__ params, float *__restrict__ y_out, unsigned *err) {
    using L = FwdLayout;
    extern __shared__ __align__(1024) uint8_t sm[];
    setup_block(sm, L::SLOT, L::MBAR, 64);
    stage_weights(sm, image, params, reinterpret_cast<float *>(sm + L::BIAS));
    const int64_t row = (int64_t)blockIdx.x * kRows + threadIdx.x;
    float f[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) f[i] = row < n ? feat[row * 16 + i] : 0.f;
    write_x_row(sm + L::X, threadIdx.x, f);
    sync_for_mma();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t *>(sm + L::SLOT);
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sm + L::MBAR);
    uint32_t phase = 0;
    float y[16];
    if (forward_tile<L>(sm, tmem, mbar, phase, 0, 0, 0, err, y) && row < n) {
#pragma unroll
        for (int i = 0; i < 16; ++i) y_out[row * 16 + i] = y[i];
    }
    teardown_block(tmem, 64);
}

// One tile of the objective gradient.  partial[tile][p] receives the tile's
// sum over rows of d(-E)/d param p; partial[tile][YM_LP_PARAMS] the sum of E.
__global__ void __launch_bounds__(kRows)
k_lp_grad(const float *__restrict__ feat, const float *__restrict__ mrec,
          const float *__restrict__ b3rec, int64_t n, const uint4 *__restrict__ image,
          const float *__restrict__ params, float *__restrict__ partial, int64_t stride,
          unsigned *err) {
    using L = GradLayout;
    extern __shared__ __align__(1024) uint8_t sm[];
    float *red = reinterpret_cast<float *>(sm + L::SLOT + 16);
    setup_block(sm, L::SLOT, L::MBAR, 256);
    stage_weights(sm, image, params, reinterpret_cast<float *>(sm + L::BIAS));
    const int r = threadIdx.x;
    const int64_t row = (int64_t)blockIdx.x * kRows + r;
    const bool valid = row < n && b3rec[row] >= 0.f;
    float f[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) f[i] = valid ? feat[row * 16 + i] : 0.f;
    write_x_row(sm + L::X, r, f);
    sync_for_mma();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t *>(sm + L::SLOT);
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sm + L::MBAR);
    const uint32_t base = umma::smem_u32(sm);
    float *out = partial + (int64_t)blockIdx.x * stride;
    uint32_t phase = 0;
    float y[16];
    bool ok = forward_tile<L>(sm, tmem, mbar, phase, 0, 64, 128, err, y);
    if (ok) {
        // objective and output gradient of this row (zero for padding rows)
        float m[18], dE[9];
#pragma unroll
        for (int i = 0; i < 18; ++i) m[i] = valid ? mrec[row * 18 + i] : 0.f;
        float e = 0.f;
        if (valid) e = objective_row(y, m, b3rec[row], dE);
        float dy[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) dy[i] = (valid && i < 9) ? -dE[i] : 0.f;
        store8(sm + L::DY, r, 0, 16, dy);
        store8(sm + L::DY, r, 8, 16, dy + 8);
        // fixed-order block sum of E
        float w = e;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
        if ((r & 31) == 0) red[r >> 5] = w;
        sync_for_mma();
        if (r == 0) {
            out[YM_LP_PARAMS] = (red[0] + red[1]) + (red[2] + red[3]);
            // dH2 = dY W3 (M128 N64 K16), dW3^T = H2^T dY (M64 N16 K128)
            mma_chain(tmem + 0, base + L::DY, 128, 256, 0, base + kOffW3, 1024, 128, 0, 1,
                      umma::idesc_bf16(128, 64, 0, 1));
            mma_chain(tmem + 160, base + L::H2, 1024, 128, 2048, base + L::DY, 256, 128, 512, 8,
                      umma::idesc_bf16(64, 16, 1, 1));
            umma::commit(mbar);
        }
        ok = wait_group(mbar, phase, err);
    }
    if (ok) {
        const int w = r >> 5, l = r & 31;
#pragma unroll 1
        for (int c = 0; c < 64; c += 16) {
            float v[16];
            umma::tmem_ld16(lane_base(tmem) + 0 + c, v);
#pragma unroll
            for (int i = 0; i < 16; ++i)
                v[i] = bf16_at(sm + L::H2, r, c + i, 64) > 0.f ? v[i] : 0.f;
            store8(sm + L::DZ2, r, c, 64, v);
            store8(sm + L::DZ2, r, c + 8, 64, v + 8);
        }
        {
            float v[16];
            umma::tmem_ld16(lane_base(tmem) + 160, v);
            if (l < 16) {
                const int in = 16 * w + l;
#pragma unroll
                for (int o = 0; o < 9; ++o) out[YM_LP_OFF_W3 + o * 64 + in] = v[o];
            }
        }
        sync_for_mma();
        if (r == 0) {
            // dH1 = dZ2 W2 (M128 N64 K64), dW2^T = H1^T dZ2 (M64 N64 K128)
            mma_chain(tmem + 64, base + L::DZ2, 128, 1024, 256, base + kOffW2, 1024, 128, 2048, 4,
                      umma::idesc_bf16(128, 64, 0, 1));
            mma_chain(tmem + 192, base + L::H1, 1024, 128, 2048, base + L::DZ2, 1024, 128, 2048, 8,
                      umma::idesc_bf16(64, 64, 1, 1));
            umma::commit(mbar);
        }
        ok = wait_group(mbar, phase, err);
    }
    if (ok) {
        const int w = r >> 5, l = r & 31;
#pragma unroll 1
        for (int c = 0; c < 64; c += 16) {
            float v[16];
            umma::tmem_ld16(lane_base(tmem) + 64 + c, v);
#pragma unroll
            for (int i = 0; i < 16; ++i)
                v[i] = bf16_at(sm + L::H1, r, c + i, 64) > 0.f ? v[i] : 0.f;
            store8(sm + L::DZ1, r, c, 64, v);
            store8(sm + L::DZ1, r, c + 8, 64, v + 8);
        }
#pragma unroll 1
        for (int c = 0; c < 64; c += 16) {
            float v[16];
            umma::tmem_ld16(lane_base(tmem) + 192 + c, v);
            if (l < 16) {
                const int in = 16 * w + l;
#pragma unroll
                for (int i = 0; i < 16; ++i) out[YM_LP_OFF_W2 + (c + i) * 64 + in] = v[i];
            }
        }
        sync_for_mma();
        if (r == 0) {
            // dW1 = dZ1^T X (M64 N16 K128)
            mma_chain(tmem + 128, base + L::DZ1, 1024, 128, 2048, base + L::X, 256, 128, 512, 8,
                      umma::idesc_bf16(64, 16, 1, 1));
            umma::commit(mbar);
        }
        ok = wait_group(mbar, phase, err);
    }
    if (ok) {
        const int w = r >> 5, l = r & 31;
        float v[16];
        umma::tmem_ld16(lane_base(tmem) + 128, v);
        if (l < 16) {
            const int o = 16 * w + l;
#pragma unroll
            for (int k = 0; k < 16; ++k) out[YM_LP_OFF_W1 + o * 16 + k] = v[k];
        }
        // bias gradients: column sums in row order
        float s = 0.f;
        if (r < 64) {
            for (int q = 0; q < kRows; ++q) s += bf16_at(sm + L::DZ2, q, r, 64);
            out[YM_LP_OFF_B2 + r] = s;
        } else {
            for (int q = 0; q < kRows; ++q) s += bf16_at(sm + L::DZ1, q, r - 64, 64);
            out[YM_LP_OFF_B1 + r - 64] = s;
        }
        if (r < 9) {
            float t = 0.f;
            for (int q = 0; q < kRows; ++q) t += bf16_at(sm + L::DY, q, r, 16);
            out[YM_LP_OFF_B3 + r] = t;
        }
    }
    teardown_block(tmem, 256);
}

__device__ __forceinline__ bool is_padding_param(int p) {
    return (p >= YM_LP_OFF_W3 + 9 * 64 && p < YM_LP_OFF_B3) || p >= YM_LP_OFF_B3 + 9;
}

// Byte offset of weight p in the BF16 image, or -1 for a bias.
__device__ __forceinline__ int image_offset(int p) {
    if (p < YM_LP_OFF_B1) return (int)kOffW1 + (int)umma::tile_offset(p / 16, p % 16, 16);
    if (p >= YM_LP_OFF_W2 && p < YM_LP_OFF_B2) {
        const int q = p - YM_LP_OFF_W2;
        return (int)kOffW2 + (int)umma::tile_offset(q / 64, q % 64, 64);
    }
    if (p >= YM_LP_OFF_W3 && p < YM_LP_OFF_B3) {
        const int q = p - YM_LP_OFF_W3;
        return (int)kOffW3 + (int)umma::tile_offset(q / 64, q % 64, 64);
    }
    return -1;
}

__global__ void k_lp_image(const float *__restrict__ params, uint8_t *__restrict__ image) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= YM_LP_PARAMS) return;
    const int off = image_offset(p);
    if (off >= 0)
        *reinterpret_cast<__nv_bfloat16 *>(image + off) = __float2bfloat16_rn(params[p]);
}

// Gradient reduction in two fixed-order stages (groups of kGroup tiles, then
// the groups in order), so the result does not depend on scheduling.
constexpr int kGroup = 64;

__global__ void k_lp_reduce_groups(const float *__restrict__ partial, int64_t n_tiles, int64_t stride,
                                   double *__restrict__ groups) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > YM_LP_PARAMS) return;                 // p == YM_LP_PARAMS is the objective
    const int64_t g = blockIdx.y, t0 = g * kGroup;
    const int64_t t1 = t0 + kGroup < n_tiles ? t0 + kGroup : n_tiles;
    double acc = 0.0;
    for (int64_t t = t0; t < t1; ++t) acc += (double)partial[t * stride + p];
    groups[g * stride + p] = acc;
}

// Sum of the groups, then Adam (bias-corrected) and the BF16 image.
// grad_out (optional) receives the mean gradient; objective_out (optional)
// the mean objective.
__global__ void k_lp_adam(const double *__restrict__ groups, int64_t n_groups, int64_t stride,
                          double inv_n, float *__restrict__ params, float *__restrict__ am,
                          float *__restrict__ av, int64_t step, float lr, int update,
                          uint8_t *__restrict__ image, float *__restrict__ grad_out,
                          double *__restrict__ objective_out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > YM_LP_PARAMS) return;
    double g = 0.0;
    for (int64_t t = 0; t < n_groups; ++t) g += groups[t * stride + p];
    if (p == YM_LP_PARAMS) {
        if (objective_out) *objective_out = g * inv_n;
        return;
    }
    const float gf = is_padding_param(p) ? 0.f : (float)(g * inv_n);
    if (grad_out) grad_out[p] = gf;
    if (!update) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float m = b1 * am[p] + (1.f - b1) * gf;
    const float v = b2 * av[p] + (1.f - b2) * gf * gf;
    am[p] = m;
    av[p] = v;
    const float mh = m / (1.f - powf(b1, (float)step));
    const float vh = v / (1.f - powf(b2, (float)step));
    const float w = is_padding_param(p) ? 0.f : params[p] - lr * mh / (sqrtf(vh) + eps);
    params[p] = w;
    const int off = image_offset(p);
    if (off >= 0) *reinterpret_cast<__nv_bfloat16 *>(image + off) = __float2bfloat16_rn(w);
}

// The learned sub-sweep (parity, MU) of a two-row ensemble.
// Persistent: each CTA allocates its tensor memory, initialises its barrier
// and stages the weight image once, then walks the tiles blockIdx.x,
// blockIdx.x + gridDim.x, ...  Every tile's three MMA groups are waited for
// before its hits, so the shared-memory operand tiles and the accumulator
// columns are free again when the next tile writes them.
template <int MU>
__global__ void __launch_bounds__(kRows, 4)
k_lp_sweep(const ChainInfo *__restrict__ chains, const Tile *__restrict__ tiles, int64_t n_tiles,
           float2 *__restrict__ links, int parity, const uint4 *__restrict__ image,
           const float *__restrict__ params, const uint64_t *__restrict__ sweep_ptr,
           unsigned long long *__restrict__ accepts, unsigned *err) {
    using namespace f32;
    using L = FwdLayout;
    extern __shared__ __align__(1024) uint8_t sm[];
    setup_block(sm, L::SLOT, L::MBAR, 64);
    stage_weights(sm, image, params, reinterpret_cast<float *>(sm + L::BIAS));
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sm + L::MBAR);
    uint32_t phase = 0;
    uint32_t tmem = 0;
    const uint64_t sweep = *sweep_ptr;
    for (int64_t ti = blockIdx.x; ti < n_tiles; ti += gridDim.x) {
        const Tile tile = tiles[ti];
        const ChainInfo c = chains[tile.chain];
        const int64_t t = tile.start + threadIdx.x;
        const bool valid = t < c.half;
        const int64_t s = (int64_t)parity * c.half + (valid ? t : 0);
        const Coord x = decode_storage(c, s);
        m3f a;
        float f[16];
        if (valid) {
            a = staple_f<MU>(links, c, x, parity);
            staple_features(a, (float)c.beta, f);
        } else {
#pragma unroll
            for (int i = 0; i < 16; ++i) f[i] = 0.f;
        }
        write_x_row(sm + L::X, threadIdx.x, f);
        sync_for_mma();
        tmem = *reinterpret_cast<volatile uint32_t *>(sm + L::SLOT);
        float y[16];
        const bool ok = forward_tile<L>(sm, tmem, mbar, phase, 0, 0, 0, err, y);
        if (!ok) break;   // block-uniform: the wait gave up and set the error bit
        unsigned accepted = 0;
        if (valid) {
            float cum[7], scale;
            proposal_from(y, cum, scale);
            m3f u = load_f(links, c, s, MU);
            const uint64_t key = link_key(c.seed, sweep, x.lex, MU);
            accepted = visit_learned_f(u, a, c.beta / 3.0, cum, scale, key);
            store_f(links, c, s, MU, u);
        }
        const unsigned warp_sum = __reduce_add_sync(0xffffffffu, accepted);
        if ((threadIdx.x & 31) == 0 && warp_sum)
            atomicAdd(accepts + tile.chain, (unsigned long long)warp_sum);
    }
    if (tmem == 0) tmem = *reinterpret_cast<volatile uint32_t *>(sm + L::SLOT);
    teardown_block(tmem, 64);
}

// The tensor-core kernels' bounded mbarrier wait on a barrier that nothing
// arrives on: it must give up after limit_ns and set the error bit.
__global__ void k_lp_wait_selftest(uint64_t limit_ns, unsigned *err) {
    __shared__ uint64_t mbar;
    if (threadIdx.x == 0) umma::mbar_init(&mbar, 1);
    __syncthreads();
    const bool ok = umma::mbar_wait(&mbar, 0, limit_ns);
    if (!ok && threadIdx.x == 0) atomicOr(err, kErrWait);
}

template <class K>
cudaError_t allow_smem(K kernel, uint32_t bytes) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace lp

// ------------------------------------------------------------------ launchers

cudaError_t launch_lp_wait_selftest(uint64_t limit_ns, unsigned *err, cudaStream_t st) {
    lp::k_lp_wait_selftest<<<1, 32, 0, st>>>(limit_ns, err);
    return cudaGetLastError();
}

cudaError_t launch_lp_records(ym_ensemble *e, int parity, int mu, float *feat, float *m, float *b3) {
    if (e->n_half_tiles == 0) return cudaSuccess;
    const dim3 grid((unsigned)e->n_half_tiles);
    const float2 *links = reinterpret_cast<const float2 *>(e->d_links);
    switch (mu) {
        case 0: lp::k_lp_records<0><<<grid, lp::kRows, 0, e->stream>>>(e->d_chains, e->d_half_tiles, links, parity, feat, m, b3); break;
        case 1: lp::k_lp_records<1><<<grid, lp::kRows, 0, e->stream>>>(e->d_chains, e->d_half_tiles, links, parity, feat, m, b3); break;
        case 2: lp::k_lp_records<2><<<grid, lp::kRows, 0, e->stream>>>(e->d_chains, e->d_half_tiles, links, parity, feat, m, b3); break;
        default: lp::k_lp_records<3><<<grid, lp::kRows, 0, e->stream>>>(e->d_chains, e->d_half_tiles, links, parity, feat, m, b3); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_lp_image(ym_proposal_model *m, cudaStream_t st) {
    lp::k_lp_image<<<(YM_LP_PARAMS + 255) / 256, 256, 0, st>>>(m->d_params, m->d_image);
    return cudaGetLastError();
}

cudaError_t launch_lp_forward(ym_proposal_model *m, const float *feat, int64_t n, float *y,
                              cudaStream_t st) {
    static thread_local int configured_device = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (configured_device != dev) {
        cudaError_t err = lp::allow_smem(lp::k_lp_forward, lp::FwdLayout::BYTES);
        if (err != cudaSuccess) return err;
        configured_device = dev;
    }
    if (n <= 0) return cudaSuccess;
    const unsigned tiles = (unsigned)((n + lp::kRows - 1) / lp::kRows);
    lp::k_lp_forward<<<tiles, lp::kRows, lp::FwdLayout::BYTES, st>>>(
        feat, n, reinterpret_cast<const uint4 *>(m->d_image), m->d_params, y, m->d_error);
    return cudaGetLastError();
}

cudaError_t launch_lp_grad(ym_proposal_model *m, const float *feat, const float *mrec,
                           const float *b3, int64_t n, cudaStream_t st) {
    static thread_local int configured_device = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (configured_device != dev) {
        cudaError_t err = lp::allow_smem(lp::k_lp_grad, lp::GradLayout::BYTES);
        if (err != cudaSuccess) return err;
        configured_device = dev;
    }
    if (n <= 0) return cudaSuccess;
    const unsigned tiles = (unsigned)((n + lp::kRows - 1) / lp::kRows);
    lp::k_lp_grad<<<tiles, lp::kRows, lp::GradLayout::BYTES, st>>>(
        feat, mrec, b3, n, reinterpret_cast<const uint4 *>(m->d_image), m->d_params, m->d_partial,
        kLpPartialStride, m->d_error);
    return cudaGetLastError();
}

cudaError_t launch_lp_adam(ym_proposal_model *m, int64_t n_tiles, int64_t n_valid, float lr,
                           int update, float *grad_out, double *objective_out, cudaStream_t st) {
    if (update) m->adam_step += 1;
    const int64_t n_groups = lp_reduce_groups(n_tiles);
    const unsigned blocks = (YM_LP_PARAMS + 1 + 255) / 256;
    lp::k_lp_reduce_groups<<<dim3(blocks, (unsigned)n_groups), 256, 0, st>>>(m->d_partial, n_tiles,
                                                                           kLpPartialStride, m->d_groups);
    lp::k_lp_adam<<<blocks, 256, 0, st>>>(m->d_groups, n_groups, kLpPartialStride, 1.0 / (double)n_valid,
                                          m->d_params, m->d_adam_m, m->d_adam_v, m->adam_step, lr,
                                          update, m->d_image, grad_out, objective_out);
    return cudaGetLastError();
}

cudaError_t launch_lp_sweep(ym_ensemble *e, ym_proposal_model *m, int parity, int mu) {
    static thread_local int configured_device = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (configured_device != dev) {
        cudaError_t err = lp::allow_smem(lp::k_lp_sweep<0>, lp::FwdLayout::BYTES);
        if (err == cudaSuccess) err = lp::allow_smem(lp::k_lp_sweep<1>, lp::FwdLayout::BYTES);
        if (err == cudaSuccess) err = lp::allow_smem(lp::k_lp_sweep<2>, lp::FwdLayout::BYTES);
        if (err == cudaSuccess) err = lp::allow_smem(lp::k_lp_sweep<3>, lp::FwdLayout::BYTES);
        if (err != cudaSuccess) return err;
        configured_device = dev;
    }
    if (e->n_half_tiles == 0) return cudaSuccess;
    static thread_local int resident_ctas = 0, resident_device = -1;
    if (resident_device != dev) {   // 4 CTAs per SM: registers, shared memory and 4 x 64 TMEM columns
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        resident_ctas = 4 * sms;
        resident_device = dev;
    }
    const int64_t n = e->n_half_tiles;
    const dim3 grid((unsigned)(n < resident_ctas ? n : resident_ctas));
    float2 *links = reinterpret_cast<float2 *>(e->d_links);
    const uint4 *img = reinterpret_cast<const uint4 *>(m->d_image);
    const uint32_t sm = lp::FwdLayout::BYTES;
    switch (mu) {
        case 0: lp::k_lp_sweep<0><<<grid, lp::kRows, sm, e->stream>>>(e->d_chains, e->d_half_tiles, n, links, parity, img, m->d_params, e->d_sweep, e->d_accepts, m->d_error); break;
        case 1: lp::k_lp_sweep<1><<<grid, lp::kRows, sm, e->stream>>>(e->d_chains, e->d_half_tiles, n, links, parity, img, m->d_params, e->d_sweep, e->d_accepts, m->d_error); break;
        case 2: lp::k_lp_sweep<2><<<grid, lp::kRows, sm, e->stream>>>(e->d_chains, e->d_half_tiles, n, links, parity, img, m->d_params, e->d_sweep, e->d_accepts, m->d_error); break;
        default: lp::k_lp_sweep<3><<<grid, lp::kRows, sm, e->stream>>>(e->d_chains, e->d_half_tiles, n, links, parity, img, m->d_params, e->d_sweep, e->d_accepts, m->d_error); break;
    }
    return cudaGetLastError();
}

}  // namespace ym
