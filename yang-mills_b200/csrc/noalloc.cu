// noalloc.cu -- average plaquette of a caller-owned device lattice without
// any device allocation (compiled with -fmad=false like the FP64 path).
//
// Some callers cannot allocate device memory: a host framework whose memory
// pool owns the whole device and hands the engine only buffers it already
// allocated, or a fixed-footprint deployment that must not call the CUDA
// allocator once it has started.  ym_su3_average_plaquette_noalloc serves
// them: the caller passes the lattice and the output, and the per-tile
// partial sums go to the file-scope array below instead of memory the
// engine would otherwise allocate.
//
// The array is a file-scope __device__ variable: every GPU that loads the
// library holds it (512 KiB) until the process exits.  In host code its name
// is only a host-side stand-in, never a device address, so the launcher
// resolves the real address with cudaGetSymbolAddress once per device (again
// after a device reset, which gives the device a new context), on that
// device's first call, and passes that pointer to the kernels.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "ym_internal.hpp"

namespace {

using namespace ym;

constexpr int kThreads = 128;
// Scratch capacity: one double per 128-site tile -> at most 65536 * 128 =
// 8,388,608 sites (e.g. 48^4 fits, 64^4 does not).
constexpr int64_t kMaxTiles = 65536;

static __device__ __align__(256) double g_plaquette_partials[kMaxTiles];

struct AosGeometry {
    int32_t n[4];
    int64_t volume;
};

// Link (lex, mu) of a lattice in the reference layout: 18 doubles at
// (lex*4 + mu)*18, row-major complex entries.
__device__ __forceinline__ m3 load_aos(const double2 *__restrict__ links, int64_t lex, int mu) {
    const double2 *p = links + (lex * 4 + mu) * 9;
    m3 o;
#pragma unroll
    for (int e = 0; e < 9; ++e) {
        const double2 v = __ldg(p + e);
        o.e[e / 3][e % 3] = cmake(v.x, v.y);
    }
    return o;
}

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double warp_vals[32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) warp_vals[warp] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    if (warp == 0) {
        v = lane < nw ? warp_vals[lane] : 0.0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    }
    return v;
}

// One tile of 128 sites: sum over the tile's sites and mu < nu of
// (1/3) Re Tr U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag, products in the
// reference order (su3_lattice.rs:168-181, su3_ensemble.rs:228-259).
__global__ void __launch_bounds__(kThreads)
k_plaquette_partials(const double2 *__restrict__ links, AosGeometry g, double *partials) {
    const int64_t lex = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    double v = 0.0;
    if (lex < g.volume) {
        int32_t x[4];
        int64_t r = lex;
        x[3] = (int32_t)(r % g.n[3]); r /= g.n[3];
        x[2] = (int32_t)(r % g.n[2]); r /= g.n[2];
        x[1] = (int32_t)(r % g.n[1]);
        x[0] = (int32_t)(r / g.n[1]);
        int64_t stride[4];
        stride[3] = 1;
        stride[2] = g.n[3];
        stride[1] = (int64_t)g.n[2] * g.n[3];
        stride[0] = (int64_t)g.n[1] * g.n[2] * g.n[3];
        bool first = true;
#pragma unroll 1
        for (int mu = 0; mu < 3; ++mu) {
            const int64_t lex_pm = x[mu] == g.n[mu] - 1 ? lex - (int64_t)(g.n[mu] - 1) * stride[mu]
                                                         : lex + stride[mu];
            const m3 umu = load_aos(links, lex, mu);
#pragma unroll 1
            for (int nu = mu + 1; nu < 4; ++nu) {
                const int64_t lex_pn = x[nu] == g.n[nu] - 1
                                           ? lex - (int64_t)(g.n[nu] - 1) * stride[nu]
                                           : lex + stride[nu];
                m3 p = mul(umu, load_aos(links, lex_pm, nu));
                p = mul_adj(p, load_aos(links, lex_pn, mu));
                const double val = retrace_mul_adj(p, load_aos(links, lex, nu)) / 3.0;
                v = first ? val : v + val;
                first = false;
            }
        }
    }
    v = block_sum(v);
    if (threadIdx.x == 0) partials[blockIdx.x] = v;
}

// Fixed-order sum of the n tile partials -> out[0] = sum / (6 V).
__global__ void k_plaquette_final(const double *partials, int64_t n, double volume, double *out) {
    double v = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x)
        v = (i == (int64_t)threadIdx.x) ? partials[i] : v + partials[i];
    v = block_sum(v);
    if (threadIdx.x == 0) out[0] = v / (6.0 * volume);
}

// Driver entry points that name the calling thread's current context.  A
// context's id is unique for the life of the process: after a device reset
// the primary context is a new one, the library's module is loaded into it
// again, and the array has a new device address.
using CtxGetCurrentFn = int (*)(void **ctx);
using CtxGetIdFn = int (*)(void *ctx, unsigned long long *id);

struct ContextIds {
    CtxGetCurrentFn get_current = nullptr;
    CtxGetIdFn get_id = nullptr;
};

const ContextIds &context_ids() {
    static const ContextIds ids = [] {
        ContextIds c;
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            c.get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            c.get_id = reinterpret_cast<CtxGetIdFn>(f);
        return c;
    }();
    return ids;
}

// Id of the current context; false when it cannot be told (no context
// current yet, or the driver lacks the entry points).
bool current_context_id(unsigned long long *id) {
    const ContextIds &c = context_ids();
    if (!c.get_current || !c.get_id) return false;
    void *ctx = nullptr;
    if (c.get_current(&ctx) != 0 || !ctx) return false;
    return c.get_id(ctx, id) == 0;
}

// Device address of g_plaquette_partials in the current context, resolved by
// cudaGetSymbolAddress with the caller's device current the first time a
// context calls, then kept per device together with that context's id.  A
// call from a later context (after a reset) resolves it again; when the
// context cannot be identified every call resolves it.  The table is shared
// by host threads and guarded by a mutex.
struct ResolvedAddress {
    unsigned long long context_id = 0;
    double *ptr = nullptr;
};
std::mutex g_address_mutex;
ResolvedAddress g_address[128];

cudaError_t partials_address(double **out) {
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (dev < 0 || dev >= 128) return cudaErrorInvalidDevice;
    unsigned long long id = 0;
    bool known = current_context_id(&id);
    std::lock_guard<std::mutex> lock(g_address_mutex);
    if (known && g_address[dev].ptr && g_address[dev].context_id == id) {
        *out = g_address[dev].ptr;
        return cudaSuccess;
    }
    void *ptr = nullptr;
    err = cudaGetSymbolAddress(&ptr, g_plaquette_partials);
    if (err != cudaSuccess) return err;
    if (!ptr) return cudaErrorInvalidSymbol;
    known = current_context_id(&id);   // the lookup has made the context current
    g_address[dev] = known ? ResolvedAddress{id, static_cast<double *>(ptr)} : ResolvedAddress{};
    *out = static_cast<double *>(ptr);
    return cudaSuccess;
}

}  // namespace

extern "C" int32_t ym_su3_average_plaquette_noalloc(const double *links, const int64_t *extents,
                                                    double *out, void *stream) {
    if (!links || !extents || !out) return YM_ERR_NULL_ARGUMENT;
    if ((reinterpret_cast<uintptr_t>(links) & 15) != 0) return YM_ERR_INVALID_ARGUMENT;
    AosGeometry g{};
    int64_t sites = 1;
    for (int d = 0; d < 4; ++d)
        if (extents[d] < 2) return YM_ERR_INVALID_LATTICE_EXTENT;
    for (int d = 0; d < 4; ++d) {
        if (extents[d] > (int64_t(1) << 30) || sites > INT64_MAX / extents[d])
            return YM_ERR_LATTICE_SIZE_OVERFLOW;
        sites *= extents[d];
        g.n[d] = (int32_t)extents[d];
    }
    g.volume = sites;
    const int64_t tiles = (sites + kThreads - 1) / kThreads;
    if (tiles > kMaxTiles) return YM_ERR_SCRATCH_TOO_SMALL;
    double *partials = nullptr;
    cudaError_t err = partials_address(&partials);
    if (err != cudaSuccess) return ym::record_cuda_status(err);
    // An error still pending from the caller's earlier work is reported as
    // it is (and left pending) rather than blamed on these launches.
    err = cudaPeekAtLastError();
    if (err != cudaSuccess) return ym::record_cuda_status(err);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_plaquette_partials<<<(unsigned)tiles, kThreads, 0, s>>>(
        reinterpret_cast<const double2 *>(links), g, partials);
    err = cudaGetLastError();
    if (err != cudaSuccess) return ym::record_cuda_status(err);
    k_plaquette_final<<<1, 256, 0, s>>>(partials, tiles, (double)sites, out);
    return ym::record_cuda_status(cudaGetLastError());
}
